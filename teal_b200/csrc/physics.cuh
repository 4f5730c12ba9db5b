// Device-side physics of the teal residual path: primitive/conserved conversion, time-step
// estimates, convective fluxes, viscous flux and boundary conditions for the compressible Euler /
// Navier–Stokes equations. Each function restates the teal routine cited beside it and keeps its
// order of floating-point operations, so FP64 results track teal's CPU results to rounding.
// `R` is the arithmetic type (double for the plain path, float for the FP32-flux form).
#pragma once

#include <cuda_runtime.h>

// Arithmetic of this translation unit. The translation units named *_exact.cu are compiled with
// TG_EXACT_TU=1 and -fmad=false: their FP64 kernels evaluate every expression with teal's own
// operations in teal's order (each quotient a division, no multiply-add contraction), so that with
// IEEE-rounded + - * / sqrt on both sides they reproduce teal's CPU results bit for bit. The other
// translation units share one reciprocal between quotients with the same denominator and let the
// compiler contract multiply-adds, within a few ulps of teal per operation and faster.
#ifndef TG_EXACT_TU
#define TG_EXACT_TU 0
#endif

namespace tg {

constexpr bool kExact = TG_EXACT_TU != 0;

template <typename R>
struct V3 {
    R x, y, z;
};

template <typename R>
__device__ __forceinline__ V3<R> v3(R x, R y, R z)
{
    return V3<R>{x, y, z};
}
template <typename R>
__device__ __forceinline__ V3<R> add(V3<R> a, V3<R> b)
{
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename R>
__device__ __forceinline__ V3<R> sub(V3<R> a, V3<R> b)
{
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename R>
__device__ __forceinline__ V3<R> mul(R s, V3<R> a)
{
    return {s * a.x, s * a.y, s * a.z};
}
template <typename R>
__device__ __forceinline__ V3<R> div(V3<R> a, R s)
{
    return {a.x / s, a.y / s, a.z / s};
}
// (a.x*b.x) + (a.y*b.y) + (a.z*b.z), left to right (src/core/vector.c vector_dot)
template <typename R>
__device__ __forceinline__ R dot(V3<R> a, V3<R> b)
{
    return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z);
}

// face basis: rows x (unit normal), y, z (tangents); row-major as teal's Matrix (src/matrix.h)
template <typename R>
struct Basis {
    V3<R> x, y, z;
};
// basis * v (src/core/matrix.c matrix_vector)
template <typename R>
__device__ __forceinline__ V3<R> to_local(const Basis<R> &b, V3<R> v)
{
    return {dot(b.x, v), dot(b.y, v), dot(b.z, v)};
}
// transpose(basis) * v
template <typename R>
__device__ __forceinline__ V3<R> to_global(const Basis<R> &b, V3<R> v)
{
    return {dot(v3(b.x.x, b.y.x, b.z.x), v), dot(v3(b.x.y, b.y.y, b.z.y), v),
            dot(v3(b.x.z, b.y.z, b.z.z), v)};
}

// Face frame from the unit normal alone: tangents t1, t2 with (n, t1, t2) orthonormal, branch-free
// (Duff, Burgess, Christensen, Hart, Kensler, Liani, Villemin: "Building an Orthonormal Basis,
// Revisited", JCGT 6(1), 2017). The convective fluxes treat the two tangential directions alike and
// linearly (and the kinetic energy is |u|^2), so they are invariant under a rotation or reflection
// of the frame about the normal: any such tangents serve in place of the mesh's stored ones, up to
// rounding, and the plain kernels read only the normal row of the stored basis.
template <typename R>
__device__ __forceinline__ Basis<R> frame_of(V3<R> n)
{
    const R sg = copysign(R(1), n.z);
    const R a = R(-1) / (sg + n.z);
    const R b = (n.x * n.y) * a;
    Basis<R> f;
    f.x = n;
    f.y = v3(R(1) + ((sg * (n.x * n.x)) * a), sg * b, -sg * n.x);
    f.z = v3(b, sg + ((n.y * n.y) * a), -n.y);
    return f;
}

// primitive state: density, velocity, pressure (src/euler.h EulerPrimitive)
template <typename R>
struct Prim {
    R rho;
    V3<R> u;
    R p;
};
// conserved state / flux: density, momentum, energy (src/euler.h EulerConserved)
template <typename R>
struct Cons {
    R rho;
    V3<R> m;
    R e;
};

// conserved -> primitive with the 1e-8 floors (src/euler/create.c:21-32)
template <typename R>
__device__ __forceinline__ Prim<R> cons_to_prim(const Cons<R> &c, R gamma)
{
    Prim<R> q;
    q.rho = fmax(R(1e-8), c.rho);
    if constexpr (kExact) {
        q.u = div(c.m, q.rho);
    }
    else {
        q.u = mul(R(1) / q.rho, c.m);  // one reciprocal for the three velocities
    }
    q.p = fmax(R(1e-8), (gamma - R(1)) * (c.e - (dot(c.m, q.u) / R(2))));
    return q;
}

// a product the compiler may not fuse into a following addition: the same bits in every kernel
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// primitive -> conserved (src/euler/create.c:34-44); several kernels form U0 with it (the step's
// last stage, the preparation of a loaded state), which must agree bit for bit
template <typename R>
__device__ __forceinline__ Cons<R> prim_to_cons(const Prim<R> &q, R gamma)
{
    Cons<R> c;
    c.rho = q.rho;
    c.m = mul(c.rho, q.u);
    if constexpr (kExact) {
        c.e = (q.p / (gamma - R(1))) + (dot(c.m, q.u) / R(2));
    }
    else {
        c.e = mul_rn(q.p, R(1) / (gamma - R(1))) + (dot(c.m, q.u) / R(2));
    }
    return c;
}

// maximum stable step of one cell (src/euler/create.c:6-19)
template <typename R>
__device__ __forceinline__ R euler_timestep(const Prim<R> &q, R gamma, R volume, V3<R> proj)
{
    R a = sqrt(gamma * q.p / q.rho);
    R lx = (fabs(q.u.x) + a) * proj.x;
    R ly = (fabs(q.u.y) + a) * proj.y;
    R lz = (fabs(q.u.z) + a) * proj.z;
    return volume / ((lx + ly) + lz);
}

// with the viscous term (src/navierstokes/create.c:7-26)
template <typename R>
__device__ __forceinline__ R navierstokes_timestep(const Prim<R> &q, R gamma, R mu, R prandtl,
                                                   R volume, V3<R> proj)
{
    R a = sqrt(gamma * q.p / q.rho);
    R lx = (fabs(q.u.x) + a) * proj.x;
    R ly = (fabs(q.u.y) + a) * proj.y;
    R lz = (fabs(q.u.z) + a) * proj.z;
    R lv = fmax(R(4) * mu / (R(3) * q.rho), gamma * mu / (q.rho * prandtl));
    return volume / (((lx + ly) + lz) + (R(4) * lv * dot(proj, proj) / volume));
}

// ---- convective fluxes (src/euler/convective.c) ------------------------------------------------

// state in the face frame (convective.c:7-25 `Euler`, global_to_local)
// FP32 fluxes: pressure and energy relative to a reference pressure p_ref, dp = p - p_ref and
// de = dp / (gamma - 1) + rho |u|^2 / 2. The normal momentum flux carries dp and the state jumps use
// de, which shifts every face's momentum flux by the constant -p_ref n A; that cancels over each
// closed cell in exact arithmetic, while FP32 no longer rounds p_ref (~1/(gamma Ma^2)) into the
// cancelling fluxes (the FP32-flux form of low-Mach flows). FP64 fluxes use p and e themselves.
template <typename R>
struct LocalRel {
    R dp;
    R de;
};
template <>
struct LocalRel<double> {
};

template <typename R>
struct Local : LocalRel<R> {
    R rho;
    V3<R> u;
    R p;
    V3<R> m;
    R e;
};

// g.p is the pressure relative to pref (FP32-flux form) or the pressure itself (pref = 0)
template <typename R>
__device__ __forceinline__ Local<R> make_local(const Prim<R> &g, R gamma, const Basis<R> &b, R pref = R(0))
{
    Local<R> s;
    s.rho = g.rho;
    s.u = to_local(b, g.u);
    if constexpr (sizeof(R) == sizeof(double)) {  // FP64: no reference pressure
        (void)pref;
        s.p = g.p;
        s.m = mul(s.rho, s.u);
        if constexpr (kExact) {
            s.e = (s.p / (gamma - R(1))) + (dot(s.m, s.u) / R(2));
        }
        else {
            s.e = (s.p * (R(1) / (gamma - R(1)))) + (dot(s.m, s.u) / R(2));
        }
    }
    else {
        s.dp = g.p;
        s.p = g.p + pref;
        s.m = mul(s.rho, s.u);
        const R kinetic = dot(s.m, s.u) / R(2);
        s.e = (s.p * (R(1) / (gamma - R(1)))) + kinetic;
        s.de = (s.dp * (R(1) / (gamma - R(1)))) + kinetic;
    }
    return s;
}

// physical flux normal to the face (convective.c:32-41)
template <typename R>
__device__ __forceinline__ Cons<R> physical_flux(const Local<R> &s)
{
    Cons<R> f;
    f.rho = s.m.x;
    if constexpr (sizeof(R) == sizeof(double)) {
        f.m.x = (s.m.x * s.u.x) + s.p;
    }
    else {
        f.m.x = (s.m.x * s.u.x) + s.dp;
    }
    f.m.y = s.m.x * s.u.y;
    f.m.z = s.m.x * s.u.z;
    f.e = (s.e + s.p) * s.u.x;
    return f;
}

template <typename R>
__device__ __forceinline__ Cons<R> jump_of(const Local<R> &l, const Local<R> &r)
{
    Cons<R> j;
    j.rho = r.rho - l.rho;
    j.m = sub(r.m, l.m);
    if constexpr (sizeof(R) == sizeof(double)) {
        j.e = r.e - l.e;
    }
    else {
        j.e = r.de - l.de;
    }
    return j;
}

// Roe-averaged velocity (convective.c:64-69)
template <typename R>
__device__ __forceinline__ V3<R> roe_velocity(R w, R sl, R sr, const Local<R> &l, const Local<R> &r)
{
    return mul(w, add(mul(sl, l.u), mul(sr, r.u)));
}

// Roe with Harten–Hyman entropy fix (convective.c:71-213)
template <typename R>
__device__ __forceinline__ Cons<R> flux_roe(const Local<R> &l, const Local<R> &r, R gamma)
{
    R gm1 = gamma - R(1);
    const R il = R(1) / l.rho, ir = R(1) / r.rho;
    R hl = kExact ? ((l.e + l.p) / l.rho) : ((l.e + l.p) * il);
    R hr = kExact ? ((r.e + r.p) / r.rho) : ((r.e + r.p) * ir);
    R sl = sqrt(l.rho);
    R sr = sqrt(r.rho);
    R w = R(1) / (sl + sr);
    V3<R> u = roe_velocity(w, sl, sr, l, r);
    R h = w * ((sl * hl) + (sr * hr));
    R u2 = dot(u, u);
    R a2 = gm1 * (h - (u2 / R(2)));
    R a = sqrt(a2);

    R eig[3] = {u.x - a, u.x, u.x + a};
    {
        R al = kExact ? sqrt((gamma * l.p) / l.rho) : sqrt((gamma * l.p) * il);
        R ar = kExact ? sqrt((gamma * r.p) / r.rho) : sqrt((gamma * r.p) * ir);
        R el[3] = {l.u.x - al, l.u.x, l.u.x + al};
        R er[3] = {r.u.x - ar, r.u.x, r.u.x + ar};
#pragma unroll
        for (int i = 0; i < 3; i++) {
            R lam = eig[i];
            R delta = fmax(R(0), fmax(lam - el[i], er[i] - lam));
            eig[i] = (fabs(lam) < delta) ? delta : fabs(lam);
        }
    }

    Cons<R> j = jump_of(l, r);
    R ws[5];
    ws[2] = j.m.y - (u.y * j.rho);
    ws[3] = j.m.z - (u.z * j.rho);
    const R jw = ((((j.rho * (h - (u.x * u.x))) + (u.x * j.m.x)) - j.e) + (ws[2] * u.y)) + (ws[3] * u.z);
    if constexpr (kExact) {
        ws[1] = (gm1 / a2) * jw;
        ws[0] = (((j.rho * (u.x + a)) - j.m.x) - (a * ws[1])) / (R(2) * a);
    }
    else {
        const R ia = R(1) / a;  // one reciprocal for the two quotients by a and a^2
        ws[1] = (gm1 * (ia * ia)) * jw;
        ws[0] = (((j.rho * (u.x + a)) - j.m.x) - (a * ws[1])) * (ia / R(2));
    }
    ws[4] = j.rho - (ws[0] + ws[1]);

    R ch[5] = {ws[0] * eig[0], ws[1] * eig[1], ws[2] * eig[1], ws[3] * eig[1], ws[4] * eig[2]};
    // dissipation = eigenvector matrix * characteristic, rows as in convective.c:151-197, summed
    // in column order; the matrix's zero entries add exact zeros for finite values and are left out
    R d0 = (ch[0] + ch[1]) + ch[4];
    R d1 = (((u.x - a) * ch[0]) + (u.x * ch[1])) + ((u.x + a) * ch[4]);
    R d2 = (((u.y * ch[0]) + (u.y * ch[1])) + ch[2]) + (u.y * ch[4]);
    R d3 = (((u.z * ch[0]) + (u.z * ch[1])) + ch[3]) + (u.z * ch[4]);
    R d4 = (((((h - (u.x * a)) * ch[0]) + ((u2 / R(2)) * ch[1])) + (u.y * ch[2])) + (u.z * ch[3])) +
           ((h + (u.x * a)) * ch[4]);

    Cons<R> fl = physical_flux(l);
    Cons<R> fr = physical_flux(r);
    Cons<R> f;
    f.rho = ((fl.rho + fr.rho) - d0) / R(2);
    f.m.x = ((fl.m.x + fr.m.x) - d1) / R(2);
    f.m.y = ((fl.m.y + fr.m.y) - d2) / R(2);
    f.m.z = ((fl.m.z + fr.m.z) - d3) / R(2);
    f.e = ((fl.e + fr.e) - d4) / R(2);
    return f;
}

// HLL average of the two physical fluxes (convective.c:215-243)
template <typename R>
__device__ __forceinline__ Cons<R> hll_average(const Local<R> &l, const Local<R> &r, R sl, R sr)
{
    Cons<R> fl = physical_flux(l);
    fl.rho *= sr;
    fl.m = mul(sr, fl.m);
    fl.e *= sr;
    Cons<R> fr = physical_flux(r);
    fr.rho *= sl;
    fr.m = mul(sl, fr.m);
    fr.e *= sl;
    R sj = sl * sr;
    Cons<R> j = jump_of(l, r);
    j.rho *= sj;
    j.m = mul(sj, j.m);
    j.e *= sj;
    R factor = R(1) / (sr - sl);
    Cons<R> f;
    f.rho = factor * ((fl.rho - fr.rho) + j.rho);
    f.m = mul(factor, add(sub(fl.m, fr.m), j.m));
    f.e = factor * ((fl.e - fr.e) + j.e);
    return f;
}

// Roe-average signal speeds shared by hll and hllc (convective.c:252-272, :307-327)
template <typename R>
__device__ __forceinline__ void einfeldt_speeds(const Local<R> &l, const Local<R> &r, R gamma,
                                                R &sl_out, R &sr_out)
{
    const R il = R(1) / l.rho, ir = R(1) / r.rho;
    R hl = kExact ? ((l.e + l.p) / l.rho) : ((l.e + l.p) * il);
    R hr = kExact ? ((r.e + r.p) / r.rho) : ((r.e + r.p) * ir);
    R sl = sqrt(l.rho);
    R sr = sqrt(r.rho);
    R w = R(1) / (sl + sr);
    V3<R> u = roe_velocity(w, sl, sr, l, r);
    R h = w * ((sl * hl) + (sr * hr));
    R u2 = dot(u, u);
    R a = sqrt((gamma - R(1)) * (h - (u2 / R(2))));
    R al = kExact ? sqrt((gamma * l.p) / l.rho) : sqrt((gamma * l.p) * il);
    R ar = kExact ? sqrt((gamma * r.p) / r.rho) : sqrt((gamma * r.p) * ir);
    sl_out = fmin(l.u.x - al, u.x - a);
    sr_out = fmax(r.u.x + ar, u.x + a);
}

template <typename R>
__device__ __forceinline__ Cons<R> flux_hll(const Local<R> &l, const Local<R> &r, R gamma)
{
    R sl, sr;
    einfeldt_speeds(l, r, gamma, sl, sr);
    if (sl >= R(0)) {
        return physical_flux(l);
    }
    if (sr <= R(0)) {
        return physical_flux(r);
    }
    return hll_average(l, r, sl, sr);
}

// star-state flux of HLLC (convective.c:276-298)
template <typename R>
__device__ __forceinline__ Cons<R> contact_flux(const Local<R> &k, R sk, R fk, R s)
{
    R factor = fk / (sk - s);
    Cons<R> star;
    star.rho = factor;
    star.m.x = factor * s;
    star.m.y = factor * k.u.y;
    star.m.z = factor * k.u.z;
    star.e = factor * ((k.e / k.rho) + ((s - k.u.x) * (s + (k.p / fk))));
    Cons<R> f = physical_flux(k);
    f.rho += sk * (star.rho - k.rho);
    f.m = add(f.m, mul(sk, sub(star.m, k.m)));
    f.e += sk * (star.e - k.e);
    return f;
}

// HLLC (convective.c:300-346)
template <typename R>
__device__ __forceinline__ Cons<R> flux_hllc(const Local<R> &l, const Local<R> &r, R gamma)
{
    R sl, sr;
    einfeldt_speeds(l, r, gamma, sl, sr);
    if (sl >= R(0)) {
        return physical_flux(l);
    }
    if (sr <= R(0)) {
        return physical_flux(r);
    }
    R fl = l.rho * (sl - l.u.x);
    R fr = r.rho * (sr - r.u.x);
    R s = (((r.p - l.p) + (fl * l.u.x)) - (fr * r.u.x)) / (fl - fr);
    if (sl <= R(0) && R(0) <= s) {
        return contact_flux(l, sl, fl, s);
    }
    return contact_flux(r, sr, fr, s);
}

// HLLE with Einfeldt's averaged sound speed (convective.c:348-389)
template <typename R>
__device__ __forceinline__ Cons<R> flux_hlle(const Local<R> &l, const Local<R> &r, R gamma)
{
    R sl = sqrt(l.rho);
    R sr = sqrt(r.rho);
    R w = R(1) / (sl + sr);
    R ux = w * ((sl * l.u.x) + (sr * r.u.x));
    R a2l = kExact ? ((gamma * l.p) / l.rho) : ((gamma * l.p) * (R(1) / l.rho));
    R a2r = kExact ? ((gamma * r.p) / r.rho) : ((gamma * r.p) * (R(1) / r.rho));
    R al = sqrt(a2l);
    R ar = sqrt(a2r);
    R a2 = w * ((sl * a2l) + (sr * a2r));
    R du = r.u.x - l.u.x;
    R vj = (w * w) * sl * sr * (du * du) / R(2);
    R a = sqrt(a2 + vj);
    R s_l = fmin(l.u.x - al, ux - a);
    R s_r = fmax(r.u.x + ar, ux + a);
    if (s_l >= R(0)) {
        return physical_flux(l);
    }
    if (s_r <= R(0)) {
        return physical_flux(r);
    }
    return hll_average(l, r, s_l, s_r);
}

// split velocity / pressure of AUSM-D and AUSM-DV for the left (+) and right (-) state
// (convective.c:391-431 and :463-503). `dv` selects the AUSM-DV form of the supersonic pressure.
template <typename R, bool DV>
__device__ __forceinline__ void ausm_split(const Local<R> &l, const Local<R> &r, R gamma, R &vpl,
                                           R &ppl, R &vmr, R &pmr)
{
    if constexpr (kExact) {  // teal's quotients, term by term
        R al = sqrt((gamma * l.p) / l.rho);
        R ar = sqrt((gamma * r.p) / r.rho);
        R a = fmax(al, ar);
        R pdl = l.p / l.rho;
        R pdr = r.p / r.rho;
        R pds = pdl + pdr;
        R ml = l.u.x / a;
        R mr = r.u.x / a;
        if (fabs(l.u.x) <= a) {
            R alpha = (R(2) * pdl) / pds;
            R f = l.u.x + a;
            vpl = ((alpha * (f * f)) / (R(4) * a)) + (((R(1) - alpha) * (l.u.x + fabs(l.u.x))) / R(2));
            ppl = ((l.p * (f * f)) / (R(4) * (a * a))) * (R(2) - ml);
        }
        else {
            vpl = (l.u.x + fabs(l.u.x)) / R(2);
            ppl = DV ? ((l.p * (l.u.x + fabs(l.u.x))) / (R(2) * l.u.x))
                     : (((l.p * (l.u.x + fabs(l.u.x))) / R(2)) / l.u.x);
        }
        if (fabs(r.u.x) <= a) {
            R alpha = (R(2) * pdr) / pds;
            R f = r.u.x - a;
            vmr = ((-alpha * (f * f)) / (R(4) * a)) + (((R(1) - alpha) * (r.u.x - fabs(r.u.x))) / R(2));
            pmr = ((r.p * (f * f)) / (R(4) * (a * a))) * (R(2) + mr);
        }
        else {
            vmr = (r.u.x - fabs(r.u.x)) / R(2);
            pmr = DV ? ((r.p * (r.u.x - fabs(r.u.x))) / (R(2) * r.u.x))
                     : (((r.p * (r.u.x - fabs(r.u.x))) / R(2)) / r.u.x);
        }
        return;
    }
    const R il = R(1) / l.rho, ir = R(1) / r.rho;
    R al = sqrt((gamma * l.p) * il);
    R ar = sqrt((gamma * r.p) * ir);
    R a = fmax(al, ar);
    const R ia = R(1) / a;
    R pdl = l.p * il;
    R pdr = r.p * ir;
    R pds = pdl + pdr;
    const R ips = R(1) / pds;
    R ml = l.u.x * ia;
    R mr = r.u.x * ia;
    if (fabs(l.u.x) <= a) {
        R alpha = (R(2) * pdl) * ips;
        R f = l.u.x + a;
        vpl = ((alpha * (f * f)) * (ia / R(4))) + (((R(1) - alpha) * (l.u.x + fabs(l.u.x))) / R(2));
        ppl = ((l.p * (f * f)) * ((ia * ia) / R(4))) * (R(2) - ml);
    }
    else {
        vpl = (l.u.x + fabs(l.u.x)) / R(2);
        ppl = DV ? ((l.p * (l.u.x + fabs(l.u.x))) / (R(2) * l.u.x))
                 : (((l.p * (l.u.x + fabs(l.u.x))) / R(2)) / l.u.x);
    }
    if (fabs(r.u.x) <= a) {
        R alpha = (R(2) * pdr) * ips;
        R f = r.u.x - a;
        vmr = ((-alpha * (f * f)) * (ia / R(4))) + (((R(1) - alpha) * (r.u.x - fabs(r.u.x))) / R(2));
        pmr = ((r.p * (f * f)) * ((ia * ia) / R(4))) * (R(2) + mr);
    }
    else {
        vmr = (r.u.x - fabs(r.u.x)) / R(2);
        pmr = DV ? ((r.p * (r.u.x - fabs(r.u.x))) / (R(2) * r.u.x))
                 : (((r.p * (r.u.x - fabs(r.u.x))) / R(2)) / r.u.x);
    }
}

// AUSM-D (convective.c:391-461)
template <typename R>
__device__ __forceinline__ Cons<R> flux_ausmd(const Local<R> &l, const Local<R> &r, R gamma)
{
    R vpl, ppl, vmr, pmr;
    ausm_split<R, false>(l, r, gamma, vpl, ppl, vmr, pmr);
    R mf = (vpl * l.rho) + (vmr * r.rho);
    R amf = fabs(mf);
    R pf = ppl + pmr;
    R hl = kExact ? ((l.e + l.p) / l.rho) : ((l.e + l.p) * (R(1) / l.rho));
    R hr = kExact ? ((r.e + r.p) / r.rho) : ((r.e + r.p) * (R(1) / r.rho));
    Cons<R> f;
    f.rho = mf;
    f.m.x = (((mf * (l.u.x + r.u.x)) - (amf * (r.u.x - l.u.x))) / R(2)) + pf;
    f.m.y = ((mf * (l.u.y + r.u.y)) - (amf * (r.u.y - l.u.y))) / R(2);
    f.m.z = ((mf * (l.u.z + r.u.z)) - (amf * (r.u.z - l.u.z))) / R(2);
    f.e = ((mf * (hl + hr)) - (amf * (hr - hl))) / R(2);
    return f;
}

// AUSM-DV (convective.c:463-547)
template <typename R>
__device__ __forceinline__ Cons<R> flux_ausmdv(const Local<R> &l, const Local<R> &r, R gamma)
{
    R vpl, ppl, vmr, pmr;
    ausm_split<R, true>(l, r, gamma, vpl, ppl, vmr, pmr);
    R mf = (vpl * l.rho) + (vmr * r.rho);
    R amf = fabs(mf);
    R pf = ppl + pmr;
    R nd = ((mf * (l.u.x + r.u.x)) - (amf * (r.u.x - l.u.x))) / R(2);
    R nv = (vpl * l.m.x) + (vmr * r.m.x);
    R pmin = fmin(l.p, r.p);
    R sw = fmin(R(1) / R(2), fmin(R(1), (R(10) * fabs(r.p - l.p)) / pmin));
    R nm = (((R(1) + sw) * nv) + ((R(1) - sw) * nd)) / R(2);
    R hl = kExact ? ((l.e + l.p) / l.rho) : ((l.e + l.p) * (R(1) / l.rho));
    R hr = kExact ? ((r.e + r.p) / r.rho) : ((r.e + r.p) * (R(1) / r.rho));
    Cons<R> f;
    f.rho = mf;
    f.m.x = nm + pf;
    f.m.y = ((mf * (l.u.y + r.u.y)) - (amf * (r.u.y - l.u.y))) / R(2);
    f.m.z = ((mf * (l.u.z + r.u.z)) - (amf * (r.u.z - l.u.z))) / R(2);
    f.e = ((mf * (hl + hr)) - (amf * (hr - hl))) / R(2);
    return f;
}

// Lax–Friedrichs (Rusanov) (convective.c:549-574)
template <typename R>
__device__ __forceinline__ Cons<R> flux_lxf(const Local<R> &l, const Local<R> &r, R gamma)
{
    R al = sqrt(gamma * l.p / l.rho);
    R ar = sqrt(gamma * r.p / r.rho);
    R s = fmax(fabs(l.u.x) + al, fabs(r.u.x) + ar);
    Cons<R> j = jump_of(l, r);
    j.rho *= s;
    j.m = mul(s, j.m);
    j.e *= s;
    Cons<R> fl = physical_flux(l);
    Cons<R> fr = physical_flux(r);
    Cons<R> f;
    f.rho = ((fl.rho + fr.rho) - j.rho) / R(2);
    f.m = div(sub(add(fl.m, fr.m), j.m), R(2));
    f.e = ((fl.e + fr.e) - j.e) / R(2);
    return f;
}

// central average (convective.c:576-591)
template <typename R>
__device__ __forceinline__ Cons<R> flux_central(const Local<R> &l, const Local<R> &r)
{
    Cons<R> fl = physical_flux(l);
    Cons<R> fr = physical_flux(r);
    Cons<R> f;
    f.rho = (fl.rho + fr.rho) / R(2);
    f.m = div(add(fl.m, fr.m), R(2));
    f.e = (fl.e + fr.e) / R(2);
    return f;
}

// Flux kinds as in the public enum (TG_FLUX_*).
enum FluxKind { FK_NONE = 0, FK_ROE, FK_HLL, FK_HLLC, FK_HLLE, FK_AUSMD, FK_AUSMDV, FK_LXF, FK_CENTRAL };

// Numerical flux in the face frame between two face-frame states.
template <int FK, typename R>
__device__ __forceinline__ Cons<R> convective_flux_local(const Local<R> &l, const Local<R> &r, R gamma)
{
    Cons<R> f;
    if constexpr (FK == FK_ROE) {
        f = flux_roe(l, r, gamma);
    }
    else if constexpr (FK == FK_HLL) {
        f = flux_hll(l, r, gamma);
    }
    else if constexpr (FK == FK_HLLC) {
        f = flux_hllc(l, r, gamma);
    }
    else if constexpr (FK == FK_HLLE) {
        f = flux_hlle(l, r, gamma);
    }
    else if constexpr (FK == FK_AUSMD) {
        f = flux_ausmd(l, r, gamma);
    }
    else if constexpr (FK == FK_AUSMDV) {
        f = flux_ausmdv(l, r, gamma);
    }
    else if constexpr (FK == FK_LXF) {
        f = flux_lxf(l, r, gamma);
    }
    else {
        f = flux_central(l, r);
    }
    return f;
}

// Numerical flux in global coordinates between two primitive states (the `Convective` plugin).
template <int FK, typename R>
__device__ __forceinline__ Cons<R> convective_flux(const Prim<R> &pl, const Prim<R> &pr, R gamma,
                                                   const Basis<R> &b)
{
    Cons<R> f = convective_flux_local<FK>(make_local(pl, gamma, b), make_local(pr, gamma, b), gamma);
    f.m = to_global(b, f.m);
    return f;
}

// ---- viscous flux (src/navierstokes/viscous.c:11-39) -------------------------------------------

// gradient of the primitive variables: d(rho), d(u) rows (du_x, du_y, du_z) x (d/dx, d/dy, d/dz),
// d(p); teal's `Gradient` (viscous.c:5-9) is the same 15 doubles in this order
template <typename R>
struct Grad {
    V3<R> rho;
    V3<R> ux, uy, uz;
    V3<R> p;
};

template <typename R>
__device__ __forceinline__ Cons<R> viscous_central(const Prim<R> &q, const Grad<R> &g, R gamma,
                                                   R mu, R prandtl, const Basis<R> &b)
{
    R div_u = (g.ux.x + g.uy.y) + g.uz.z;
    const R div3 = kExact ? (div_u / R(3)) : (div_u * (R(1) / R(3)));
    R txx = R(2) * mu * (g.ux.x - div3);
    R tyy = R(2) * mu * (g.uy.y - div3);
    R tzz = R(2) * mu * (g.uz.z - div3);
    R txy = mu * (g.ux.y + g.uy.x);
    R txz = mu * (g.ux.z + g.uz.x);
    R tyz = mu * (g.uy.z + g.uz.y);
    V3<R> tx = v3(txx, txy, txz);
    V3<R> ty = v3(txy, tyy, tyz);
    V3<R> tz = v3(txz, tyz, tzz);

    R factor = -mu * gamma / ((gamma - R(1)) * prandtl * (q.rho * q.rho));
    V3<R> heat = mul(factor, sub(mul(q.rho, g.p), mul(q.p, g.rho)));
    V3<R> tu = v3(dot(tx, q.u), dot(ty, q.u), dot(tz, q.u));
    V3<R> theta = sub(tu, heat);

    Cons<R> f;
    f.rho = R(0);
    f.m = v3(dot(tx, b.x), dot(ty, b.x), dot(tz, b.x));
    f.e = dot(theta, b.x);
    return f;
}

// ---- boundary conditions (src/euler/boundary.c, src/navierstokes/boundary.c) --------------------

enum BcKind {
    BC_NONE = 0,
    BC_SYMMETRY = 1,
    BC_SUPERSONIC_INFLOW = 2,
    BC_SUPERSONIC_OUTFLOW = 3,
    BC_SUBSONIC_INFLOW = 4,
    BC_SUBSONIC_OUTFLOW = 5,
    BC_PRESSURE_OUTFLOW = 6,
    BC_FARFIELD = 7,
    BC_ADIABATIC_WALL = 8,
    BC_CUSTOM = 9  // a device function writes the ghost rows
};

// characteristic far-field state (boundary.c:134-271)
template <typename R>
__device__ __forceinline__ Prim<R> bc_farfield(const Prim<R> &inner_g, const Prim<R> &ctx, R gamma,
                                               const Basis<R> &b)
{
    Local<R> o = make_local(ctx, gamma, b);
    Local<R> in = make_local(inner_g, gamma, b);
    R gm1 = gamma - R(1);
    R u2 = dot(in.u, in.u);
    R a2 = gamma * in.p / in.rho;
    R a = sqrt(a2);
    R h = (u2 / R(2)) + (a2 / gm1);
    R ux = in.u.x, uy = in.u.y, uz = in.u.z;

    R li[5][5] = {
        {h + ((a / gm1) * (ux - a)), -(ux + (a / gm1)), -uy, -uz, R(1)},
        {(R(-2) * h) + ((R(4) / gm1) * a2), R(2) * ux, R(2) * uy, R(2) * uz, R(-2)},
        {((R(-2) * uy) * a2) / gm1, R(0), (R(2) * a2) / gm1, R(0), R(0)},
        {((R(-2) * uz) * a2) / gm1, R(0), R(0), (R(2) * a2) / gm1, R(0)},
        {h - ((a / gm1) * (ux + a)), -ux + (a / gm1), -uy, -uz, R(1)},
    };
    R factor = gm1 / (R(2) * a2);
    R ci_[5] = {in.rho, in.m.x, in.m.y, in.m.z, in.e};
    R cg_[5] = {o.rho, o.m.x, o.m.y, o.m.z, o.e};
    R chi[5], chg[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        R si = R(0), sg = R(0);
#pragma unroll
        for (int j = 0; j < 5; j++) {
            si += li[i][j] * ci_[j];
            sg += li[i][j] * cg_[j];
        }
        chi[i] = si * factor;
        chg[i] = sg * factor;
    }
    R ag = sqrt(gamma * o.p / o.rho);
    if (o.u.x - ag > R(0)) {
        chg[0] = chi[0];
    }
    if (o.u.x > R(0)) {
        chg[1] = chi[1];
        chg[2] = chi[2];
        chg[3] = chi[3];
    }
    if (o.u.x + ag > R(0)) {
        chg[4] = chi[4];
    }
    R ev[5][5] = {
        {R(1), R(1), R(0), R(0), R(1)},
        {ux - a, ux, R(0), R(0), ux + a},
        {uy, uy, R(1), R(0), uy},
        {uz, uz, R(0), R(1), uz},
        {h - (ux * a), u2 / R(2), uy, uz, h + (ux * a)},
    };
    R cg[5];
#pragma unroll
    for (int i = 0; i < 5; i++) {
        R s = R(0);
#pragma unroll
        for (int j = 0; j < 5; j++) {
            s += ev[i][j] * chg[j];
        }
        cg[i] = s;
    }
    // back to primitive in global coordinates (boundary.c:118-127)
    V3<R> m = v3(cg[1], cg[2], cg[3]);
    V3<R> ul = div(m, cg[0]);
    R p = gm1 * (cg[4] - (dot(m, ul) / R(2)));
    Prim<R> out;
    out.rho = fmax(R(1e-8), cg[0]);
    out.u = to_global(b, ul);
    out.p = fmax(R(1e-8), p);
    return out;
}

// ghost (outer) primitive state from the inner state (the `Boundary` plugin)
template <typename R>
__device__ __forceinline__ Prim<R> boundary_state(int kind, const Prim<R> &in, const Prim<R> &ctx,
                                                  R gamma, const Basis<R> &b)
{
    Prim<R> o;
    switch (kind) {
        case BC_SYMMETRY: {  // boundary.c:7-21
            R un = dot(in.u, b.x);
            o.rho = in.rho;
            o.u = sub(in.u, mul(R(2) * un, b.x));
            o.p = in.p;
            return o;
        }
        case BC_SUPERSONIC_INFLOW:  // boundary.c:23-34
            return ctx;
        case BC_SUPERSONIC_OUTFLOW:  // boundary.c:36-47
            return in;
        case BC_SUBSONIC_INFLOW: {  // boundary.c:49-70
            R rho = in.rho;
            R a2 = gamma * in.p / in.rho;
            R a = sqrt(a2);
            R un = dot(sub(ctx.u, in.u), b.x);
            R f1 = rho * a;
            o.p = ((ctx.p + in.p) - (f1 * un)) / R(2);
            o.rho = ctx.rho + ((o.p - ctx.p) / a2);
            R f2 = (ctx.p - o.p) / f1;
            o.u = sub(ctx.u, mul(f2, b.x));
            return o;
        }
        case BC_SUBSONIC_OUTFLOW: {  // boundary.c:72-89
            R rho = in.rho;
            R a2 = gamma * in.p / in.rho;
            R a = sqrt(a2);
            o.p = ctx.p;
            o.rho = in.rho + ((o.p - in.p) / a2);
            R f = (in.p - o.p) / (rho * a);
            o.u = sub(in.u, mul(f, b.x));
            return o;
        }
        case BC_PRESSURE_OUTFLOW: {  // boundary.c:91-106
            R a = sqrt(gamma * in.p / in.rho);
            R un = dot(in.u, b.x);
            R p = (un / a < R(1)) ? ctx.p : in.p;
            o.rho = in.rho * p / in.p;
            o.u = in.u;
            o.p = p;
            return o;
        }
        case BC_FARFIELD:
            return bc_farfield(in, ctx, gamma, b);
        case BC_ADIABATIC_WALL:  // navierstokes/boundary.c:6-18
            o.rho = in.rho;
            o.u = mul(R(-1), in.u);
            o.p = in.p;
            return o;
        default:
            return in;
    }
}

}  // namespace tg
