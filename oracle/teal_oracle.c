/*
 * CPU restatement of teal's residual / time-integration path — TEST INFRASTRUCTURE ONLY (the
 * oracle). Each function states the reference routine it follows (paths inside the teal tree) and
 * keeps its loop order and floating-point evaluation order, so with ISO C (no contraction) it
 * reproduces the reference bit for bit; tests pin it against oracle/_ref and tests/golden.
 */
#include "teal_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double x, y, z;
} V;

static V vadd(V a, V b) { return (V){a.x + b.x, a.y + b.y, a.z + b.z}; }
static V vsub(V a, V b) { return (V){a.x - b.x, a.y - b.y, a.z - b.z}; }
static V vmul(double s, V a) { return (V){s * a.x, s * a.y, s * a.z}; }
static V vdiv(V a, double s) { return (V){a.x / s, a.y / s, a.z / s}; }
static double vdot(V a, V b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }

typedef struct {
    V x, y, z;
} M;

static V mv(M m, V v) { return (V){vdot(m.x, v), vdot(m.y, v), vdot(m.z, v)}; }
static M mt(M m)
{
    return (M){{m.x.x, m.y.x, m.z.x}, {m.x.y, m.y.y, m.z.y}, {m.x.z, m.y.z, m.z.z}};
}

static int is_close(double a, double b) /* src/core/utils.c:29-34 */
{
    return islessequal(fabs(a - b), fmax(1e-8, 1e-5 * fmax(fabs(a), fabs(b))));
}

typedef struct {
    double rho;
    V u;
    double p;
} P; /* EulerPrimitive */
typedef struct {
    double rho;
    V m;
    double e;
} U; /* EulerConserved */

static P getp(const double *a) { return (P){a[0], {a[1], a[2], a[3]}, a[4]}; }
static void putp(double *a, P p)
{
    a[0] = p.rho, a[1] = p.u.x, a[2] = p.u.y, a[3] = p.u.z, a[4] = p.p;
}
static M basis_of(const tg_mesh *m, int f)
{
    const double *b = m->face_basis + 9 * (size_t)f;
    return (M){{b[0], b[1], b[2]}, {b[3], b[4], b[5]}, {b[6], b[7], b[8]}};
}
static V vec_at(const double *a, size_t i) { return (V){a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

/* ---- src/euler/create.c:6-44 -------------------------------------------------------------------- */

static double euler_timestep(P q, double gamma, double volume, V proj)
{
    double a = sqrt(gamma * q.p / q.rho);
    double lx = (fabs(q.u.x) + a) * proj.x;
    double ly = (fabs(q.u.y) + a) * proj.y;
    double lz = (fabs(q.u.z) + a) * proj.z;
    return volume / (lx + ly + lz);
}

static double navierstokes_timestep(P q, const double *prop, double volume, V proj) /* ns/create.c:7-26 */
{
    double gamma = prop[0], mu = prop[1], pr = prop[2];
    double a = sqrt(gamma * q.p / q.rho);
    double lx = (fabs(q.u.x) + a) * proj.x;
    double ly = (fabs(q.u.y) + a) * proj.y;
    double lz = (fabs(q.u.z) + a) * proj.z;
    double lv = fmax(4 * mu / (3 * q.rho), gamma * mu / (q.rho * pr));
    return volume / (lx + ly + lz + (4 * lv * vdot(proj, proj) / volume));
}

static P to_prim(U c, double gamma)
{
    P q;
    q.rho = fmax(1e-8, c.rho);
    q.u = vdiv(c.m, q.rho);
    q.p = fmax(1e-8, (gamma - 1) * (c.e - (vdot(c.m, q.u) / 2)));
    return q;
}

static U to_cons(P q, double gamma)
{
    U c;
    c.rho = q.rho;
    c.m = vmul(c.rho, q.u);
    c.e = (q.p / (gamma - 1)) + (vdot(c.m, q.u) / 2);
    return c;
}

/* ---- convective fluxes (src/euler/convective.c) --------------------------------------------------- */

typedef struct {
    double rho;
    V u;
    double p;
    V m;
    double e;
} L;

static L local(P g, double gamma, M b) /* convective.c:15-25 */
{
    L s;
    s.rho = g.rho;
    s.u = mv(b, g.u);
    s.p = g.p;
    s.m = vmul(s.rho, s.u);
    s.e = (s.p / (gamma - 1)) + (vdot(s.m, s.u) / 2);
    return s;
}

static U phys(L s) /* convective.c:32-41 */
{
    U f;
    f.rho = s.m.x;
    f.m.x = (s.m.x * s.u.x) + s.p;
    f.m.y = (s.m.x * s.u.y);
    f.m.z = (s.m.x * s.u.z);
    f.e = (s.e + s.p) * s.u.x;
    return f;
}

static U jump(L l, L r)
{
    U j;
    j.rho = r.rho - l.rho;
    j.m = vsub(r.m, l.m);
    j.e = r.e - l.e;
    return j;
}

static V roe_vel(double w, double sl, double sr, L l, L r)
{
    return vmul(w, vadd(vmul(sl, l.u), vmul(sr, r.u)));
}

static U roe(L l, L r, double gamma) /* convective.c:71-213 */
{
    double gm1 = gamma - 1;
    double hl = (l.e + l.p) / l.rho, hr = (r.e + r.p) / r.rho;
    double sl = sqrt(l.rho), sr = sqrt(r.rho);
    double w = 1 / (sl + sr);
    V u = roe_vel(w, sl, sr, l, r);
    double h = w * ((sl * hl) + (sr * hr));
    double u2 = vdot(u, u);
    double a2 = gm1 * (h - (u2 / 2));
    double a = sqrt(a2);
    double eig[3] = {u.x - a, u.x, u.x + a};
    double al = sqrt(gamma * l.p / l.rho), ar = sqrt(gamma * r.p / r.rho);
    double el[3] = {l.u.x - al, l.u.x, l.u.x + al};
    double er[3] = {r.u.x - ar, r.u.x, r.u.x + ar};
    for (int i = 0; i < 3; i++) {
        double lam = eig[i];
        double d = fmax(0, fmax(lam - el[i], er[i] - lam));
        eig[i] = (fabs(lam) < d) ? d : fabs(lam);
    }
    U j = jump(l, r);
    double ws[5];
    ws[2] = j.m.y - (u.y * j.rho);
    ws[3] = j.m.z - (u.z * j.rho);
    ws[1] = gm1 / a2 *
            ((j.rho * (h - (u.x * u.x))) + (u.x * j.m.x) - j.e + (ws[2] * u.y) + (ws[3] * u.z));
    ws[0] = ((j.rho * (u.x + a)) - j.m.x - (a * ws[1])) / (2 * a);
    ws[4] = j.rho - (ws[0] + ws[1]);
    double ev[5][5] = {
        {1, 1, 0, 0, 1},
        {u.x - a, u.x, 0, 0, u.x + a},
        {u.y, u.y, 1, 0, u.y},
        {u.z, u.z, 0, 1, u.z},
        {h - (u.x * a), u2 / 2, u.y, u.z, h + (u.x * a)},
    };
    double ch[5] = {ws[0] * eig[0], ws[1] * eig[1], ws[2] * eig[1], ws[3] * eig[1], ws[4] * eig[2]};
    double d[5];
    for (int i = 0; i < 5; i++) {
        d[i] = 0;
        for (int k = 0; k < 5; k++) {
            d[i] += ev[i][k] * ch[k];
        }
    }
    U fl = phys(l), fr = phys(r), f;
    f.rho = (fl.rho + fr.rho - d[0]) / 2;
    f.m.x = (fl.m.x + fr.m.x - d[1]) / 2;
    f.m.y = (fl.m.y + fr.m.y - d[2]) / 2;
    f.m.z = (fl.m.z + fr.m.z - d[3]) / 2;
    f.e = (fl.e + fr.e - d[4]) / 2;
    return f;
}

static U hll_avg(L l, L r, double sl, double sr) /* convective.c:215-243 */
{
    U fl = phys(l);
    fl.rho *= sr;
    fl.m = vmul(sr, fl.m);
    fl.e *= sr;
    U fr = phys(r);
    fr.rho *= sl;
    fr.m = vmul(sl, fr.m);
    fr.e *= sl;
    double sj = sl * sr;
    U j = jump(l, r);
    j.rho *= sj;
    j.m = vmul(sj, j.m);
    j.e *= sj;
    double fac = 1 / (sr - sl);
    U f;
    f.rho = fac * (fl.rho - fr.rho + j.rho);
    f.m = vmul(fac, vadd(vsub(fl.m, fr.m), j.m));
    f.e = fac * (fl.e - fr.e + j.e);
    return f;
}

static void speeds(L l, L r, double gamma, double *s_l, double *s_r) /* convective.c:252-272 */
{
    double hl = (l.e + l.p) / l.rho, hr = (r.e + r.p) / r.rho;
    double sl = sqrt(l.rho), sr = sqrt(r.rho);
    double w = 1 / (sl + sr);
    V u = roe_vel(w, sl, sr, l, r);
    double h = w * ((sl * hl) + (sr * hr));
    double u2 = vdot(u, u);
    double a = sqrt((gamma - 1) * (h - (u2 / 2)));
    double al = sqrt(gamma * l.p / l.rho), ar = sqrt(gamma * r.p / r.rho);
    *s_l = fmin(l.u.x - al, u.x - a);
    *s_r = fmax(r.u.x + ar, u.x + a);
}

static U hll(L l, L r, double gamma)
{
    double sl, sr;
    speeds(l, r, gamma, &sl, &sr);
    if (sl >= 0) return phys(l);
    if (sr <= 0) return phys(r);
    return hll_avg(l, r, sl, sr);
}

static U contact(L k, double sk, double fk, double s) /* convective.c:276-298 */
{
    double fac = fk / (sk - s);
    U st;
    st.rho = fac;
    st.m.x = fac * s;
    st.m.y = fac * k.u.y;
    st.m.z = fac * k.u.z;
    st.e = fac * ((k.e / k.rho) + ((s - k.u.x) * (s + (k.p / fk))));
    U f = phys(k);
    f.rho += sk * (st.rho - k.rho);
    f.m = vadd(f.m, vmul(sk, vsub(st.m, k.m)));
    f.e += sk * (st.e - k.e);
    return f;
}

static U hllc(L l, L r, double gamma) /* convective.c:300-346 */
{
    double sl, sr;
    speeds(l, r, gamma, &sl, &sr);
    if (sl >= 0) return phys(l);
    if (sr <= 0) return phys(r);
    double fl = l.rho * (sl - l.u.x), fr = r.rho * (sr - r.u.x);
    double s = (r.p - l.p + (fl * l.u.x) - (fr * r.u.x)) / (fl - fr);
    if (sl <= 0 && 0 <= s) return contact(l, sl, fl, s);
    return contact(r, sr, fr, s);
}

static U hlle(L l, L r, double gamma) /* convective.c:348-389 */
{
    double sl = sqrt(l.rho), sr = sqrt(r.rho);
    double w = 1 / (sl + sr);
    double ux = w * ((sl * l.u.x) + (sr * r.u.x));
    double a2l = gamma * l.p / l.rho, a2r = gamma * r.p / r.rho;
    double al = sqrt(a2l), ar = sqrt(a2r);
    double a2 = w * ((sl * a2l) + (sr * a2r));
    double vj = (w * w) * sl * sr * ((r.u.x - l.u.x) * (r.u.x - l.u.x)) / 2;
    double a = sqrt(a2 + vj);
    double s_l = fmin(l.u.x - al, ux - a), s_r = fmax(r.u.x + ar, ux + a);
    if (s_l >= 0) return phys(l);
    if (s_r <= 0) return phys(r);
    return hll_avg(l, r, s_l, s_r);
}

static U ausm(L l, L r, double gamma, int dv) /* convective.c:391-547 */
{
    double al = sqrt(gamma * l.p / l.rho), ar = sqrt(gamma * r.p / r.rho);
    double a = fmax(al, ar);
    double pdl = l.p / l.rho, pdr = r.p / r.rho, pds = pdl + pdr;
    double ml = l.u.x / a, mr = r.u.x / a;
    double vpl, ppl, vmr, pmr;
    if (fabs(l.u.x) <= a) {
        double alpha = 2 * pdl / pds, f = l.u.x + a;
        vpl = (alpha * (f * f) / (4 * a)) + ((1 - alpha) * (l.u.x + fabs(l.u.x)) / 2);
        ppl = (l.p * (f * f) / (4 * (a * a))) * (2 - ml);
    }
    else {
        vpl = (l.u.x + fabs(l.u.x)) / 2;
        ppl = dv ? l.p * (l.u.x + fabs(l.u.x)) / (2 * l.u.x) : (l.p * (l.u.x + fabs(l.u.x)) / 2) / l.u.x;
    }
    if (fabs(r.u.x) <= a) {
        double alpha = 2 * pdr / pds, f = r.u.x - a;
        vmr = (-alpha * (f * f) / (4 * a)) + ((1 - alpha) * (r.u.x - fabs(r.u.x)) / 2);
        pmr = (r.p * (f * f) / (4 * (a * a))) * (2 + mr);
    }
    else {
        vmr = (r.u.x - fabs(r.u.x)) / 2;
        pmr = dv ? r.p * (r.u.x - fabs(r.u.x)) / (2 * r.u.x) : (r.p * (r.u.x - fabs(r.u.x)) / 2) / r.u.x;
    }
    double mf = (vpl * l.rho) + (vmr * r.rho), amf = fabs(mf), pf = ppl + pmr;
    double hl = (l.e + l.p) / l.rho, hr = (r.e + r.p) / r.rho;
    U f;
    f.rho = mf;
    double nd = ((mf * (l.u.x + r.u.x)) - (amf * (r.u.x - l.u.x))) / 2;
    if (dv) {
        double nv = (vpl * l.m.x) + (vmr * r.m.x);
        double pmin = fmin(l.p, r.p);
        double sw = fmin(1.0 / 2, fmin(1, (10 * fabs(r.p - l.p)) / pmin));
        f.m.x = ((((1 + sw) * nv) + ((1 - sw) * nd)) / 2) + pf;
    }
    else {
        f.m.x = nd + pf;
    }
    f.m.y = ((mf * (l.u.y + r.u.y)) - (amf * (r.u.y - l.u.y))) / 2;
    f.m.z = ((mf * (l.u.z + r.u.z)) - (amf * (r.u.z - l.u.z))) / 2;
    f.e = ((mf * (hl + hr)) - (amf * (hr - hl))) / 2;
    return f;
}

static U lxf(L l, L r, double gamma) /* convective.c:549-574 */
{
    double al = sqrt(gamma * l.p / l.rho), ar = sqrt(gamma * r.p / r.rho);
    double s = fmax(fabs(l.u.x) + al, fabs(r.u.x) + ar);
    U j = jump(l, r);
    j.rho *= s;
    j.m = vmul(s, j.m);
    j.e *= s;
    U fl = phys(l), fr = phys(r), f;
    f.rho = (fl.rho + fr.rho - j.rho) / 2;
    f.m = vdiv(vsub(vadd(fl.m, fr.m), j.m), 2);
    f.e = (fl.e + fr.e - j.e) / 2;
    return f;
}

static U central(L l, L r) /* convective.c:576-591 */
{
    U fl = phys(l), fr = phys(r), f;
    f.rho = (fl.rho + fr.rho) / 2;
    f.m = vdiv(vadd(fl.m, fr.m), 2);
    f.e = (fl.e + fr.e) / 2;
    return f;
}

static void convective(int kind, double *flux, const double *pl, const double *pr, double gamma, M b)
{
    L l = local(getp(pl), gamma, b), r = local(getp(pr), gamma, b);
    U f;
    switch (kind) {
        case TG_FLUX_ROE: f = roe(l, r, gamma); break;
        case TG_FLUX_HLL: f = hll(l, r, gamma); break;
        case TG_FLUX_HLLC: f = hllc(l, r, gamma); break;
        case TG_FLUX_HLLE: f = hlle(l, r, gamma); break;
        case TG_FLUX_AUSMD: f = ausm(l, r, gamma, 0); break;
        case TG_FLUX_AUSMDV: f = ausm(l, r, gamma, 1); break;
        case TG_FLUX_LXF: f = lxf(l, r, gamma); break;
        default: f = central(l, r); break;
    }
    f.m = mv(mt(b), f.m); /* local_to_global (convective.c:27-30) */
    flux[0] = f.rho, flux[1] = f.m.x, flux[2] = f.m.y, flux[3] = f.m.z, flux[4] = f.e;
}

/* ---- viscous flux (src/navierstokes/viscous.c:11-39) ---------------------------------------------- */

static void viscous(double *flux, const double *q, const V *g, const double *prop, M b)
{
    double gamma = prop[0], mu = prop[1], pr = prop[2];
    M tau;
    double dv = g[1].x + g[2].y + g[3].z;
    tau.x.x = 2 * mu * (g[1].x - (dv / 3));
    tau.y.y = 2 * mu * (g[2].y - (dv / 3));
    tau.z.z = 2 * mu * (g[3].z - (dv / 3));
    tau.y.x = tau.x.y = mu * (g[1].y + g[2].x);
    tau.z.x = tau.x.z = mu * (g[1].z + g[3].x);
    tau.z.y = tau.y.z = mu * (g[2].z + g[3].y);
    double fac = -mu * gamma / ((gamma - 1) * pr * (q[0] * q[0]));
    V heat = vmul(fac, vsub(vmul(q[0], g[4]), vmul(q[4], g[0])));
    V theta = vsub(mv(tau, (V){q[1], q[2], q[3]}), heat);
    V m = mv(tau, b.x);
    flux[0] = 0, flux[1] = m.x, flux[2] = m.y, flux[3] = m.z, flux[4] = vdot(theta, b.x);
}

/* ---- boundary conditions (src/euler/boundary.c, src/navierstokes/boundary.c) ---------------------- */

static P farfield(P in_g, P ctx, double gamma, M b) /* boundary.c:134-271 */
{
    L o = local(ctx, gamma, b), in = local(in_g, gamma, b);
    double gm1 = gamma - 1;
    double u2 = vdot(in.u, in.u), a2 = gamma * in.p / in.rho, a = sqrt(a2);
    double h = (u2 / 2) + (a2 / gm1);
    double ux = in.u.x, uy = in.u.y, uz = in.u.z;
    double li[5][5] = {
        {h + (a / gm1 * (ux - a)), -(ux + (a / gm1)), -uy, -uz, 1},
        {(-2 * h) + (4 / gm1 * a2), 2 * ux, 2 * uy, 2 * uz, -2},
        {-2 * uy * a2 / gm1, 0, 2 * a2 / gm1, 0, 0},
        {-2 * uz * a2 / gm1, 0, 0, 2 * a2 / gm1, 0},
        {h - (a / gm1 * (ux + a)), -ux + (a / gm1), -uy, -uz, 1},
    };
    double fac = gm1 / (2 * a2);
    double ci[5] = {in.rho, in.m.x, in.m.y, in.m.z, in.e};
    double cg[5] = {o.rho, o.m.x, o.m.y, o.m.z, o.e};
    double chi[5], chg[5];
    for (int i = 0; i < 5; i++) {
        chi[i] = 0, chg[i] = 0;
        for (int k = 0; k < 5; k++) {
            chi[i] += li[i][k] * ci[k];
            chg[i] += li[i][k] * cg[k];
        }
        chi[i] *= fac;
        chg[i] *= fac;
    }
    double ag = sqrt(gamma * o.p / o.rho);
    if (o.u.x - ag > 0) chg[0] = chi[0];
    if (o.u.x > 0) chg[1] = chi[1], chg[2] = chi[2], chg[3] = chi[3];
    if (o.u.x + ag > 0) chg[4] = chi[4];
    double ev[5][5] = {
        {1, 1, 0, 0, 1},
        {ux - a, ux, 0, 0, ux + a},
        {uy, uy, 1, 0, uy},
        {uz, uz, 0, 1, uz},
        {h - (ux * a), u2 / 2, uy, uz, h + (ux * a)},
    };
    for (int i = 0; i < 5; i++) {
        cg[i] = 0;
        for (int k = 0; k < 5; k++) cg[i] += ev[i][k] * chg[k];
    }
    V m = {cg[1], cg[2], cg[3]};
    V ul = vdiv(m, cg[0]);
    double p = (gamma - 1) * (cg[4] - (vdot(m, ul) / 2));
    P out;
    out.rho = fmax(1e-8, cg[0]);
    out.u = mv(mt(b), ul);
    out.p = fmax(1e-8, p);
    return out;
}

static P boundary_state(int kind, P in, P ctx, double gamma, M b)
{
    P o;
    switch (kind) {
        case TG_BC_SYMMETRY: {
            double un = vdot(in.u, b.x);
            o.rho = in.rho, o.u = vsub(in.u, vmul(2 * un, b.x)), o.p = in.p;
            return o;
        }
        case TG_BC_SUPERSONIC_INFLOW: return ctx;
        case TG_BC_SUPERSONIC_OUTFLOW: return in;
        case TG_BC_SUBSONIC_INFLOW: {
            double a2 = gamma * in.p / in.rho, a = sqrt(a2);
            double un = vdot(vsub(ctx.u, in.u), b.x);
            double f1 = in.rho * a;
            o.p = (ctx.p + in.p - (f1 * un)) / 2;
            o.rho = ctx.rho + ((o.p - ctx.p) / a2);
            o.u = vsub(ctx.u, vmul((ctx.p - o.p) / f1, b.x));
            return o;
        }
        case TG_BC_SUBSONIC_OUTFLOW: {
            double a2 = gamma * in.p / in.rho, a = sqrt(a2);
            o.p = ctx.p;
            o.rho = in.rho + ((o.p - in.p) / a2);
            o.u = vsub(in.u, vmul((in.p - o.p) / (in.rho * a), b.x));
            return o;
        }
        case TG_BC_PRESSURE_OUTFLOW: {
            double a = sqrt(gamma * in.p / in.rho);
            double p = (vdot(in.u, b.x) / a < 1) ? ctx.p : in.p;
            o.rho = in.rho * p / in.p, o.u = in.u, o.p = p;
            return o;
        }
        case TG_BC_FARFIELD: return farfield(in, ctx, gamma, b);
        case TG_BC_ADIABATIC_WALL: o.rho = in.rho, o.u = vmul(-1, in.u), o.p = in.p; return o;
        default: return in;
    }
}

/* ---- residual (src/equations) --------------------------------------------------------------- */

/* periodic ghosts receive their owners' rows: the single-process exchange (exchange.c:8-36) */
static void exchange(const tg_mesh *m, double *buf, int len)
{
    int n = m->num_neighbors;
    char *used = calloc(n ? n : 1, 1);
    for (int k = 0; k < n; k++) {
        int tag = m->neighbor_tag[2 * k];
        for (int j = 0; j < n; j++) {
            if (!used[j] && m->neighbor_tag[2 * j + 1] == tag) {
                used[j] = 1;
                int cnt = m->neighbor_recv_off[k + 1] - m->neighbor_recv_off[k];
                for (int i = 0; i < cnt; i++) {
                    int dst = m->neighbor_recv_off[k] + i;
                    int src = m->neighbor_send_idx[m->neighbor_send_off[j] + i];
                    memcpy(buf + (size_t)dst * len, buf + (size_t)src * len, sizeof(double) * len);
                }
                break;
            }
        }
    }
    free(used);
}

static void boundary(const tg_mesh *m, const tg_equations *e, double *prim) /* boundary.c:5-43 */
{
    for (int i = 0; i < e->num_boundaries; i++) {
        int ent = m->num_inner_entities + i;
        const double *c = e->boundary_context ? e->boundary_context + 5 * i : 0;
        P ctx = c ? getp(c) : (P){0, {0, 0, 0}, 0};
        for (int f = m->entity_face_off[ent]; f < m->entity_face_off[ent + 1]; f++) {
            int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
            putp(prim + 5 * (size_t)r,
                 boundary_state(e->boundary_kind[i], getp(prim + 5 * (size_t)l), ctx, e->property[0],
                                basis_of(m, f)));
        }
    }
}

static void gradient(const tg_mesh *m, double *prim, V *grad) /* gradient.c:7-58 */
{
    exchange(m, prim, 5);
    memset(grad, 0, sizeof(V) * 5 * m->num_cells);
    for (int f = 0; f < m->num_faces; f++) {
        int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
        V wl = vec_at(m->face_weight, 2 * (size_t)f), wr = vec_at(m->face_weight, 2 * (size_t)f + 1);
        for (int j = 0; j < 5; j++) {
            double diff = prim[5 * (size_t)r + j] - prim[5 * (size_t)l + j];
            grad[5 * (size_t)l + j] = vadd(grad[5 * (size_t)l + j], vmul(diff, wl));
            if (f < m->num_inner_faces) {
                grad[5 * (size_t)r + j] = vadd(grad[5 * (size_t)r + j], vmul(-diff, wr));
            }
        }
    }
}

static double *venkat_eps2(const tg_mesh *m, const tg_equations *e) /* limiter.c:8-21 */
{
    double *eps2 = malloc(sizeof(double) * m->num_inner_cells);
    for (int i = 0; i < m->num_inner_cells; i++) {
        if (e->limiter_parameter) {
            eps2[i] = e->limiter_parameter[i];
        }
        else {
            double x = e->limiter_coefficient * cbrt(m->cell_volume[i]);
            eps2[i] = x * x * x;
        }
    }
    return eps2;
}

static void limiter(const tg_mesh *m, const tg_equations *e, const double *prim, V *grad) /* limiter.c */
{
    double *eps2 = e->limiter == TG_LIMITER_VENKATAKRISHNAN ? venkat_eps2(m, e) : 0;
    for (int i = 0; i < m->num_inner_cells; i++) {
        double mn[5], mx[5], psi[5];
        for (int k = 0; k < 5; k++) mn[k] = mx[k] = prim[5 * (size_t)i + k];
        for (int j = m->cell_cell_off[i]; j < m->cell_cell_off[i + 1]; j++) {
            int o = m->cell_cell_idx[j];
            for (int k = 0; k < 5; k++) {
                mn[k] = fmin(mn[k], prim[5 * (size_t)o + k]);
                mx[k] = fmax(mx[k], prim[5 * (size_t)o + k]);
            }
        }
        for (int k = 0; k < 5; k++) psi[k] = 1;
        for (int j = m->cell_cell_off[i]; j < m->cell_cell_off[i + 1]; j++) {
            V off = vec_at(m->cell_offset, j);
            for (int k = 0; k < 5; k++) {
                double d2 = vdot(grad[5 * (size_t)i + k], off);
                if (is_close(d2, 0)) continue;
                double d1 = ((d2 > 0) ? mx[k] : mn[k]) - prim[5 * (size_t)i + k];
                if (e->limiter == TG_LIMITER_BARTH_JESPERSEN) {
                    psi[k] = fmin(psi[k], fmin(1, d1 / d2));
                }
                else {
                    double top = (((d1 * d1) + eps2[i]) * d2) + (2 * (d2 * d2) * d1);
                    double bot = (d1 * d1) + (2 * (d2 * d2)) + (d1 * d2) + eps2[i];
                    psi[k] = fmin(psi[k], top / bot / d2);
                }
            }
        }
        for (int k = 0; k < 5; k++) grad[5 * (size_t)i + k] = vmul(psi[k], grad[5 * (size_t)i + k]);
    }
    free(eps2);
}

int oracle_gradient(const tg_mesh *m, const tg_equations *e, double *prim, int limited, double *g)
{
    boundary(m, e, prim);
    gradient(m, prim, (V *)g);
    if (limited && e->limiter != TG_LIMITER_NONE) limiter(m, e, prim, (V *)g);
    return 0;
}

int oracle_derivative(const tg_mesh *m, const tg_equations *e, double *prim, double *d, double time)
{
    (void)time;
    int C = m->num_inner_cells, F = m->num_faces;
    const double *prop = e->property;
    memset(d, 0, sizeof(double) * 5 * C);
    boundary(m, e, prim);
    double flux[5];
    if (e->space_order == 1) { /* derivative.c:18-69 */
        exchange(m, prim, 5);
        for (int f = 0; f < F; f++) {
            int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
            convective(e->convective, flux, prim + 5 * (size_t)l, prim + 5 * (size_t)r, prop[0], basis_of(m, f));
            for (int j = 0; j < 5; j++) {
                d[5 * (size_t)l + j] += flux[j] * m->face_area[f];
                if (f < m->num_inner_faces) d[5 * (size_t)r + j] -= flux[j] * m->face_area[f];
            }
        }
    }
    else {
        V *g = calloc((size_t)5 * m->num_cells, sizeof(V));
        gradient(m, prim, g);
        if (e->viscous == TG_VISCOUS_CENTRAL) { /* derivative.c:91-156 */
            exchange(m, (double *)g, 15);
            for (int f = 0; f < F; f++) {
                int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
                int bnd = f >= m->num_inner_faces && f < m->off_boundary_faces;
                const double *ql = prim + 5 * (size_t)l, *qr = prim + 5 * (size_t)r;
                double qm[5];
                V gm[5];
                for (int j = 0; j < 5; j++) qm[j] = (ql[j] + qr[j]) / 2;
                for (int j = 0; j < 5; j++) {
                    V a = g[5 * (size_t)l + j], b = g[5 * (size_t)r + j];
                    gm[j] = bnd ? a : (V){(a.x + b.x) / 2, (a.y + b.y) / 2, (a.z + b.z) / 2};
                }
                const double *cr = m->face_correction + 4 * (size_t)f;
                V unit = {cr[0], cr[1], cr[2]};
                for (int j = 0; j < 5; j++) { /* correct (derivative.c:81-89) */
                    double adj = vdot(gm[j], unit) - ((qr[j] - ql[j]) / cr[3]);
                    gm[j] = vsub(gm[j], vmul(adj, unit));
                }
                viscous(flux, qm, gm, prop, basis_of(m, f));
                for (int j = 0; j < 5; j++) {
                    d[5 * (size_t)l + j] -= flux[j] * m->face_area[f];
                    if (f < m->num_inner_faces) d[5 * (size_t)r + j] += flux[j] * m->face_area[f];
                }
            }
        }
        if (e->limiter != TG_LIMITER_NONE) limiter(m, e, prim, g);
        if (e->convective != TG_FLUX_NONE) { /* derivative.c:166-227 */
            exchange(m, (double *)g, 15);
            for (int f = 0; f < F; f++) {
                int l = m->face_cell[2 * f], r = m->face_cell[2 * f + 1];
                int bnd = f >= m->num_inner_faces && f < m->off_boundary_faces;
                double pl[5], pr[5];
                const double *o = m->face_offset + 6 * (size_t)f;
                V ol = {o[0], o[1], o[2]}, orr = {o[3], o[4], o[5]};
                for (int j = 0; j < 5; j++) {
                    pl[j] = prim[5 * (size_t)l + j] + vdot(g[5 * (size_t)l + j], ol);
                    pr[j] = bnd ? prim[5 * (size_t)r + j] : prim[5 * (size_t)r + j] + vdot(g[5 * (size_t)r + j], orr);
                }
                convective(e->convective, flux, pl, pr, prop[0], basis_of(m, f));
                for (int j = 0; j < 5; j++) {
                    d[5 * (size_t)l + j] += flux[j] * m->face_area[f];
                    if (f < m->num_inner_faces) d[5 * (size_t)r + j] -= flux[j] * m->face_area[f];
                }
            }
        }
        free(g);
    }
    /* finalize_derivative (derivative.c:229-267), with the source kinds of the run cases:
     * body force (run/rayleigh_taylor_instability/run.c:17-24) and bulk forcing, whose prepare pass
     * averages the state over the inner cells (run/periodic_hill/run.c:8-21, average.c:8-40) */
    const double *sp = e->source_parameter;
    double avg[5] = {0, 0, 0, 0, 0};
    if (e->source == TG_SOURCE_BULK_FORCING) {
        for (int i = 0; i < C; i++) {
            for (int j = 0; j < 5; j++) avg[j] += m->cell_volume[i] * prim[5 * (size_t)i + j];
        }
        for (int j = 0; j < 5; j++) avg[j] /= m->sum_volume;
    }
    for (int i = 0; i < C; i++) {
        const double *q = prim + 5 * (size_t)i;
        double src[5] = {0, 0, 0, 0, 0};
        if (e->source == TG_SOURCE_BODY_FORCE) {
            src[1] = sp[0] * q[0];
            src[2] = sp[1] * q[0];
            src[3] = sp[2] * q[0];
            src[4] = ((src[1] * q[1]) + (src[2] * q[2])) + (src[3] * q[3]);
        }
        else if (e->source == TG_SOURCE_BULK_FORCING) {
            double s1 = q[0] * (sp[0] - avg[1]) / sp[1];
            src[1] = s1;
            src[4] = q[1] * s1;
        }
        for (int j = 0; j < 5; j++) {
            d[5 * (size_t)i + j] = -d[5 * (size_t)i + j] / m->cell_volume[i];
            if (e->source != TG_SOURCE_NONE) d[5 * (size_t)i + j] = d[5 * (size_t)i + j] + src[j];
        }
    }
    return 0;
}

double oracle_timestep(const tg_mesh *m, const tg_equations *e, const double *prim)
{
    double mn = DBL_MAX;
    for (int i = 0; i < m->num_inner_cells; i++) {
        P q = getp(prim + 5 * (size_t)i);
        V proj = vec_at(m->cell_projection, i);
        double s = e->physics == TG_NAVIERSTOKES ? navierstokes_timestep(q, e->property, m->cell_volume[i], proj)
                                                 : euler_timestep(q, e->property[0], m->cell_volume[i], proj);
        if (s < mn) mn = s;
    }
    return mn;
}

void oracle_residual(const tg_mesh *m, const double *d, double *res)
{
    for (int j = 0; j < 5; j++) res[j] = 0;
    for (int i = 0; i < m->num_inner_cells; i++) {
        for (int j = 0; j < 5; j++) res[j] += m->cell_volume[i] * (d[5 * (size_t)i + j] * d[5 * (size_t)i + j]);
    }
    for (int j = 0; j < 5; j++) res[j] = sqrt(res[j] / m->sum_volume);
}

/* ---- time integration (src/simulation/advance.c, gmres.c) ----------------------------------------- */

static const double ALPHA[3][6][7] = {
    {{0, 1.0000}, {0, 0.3333, 1.0000}, {0, 0.1481, 0.4000, 1.0000}, {0, 0.0833, 0.2069, 0.4265, 1.0000},
     {0, 0.0533, 0.1263, 0.2375, 0.4414, 1.0000}, {0, 0.0370, 0.0851, 0.1521, 0.2562, 0.4512, 1.0000}},
    {{0, 1.0000}, {0, 0.4242, 1.0000}, {0, 0.1918, 0.4929, 1.0000}, {0, 0.1084, 0.2602, 0.5052, 1.0000},
     {0, 0.0695, 0.1602, 0.2898, 0.5060, 1.0000}, {0, 0.0482, 0.1085, 0.1885, 0.3050, 0.5063, 1.0000}},
    {{0, 1.0000}, {0, 0.6612, 1.0000}, {0, 0.2884, 0.5010, 1.0000}, {0, 0.1666, 0.3027, 0.5275, 1.0000},
     {0, 0.1067, 0.1979, 0.3232, 0.5201, 1.0000}, {0, 0.0742, 0.1393, 0.2198, 0.3302, 0.5181, 1.0000}},
};

double oracle_lserk(const tg_mesh *m, const tg_equations *e, double *prim, double *time, double *res,
                    double max_step, double courant, int order, int stages)
{
    int C = m->num_inner_cells;
    double gamma = e->property[0];
    const double *alpha = ALPHA[order - 1][stages - 1];
    double step0 = courant * oracle_timestep(m, e, prim);
    double step = fmin(step0, max_step);
    double *u0 = malloc(sizeof(double) * 5 * C), *d = malloc(sizeof(double) * 5 * C);
    for (int i = 0; i < C; i++) {
        U c = to_cons(getp(prim + 5 * (size_t)i), gamma);
        double *o = u0 + 5 * (size_t)i;
        o[0] = c.rho, o[1] = c.m.x, o[2] = c.m.y, o[3] = c.m.z, o[4] = c.e;
    }
    for (int s = 0; s < stages; s++) {
        oracle_derivative(m, e, prim, d, *time + (alpha[s] * step));
        for (int i = 0; i < C; i++) {
            double c[5];
            for (int k = 0; k < 5; k++) c[k] = u0[5 * (size_t)i + k] + (d[5 * (size_t)i + k] * alpha[s + 1] * step);
            putp(prim + 5 * (size_t)i, to_prim((U){c[0], {c[1], c[2], c[3]}, c[4]}, gamma));
        }
    }
    *time += step;
    oracle_residual(m, d, res);
    free(u0);
    free(d);
    return step0;
}

double oracle_euler(const tg_mesh *m, const tg_equations *e, double *prim, double *time, double *res,
                    double max_step, double courant)
{
    int C = m->num_inner_cells;
    double gamma = e->property[0];
    double step0 = courant * oracle_timestep(m, e, prim);
    double step = fmin(step0, max_step);
    double *d = malloc(sizeof(double) * 5 * C);
    oracle_derivative(m, e, prim, d, *time);
    for (int i = 0; i < C; i++) {
        U c = to_cons(getp(prim + 5 * (size_t)i), gamma);
        double *di = d + 5 * (size_t)i;
        c.rho += di[0] * step, c.m.x += di[1] * step, c.m.y += di[2] * step, c.m.z += di[3] * step;
        c.e += di[4] * step;
        putp(prim + 5 * (size_t)i, to_prim(c, gamma));
    }
    *time += step;
    oracle_residual(m, d, res);
    free(d);
    return step0;
}

static double dot(const double *a, const double *b, long n)
{
    double s = 0;
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static void cons_to_prim_all(const tg_mesh *m, const double *u, double *prim, double gamma)
{
    for (int i = 0; i < m->num_inner_cells; i++) {
        const double *c = u + 5 * (size_t)i;
        putp(prim + 5 * (size_t)i, to_prim((U){c[0], {c[1], c[2], c[3]}, c[4]}, gamma));
    }
}

/* gmres.c:52-149 with the finite-difference matvec of gmres.c:12-50 */
static void gmres(const tg_mesh *m, const tg_equations *e, const double *u, const double *d, const double *r,
                  double *inc, double time, double step, double norm, double fd, double ktol, int dim)
{
    long n = 5L * m->num_inner_cells;
    memset(inc, 0, sizeof(double) * n);
    if (norm <= 0) return;
    double *rhs = calloc(dim + 1, sizeof(double)), *V = calloc((size_t)(dim + 1) * n, sizeof(double));
    double *w = calloc(n, sizeof(double)), *H = calloc((size_t)(dim + 1) * dim, sizeof(double));
    double *cs = calloc(dim, sizeof(double)), *sn = calloc(dim, sizeof(double)), *coef = calloc(dim, sizeof(double));
    double *p1 = calloc((size_t)5 * m->num_cells, sizeof(double)), *d1 = calloc(n, sizeof(double));
    double *pert = malloc(sizeof(double) * n);
    rhs[0] = norm;
    for (long i = 0; i < n; i++) V[i] = -r[i] / norm;
    double tol = ktol * norm;
    int k = 0;
    for (; k < dim; k++) {
        double *vk = V + (long)k * n;
        double eps = fd / sqrt(dot(vk, vk, n));
        for (long i = 0; i < n; i++) pert[i] = u[i] + (eps * vk[i]);
        memset(p1, 0, sizeof(double) * 5 * m->num_cells);
        cons_to_prim_all(m, pert, p1, e->property[0]);
        oracle_derivative(m, e, p1, d1, time);
        for (long i = 0; i < n; i++) w[i] = vk[i] - (step * (d1[i] - d[i]) / eps);
        for (int i = 0; i < k + 1; i++) {
            double h = dot(V + (long)i * n, w, n);
            H[i * dim + k] = h;
            for (long j = 0; j < n; j++) w[j] -= h * V[(long)i * n + j];
        }
        H[(k + 1) * dim + k] = sqrt(dot(w, w, n));
        for (int i = 0; i < k; i++) {
            double tmp = (cs[i] * H[i * dim + k]) + (sn[i] * H[(i + 1) * dim + k]);
            H[(i + 1) * dim + k] = (-sn[i] * H[i * dim + k]) + (cs[i] * H[(i + 1) * dim + k]);
            H[i * dim + k] = tmp;
        }
        double rot = sqrt((H[k * dim + k] * H[k * dim + k]) + (H[(k + 1) * dim + k] * H[(k + 1) * dim + k]));
        cs[k] = H[k * dim + k] / rot;
        sn[k] = H[(k + 1) * dim + k] / rot;
        H[k * dim + k] = rot;
        rhs[k + 1] = -sn[k] * rhs[k];
        rhs[k] = cs[k] * rhs[k];
        if (fabs(rhs[k + 1]) < tol) {
            k += 1;
            break;
        }
        for (long i = 0; i < n; i++) V[(long)(k + 1) * n + i] = w[i] / H[(k + 1) * dim + k];
    }
    for (int i = k - 1; i >= 0; i--) {
        coef[i] = rhs[i];
        for (int j = i + 1; j < k; j++) coef[i] -= H[i * dim + j] * coef[j];
        coef[i] /= H[i * dim + i];
        for (long j = 0; j < n; j++) inc[j] += coef[i] * V[(long)i * n + j];
    }
    free(rhs), free(V), free(w), free(H), free(cs), free(sn), free(coef), free(p1), free(d1), free(pert);
}

double oracle_implicit_euler(const tg_mesh *m, const tg_equations *e, double *prim, double *time, double *res,
                             double max_step, double courant, double ntol, double ktol, int dim)
{
    int C = m->num_inner_cells;
    long n = 5L * C;
    double gamma = e->property[0];
    double step0 = courant * oracle_timestep(m, e, prim);
    double step = fmin(step0, max_step);
    double *u = calloc(n, sizeof(double)), *u0 = calloc(n, sizeof(double)), *d = calloc(n, sizeof(double));
    double *r = calloc(n, sizeof(double)), *inc = calloc(n, sizeof(double));
    for (int i = 0; i < C; i++) {
        U c = to_cons(getp(prim + 5 * (size_t)i), gamma);
        double *o = u + 5 * (size_t)i;
        o[0] = c.rho, o[1] = c.m.x, o[2] = c.m.y, o[3] = c.m.z, o[4] = c.e;
    }
    memcpy(u0, u, sizeof(double) * n);
    *time += step;
    oracle_derivative(m, e, prim, d, *time);
    for (long i = 0; i < n; i++) r[i] = -d[i] * step;
    double norm = sqrt(dot(r, r, n));
    double fd = 1e-6 * fmax(1, sqrt(dot(u, u, n))) / fmax(1, norm);
    double tol = ntol * norm;
    long max_iter = 128L * (C + 1);
    for (long it = 0; it < max_iter && norm > tol; it++) {
        gmres(m, e, u, d, r, inc, *time, step, norm, fd, ktol, dim);
        for (long i = 0; i < n; i++) u[i] += inc[i];
        cons_to_prim_all(m, u, prim, gamma);
        oracle_derivative(m, e, prim, d, *time);
        for (long i = 0; i < n; i++) r[i] = u[i] - u0[i] - (d[i] * step);
        norm = sqrt(dot(r, r, n));
        fd = 1e-6 * fmax(1, sqrt(dot(u, u, n))) / fmax(1, norm);
    }
    oracle_residual(m, d, res);
    free(u), free(u0), free(d), free(r), free(inc);
    return step0;
}
