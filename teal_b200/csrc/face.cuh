// Face-flux kernel: reconstruction, viscous and convective flux of one face per thread.
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace tg {

// ---- face fluxes (src/equations/derivative.c:18-227) ------------------------------------------
//
// Writes the flux record G[f] = (convective - viscous) flux * area; the cell gather adds it to the
// left cell and subtracts it from the right one, as teal's face loops do.

// Reconstructed face state of one side: q + (psi * grad) . offset per variable, streamed one
// variable at a time from the cell's gradient record so only the result stays live
// (derivative.c:158-164)
template <typename R, bool FOLD>
__device__ __forceinline__ void reconstruct(const Prim<R> &q, const R *__restrict__ rec, int c, V3<R> off,
                                            R (&out)[5])
{
    R qv[5] = {q.rho, q.u.x, q.u.y, q.u.z, q.p};
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R gx, gy, gz, ps;
        grad_rec_load(rec, c, v, gx, gy, gz, ps);
        V3<R> gv = v3(gx, gy, gz);
        if (!FOLD) {
            gv = v3(gv.x * ps, gv.y * ps, gv.z * ps);
        }
        out[v] = qv[v] + dot(gv, off);
    }
}

// Two ways to reach the geometry of a face: straight from the SoA arrays (DirectGeo, one face per
// thread, loads issued by the thread) or from a tile staged in shared memory (FaceTile, bulk
// asynchronous copies). Both expose the same accessors; `i` is the face's element in the tile.

template <typename R>
struct DirectGeo {
    const Geometry<R> &g;
    int F, f;
    __device__ __forceinline__ int2 cells(int) const { return g.lr[f]; }
    __device__ __forceinline__ V3<R> normal(int) const { return load_v3(g.basis, F, f); }
    __device__ __forceinline__ Basis<R> basis(int) const { return load_basis(g.basis, F, f); }
    // the basis again later in the thread: re-read (L1) instead of kept live in registers
    __device__ __forceinline__ Basis<R> basis_again(int) const { return reload_basis(g.basis, F, f); }
    __device__ __forceinline__ V3<R> normal_again(int) const
    {
        return v3(reload(g.basis + f), reload(g.basis + F + f), reload(g.basis + 2 * F + f));
    }
    __device__ __forceinline__ V3<R> offl(int) const { return load_v3(g.offl, F, f); }
    __device__ __forceinline__ V3<R> offr(int) const { return load_v3(g.offr, F, f); }
    __device__ __forceinline__ R area(int) const { return __ldg(g.area + f); }
    __device__ __forceinline__ V3<R> corr(int) const { return load_v3(g.corr, F, f); }
    __device__ __forceinline__ R corr_norm(int) const { return __ldg(g.corr + 3 * F + f); }
};

// Geometry of one tile of FACE_BLOCK consecutive faces in shared memory, staged by bulk
// asynchronous copies (one per SoA row, all in flight at once, completing on one mbarrier) so the
// streamed face geometry costs the threads neither registers nor load instructions; rows: area,
// basis (9 in the exact form; the normal's 3 otherwise, see frame_of), offsets left / right
// (3 + 3, second order), correction (4, Navier-Stokes).
template <typename R, int ORDER, bool NS>
struct FaceTile {
    static constexpr int PAD = 16 / int(sizeof(R));
    static constexpr int SROW = FACE_BLOCK + PAD;
    static constexpr int NBASIS = kExact ? 9 : 3;
    static constexpr int ROWS = 1 + NBASIS + (ORDER == 2 ? 6 + (NS ? 4 : 0) : 0);
    static constexpr int R_AREA = 0, R_BASIS = 1, R_OFFL = 1 + NBASIS, R_OFFR = R_OFFL + 3;
    static constexpr int R_CORR = (ORDER == 2) ? R_OFFR + 3 : R_OFFL;
    R geo[ROWS][SROW];
    int2 lr[FACE_BLOCK + 2];
    uint64_t bar;
    uint8_t shift[ROWS + 1];  // elements before the tile's first face in each staged row

    __device__ __forceinline__ const R *row_src(const Geometry<R> &g, int F, int r) const
    {
        if (r == R_AREA) return g.area;
        if (r < R_BASIS + NBASIS) return g.basis + (size_t)(r - R_BASIS) * F;
        if (ORDER == 2 && r < R_OFFL + 3) return g.offl + (size_t)(r - R_OFFL) * F;
        if (ORDER == 2 && r < R_OFFR + 3) return g.offr + (size_t)(r - R_OFFR) * F;
        return g.corr + (size_t)(r - R_CORR) * F;
    }

    // thread 0 issues the copies of faces [f0, f0 + n); every thread then waits (bounded).
    // Returns false after a wait that gave up (the error word then has the timeout bit); the
    // decision is the same in every thread of the block.
    // `polls` bounds the first wait (MBAR_POLLS normally; a smaller value lets a test make it give up);
    // the drain after a wait that gave up always uses the full MBAR_POLLS.
    __device__ __forceinline__ bool stage(const Geometry<R> &g, int F, int f0, int n, int *err, int polls)
    {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            uint32_t total = stage_span(lr, g.lr + f0, n, &bar, false, &shift[ROWS]);
            for (int r = 0; r < ROWS; r++) {
                total += stage_span(geo[r], row_src(g, F, r) + f0, n, &bar, false, &shift[r]);
            }
            mbar_arrive_expect_tx(&bar, total);
            stage_span(lr, g.lr + f0, n, &bar, true, nullptr);
            for (int r = 0; r < ROWS; r++) {
                stage_span(geo[r], row_src(g, F, r) + f0, n, &bar, true, nullptr);
            }
        }
        __syncthreads();
        const bool ok = mbar_wait_bounded(&bar, 0, polls);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicOr(err, ERR_TIMEOUT);
            }
            mbar_wait_bounded(&bar, 0, MBAR_POLLS);  // let copies still in flight land before the block exits
            return false;
        }
        return true;
    }

    __device__ __forceinline__ R at(int r, int i) const { return geo[r][shift[r] + i]; }
    __device__ __forceinline__ V3<R> v3_at(int r, int i) const { return v3(at(r, i), at(r + 1, i), at(r + 2, i)); }
    __device__ __forceinline__ int2 cells(int i) const { return lr[shift[ROWS] + i]; }
    __device__ __forceinline__ V3<R> normal(int i) const { return v3_at(R_BASIS, i); }
    template <int NB = NBASIS>
    __device__ __forceinline__ Basis<R> basis(int i) const
    {
        static_assert(NB == 9, "the full basis is staged in the exact form only");
        Basis<R> b;
        b.x = v3_at(R_BASIS, i);
        b.y = v3_at(R_BASIS + 3, i);
        b.z = v3_at(R_BASIS + 6, i);
        return b;
    }
    template <int NB = NBASIS>
    __device__ __forceinline__ Basis<R> basis_again(int i) const { return basis<NB>(i); }
    __device__ __forceinline__ V3<R> normal_again(int i) const { return normal(i); }
    __device__ __forceinline__ V3<R> offl(int i) const { return v3_at(R_OFFL, i); }
    __device__ __forceinline__ V3<R> offr(int i) const { return v3_at(R_OFFR, i); }
    __device__ __forceinline__ R area(int i) const { return at(R_AREA, i); }
    __device__ __forceinline__ V3<R> corr(int i) const { return v3_at(R_CORR, i); }
    __device__ __forceinline__ R corr_norm(int i) const { return at(R_CORR + 3, i); }
};

// Viscous flux of face f (element i of its tile): the face average of both cells' states and
// unlimited gradients, corrected along the centre-to-centre direction, in the face normal's frame
template <typename R, typename Geo>
__device__ __forceinline__ Cons<R> viscous_face(const Geo &geo, int i, bool boundary, int2 c, int N,
                                                const double *__restrict__ q, const R *__restrict__ rec, R gamma,
                                                R mu, R prandtl)
{
    // face average corrected along the centre-to-centre direction (derivative.c:71-89)
    Prim<R> ql = reload_prim<R>(q, N, c.x);
    Prim<R> qr = reload_prim<R>(q, N, c.y);
    R qlv[5] = {ql.rho, ql.u.x, ql.u.y, ql.u.z, ql.p};
    R qrv[5] = {qr.rho, qr.u.x, qr.u.y, qr.u.z, qr.p};
    R qm[5], gm[15];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        qm[v] = (qlv[v] + qrv[v]) / R(2);
    }
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R ax, ay, az, ap, bx, by, bz, bp;
        grad_rec_load(rec, c.x, v, ax, ay, az, ap);
        if (boundary) {
            gm[3 * v] = ax, gm[3 * v + 1] = ay, gm[3 * v + 2] = az;
        }
        else {
            grad_rec_load(rec, c.y, v, bx, by, bz, bp);
            gm[3 * v] = (ax + bx) / R(2), gm[3 * v + 1] = (ay + by) / R(2), gm[3 * v + 2] = (az + bz) / R(2);
        }
    }
    V3<R> unit = geo.corr(i);
    const R cnorm = geo.corr_norm(i);
    const R inv_norm = R(1) / cnorm;
#pragma unroll
    for (int v = 0; v < 5; v++) {
        V3<R> gv = v3(gm[3 * v], gm[3 * v + 1], gm[3 * v + 2]);
        const R dq = qrv[v] - qlv[v];
        R adjust = dot(gv, unit) - (kExact ? (dq / cnorm) : (dq * inv_norm));
        gv = sub(gv, mul(adjust, unit));
        gm[3 * v] = gv.x;
        gm[3 * v + 1] = gv.y;
        gm[3 * v + 2] = gv.z;
    }
    Grad<R> gg;
    gg.rho = v3(gm[0], gm[1], gm[2]);
    gg.ux = v3(gm[3], gm[4], gm[5]);
    gg.uy = v3(gm[6], gm[7], gm[8]);
    gg.uz = v3(gm[9], gm[10], gm[11]);
    gg.p = v3(gm[12], gm[13], gm[14]);
    // the viscous flux needs only the normal row of the basis
    Basis<R> nb;
    nb.x = geo.normal_again(i);
    nb.y = nb.x;
    nb.z = nb.x;
    return viscous_central(prim_from(qm), gg, gamma, mu, prandtl, nb);
}

// The flux record of face f (element i of its tile). The convective flux comes first (its
// reconstruction streams the limited gradients), the viscous flux second (its face-averaged
// gradient re-reads the unlimited gradients, which are still in L1).
// Records: G[f] = (convective - viscous) * area; in the exact translation units with a viscous
// flux, G[f] = convective * area and G[flux_rec2_offset(F) + f] = viscous * area instead, because teal adds all of a
// cell's viscous terms before its convective ones (derivative.c:279-292) and the cell gather must
// repeat that order.
template <typename R, int FK, bool NS, int ORDER, bool FOLD, typename Geo>
__device__ __forceinline__ void face_flux(const Geo &geo, int i, int f, const Sizes &s, const double *__restrict__ q,
                                          const R *__restrict__ rec, R gamma, R mu, R prandtl, R *__restrict__ G,
                                          const PressureRefOf<R> &pr_ref)
{
    const int N = s.N;
    const bool boundary = (f >= s.F_in) && (f < s.F_bd);
    const int2 c = geo.cells(i);
    // FP32 fluxes work with the pressure relative to the instance's reference (Local::dp); the
    // difference is taken in FP64, before the rounding to FP32
    double pref = 0.0;
    if constexpr (sizeof(R) == sizeof(float)) {
        pref = pr_ref.of(c.x);
    }

    // convective flux: the basis and the cell states are dead while the flux runs in the face frame
    // and are re-read afterwards
    Cons<R> fc{R(0), v3(R(0), R(0), R(0)), R(0)};
    if (FK != FK_NONE) {
        Local<R> l, r;
        {
            Prim<R> ql, qr;
            if constexpr (sizeof(R) == sizeof(float)) {
                ql = load_prim_rel<R>(q, N, c.x, pref);
                qr = load_prim_rel<R>(q, N, c.y, pref);
            }
            else {
                ql = load_prim<R>(q, N, c.x);
                qr = load_prim<R>(q, N, c.y);
            }
            // the stored basis in the exact form; the normal and tangents of its own otherwise
            Basis<R> b;
            if constexpr (kExact) {
                b = geo.basis(i);
            }
            else {
                b = frame_of(geo.normal(i));
            }
            if (ORDER == 1) {
                l = make_local(ql, gamma, b, R(pref));
                r = make_local(qr, gamma, b, R(pref));
            }
            else {
                R pl[5], pr[5];
                reconstruct<R, FOLD>(ql, rec, c.x, geo.offl(i), pl);
                if (boundary) {  // the ghost state enters unreconstructed (derivative.c:203-211)
                    pr[0] = qr.rho, pr[1] = qr.u.x, pr[2] = qr.u.y, pr[3] = qr.u.z, pr[4] = qr.p;
                }
                else {
                    reconstruct<R, FOLD>(qr, rec, c.y, geo.offr(i), pr);
                }
                l = make_local(prim_from(pl), gamma, b, R(pref));
                r = make_local(prim_from(pr), gamma, b, R(pref));
            }
        }
        fc = convective_flux_local<FK>(l, r, gamma);
        if constexpr (kExact) {
            fc.m = to_global(geo.basis_again(i), fc.m);
        }
        else {
            fc.m = to_global(frame_of(geo.normal_again(i)), fc.m);
        }
    }
    R area = geo.area(i);
    R gf[5] = {fc.rho * area, fc.m.x * area, fc.m.y * area, fc.m.z * area, fc.e * area};

    if (NS && ORDER == 2) {
        const Cons<R> fv = viscous_face<R>(geo, i, boundary, c, N, q, rec, gamma, mu, prandtl);
        if constexpr (kExact) {
            const R gv[5] = {fv.rho * area, fv.m.x * area, fv.m.y * area, fv.m.z * area, fv.e * area};
            flux_rec_store(G + flux_rec2_offset(s.F), s.F, f, gv);
        }
        else {
            gf[0] -= fv.rho * area;
            gf[1] -= fv.m.x * area;
            gf[2] -= fv.m.y * area;
            gf[3] -= fv.m.z * area;
            gf[4] -= fv.e * area;
        }
    }
    flux_rec_store(G, s.F, f, gf);
}

// One thread per face, geometry loaded by the threads. face_minb caps the registers so that
// several blocks stay resident per SM.
// X: this is the exact translation unit's instantiation (a distinct kernel name per arithmetic).
template <typename R, int FK, bool NS, int ORDER, bool FOLD, bool X>
__global__ void __launch_bounds__(FACE_BLOCK, face_minb<R>(NS)) k_face(Sizes s, Geometry<R> g, const double *__restrict__ q,
                                                   const R *__restrict__ rec, R gamma, R mu, R prandtl,
                                                   R *__restrict__ G, PressureRefOf<R> pr_ref)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    const int f = s.lo + blockIdx.x * FACE_BLOCK + threadIdx.x;
    if (f >= s.hi) {
        return;
    }
    DirectGeo<R> geo{g, s.F, f};
    face_flux<R, FK, NS, ORDER, FOLD>(geo, 0, f, s, q, rec, gamma, mu, prandtl, G, pr_ref);
}

// One tile of FACE_BLOCK faces per block, its geometry staged in shared memory by bulk copies
// before the threads (one face each) start. A wait that gives up sets ERR_TIMEOUT in the error
// word and ends the block.
template <typename R, int FK, bool NS, int ORDER, bool FOLD, bool X>
__global__ void __launch_bounds__(FACE_BLOCK, face_minb<R>(NS)) k_face_staged(Sizes s, Geometry<R> g,
                                                          const double *__restrict__ q,
                                                          const R *__restrict__ rec, R gamma, R mu,
                                                          R prandtl, R *__restrict__ G, int *err,
                                                          PressureRefOf<R> pr_ref, int polls)
{
    static_assert(X == kExact, "exact kernels live in the exact translation units only");
    __shared__ __align__(16) FaceTile<R, ORDER, NS> t;
    const int f0 = s.lo + blockIdx.x * FACE_BLOCK;
    const int n = min(FACE_BLOCK, s.hi - f0);
    if (!t.stage(g, s.F, f0, n, err, polls)) {
        return;
    }
    if (threadIdx.x < n) {
        face_flux<R, FK, NS, ORDER, FOLD>(t, threadIdx.x, f0 + threadIdx.x, s, q, rec, gamma, mu, prandtl, G,
                                          pr_ref);
    }
}

}  // namespace tg
