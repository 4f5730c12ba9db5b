// Face-flux kernel: reconstruction, viscous and convective flux of one face per thread.
#pragma once

#include "common.cuh"

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

// One thread per face. The convective flux comes first (its reconstruction streams the limited
// gradients), the viscous flux second (its face-averaged gradient re-reads the unlimited gradients,
// which are still in L1); FACE_MINB caps the registers so that many blocks stay resident per SM.
template <typename R, int FK, bool NS, int ORDER, bool FOLD>
__global__ void __launch_bounds__(FACE_BLOCK, FACE_MINB) k_face(Sizes s, Geometry<R> g, const double *__restrict__ q,
                                                   const R *__restrict__ rec, R gamma, R mu, R prandtl,
                                                   R *__restrict__ G)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= s.F) {
        return;
    }
    const int F = s.F, N = s.N;
    const bool boundary = (f >= s.F_in) && (f < s.F_bd);
    int2 c = g.lr[f];

    // convective flux: the basis and the cell states are dead while the flux runs in the face frame
    // and are re-read afterwards
    Cons<R> fc{R(0), v3(R(0), R(0), R(0)), R(0)};
    if (FK != FK_NONE) {
        Local<R> l, r;
        {
            Prim<R> ql = load_prim<R>(q, N, c.x);
            Prim<R> qr = load_prim<R>(q, N, c.y);
            Basis<R> b = load_basis(g.basis, F, f);
            if (ORDER == 1) {
                l = make_local(ql, gamma, b);
                r = make_local(qr, gamma, b);
            }
            else {
                R pl[5], pr[5];
                reconstruct<R, FOLD>(ql, rec, c.x, load_v3(g.offl, F, f), pl);
                if (boundary) {  // the ghost state enters unreconstructed (derivative.c:203-211)
                    pr[0] = qr.rho, pr[1] = qr.u.x, pr[2] = qr.u.y, pr[3] = qr.u.z, pr[4] = qr.p;
                }
                else {
                    reconstruct<R, FOLD>(qr, rec, c.y, load_v3(g.offr, F, f), pr);
                }
                l = make_local(prim_from(pl), gamma, b);
                r = make_local(prim_from(pr), gamma, b);
            }
        }
        fc = convective_flux_local<FK>(l, r, gamma);
        fc.m = to_global(reload_basis(g.basis, F, f), fc.m);
    }
    R area = __ldg(g.area + f);
    R gf[5] = {fc.rho * area, fc.m.x * area, fc.m.y * area, fc.m.z * area, fc.e * area};

    if (NS && ORDER == 2) {
        // face average corrected along the centre-to-centre direction (derivative.c:71-89)
        Prim<R> ql = reload_prim<R>(q, N, c.x);
        Prim<R> qr = reload_prim<R>(q, N, c.y);
        Basis<R> b = reload_basis(g.basis, F, f);
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
        V3<R> unit = load_v3(g.corr, F, f);
        R norm = __ldg(g.corr + 3 * F + f);
#pragma unroll
        for (int v = 0; v < 5; v++) {
            V3<R> gv = v3(gm[3 * v], gm[3 * v + 1], gm[3 * v + 2]);
            R adjust = dot(gv, unit) - ((qrv[v] - qlv[v]) / norm);
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
        Cons<R> fv = viscous_central(prim_from(qm), gg, gamma, mu, prandtl, b);
        gf[0] -= fv.rho * area;
        gf[1] -= fv.m.x * area;
        gf[2] -= fv.m.y * area;
        gf[3] -= fv.m.z * area;
        gf[4] -= fv.e * area;
    }
    flux_rec_store(G, f, gf);
}

}  // namespace tg
