// Face-flux kernel: reconstruction, viscous and convective flux of one face per thread.
#pragma once

#include "common.cuh"

namespace tg {

// ---- face fluxes (src/equations/derivative.c:18-227) ------------------------------------------
//
// Writes G[v][f] = (convective - viscous) flux * area; the cell gather adds G to the left cell and
// subtracts it from the right one, as teal's face loops do.
template <typename R>
__device__ __forceinline__ void load_grad(const R *__restrict__ grad, int C, int c, R (&g)[15])
{
#pragma unroll
    for (int k = 0; k < 15; k++) {
        g[k] = __ldg(grad + k * C + c);
    }
}

template <typename R, int FK, bool NS, int ORDER, bool FOLD>
__global__ void __launch_bounds__(BLOCK) k_face(Sizes s, Geometry<R> g, const double *__restrict__ q,
                                                const R *__restrict__ grad, const R *__restrict__ psi,
                                                R gamma, R mu, R prandtl, R *__restrict__ G)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= s.F) {
        return;
    }
    const int F = s.F, C = s.C, N = s.N;
    const bool boundary = (f >= s.F_in) && (f < s.F_bd);
    int2 c = g.lr[f];
    Prim<R> ql = load_prim<R>(q, N, c.x);
    Prim<R> qr = load_prim<R>(q, N, c.y);
    Basis<R> b = load_basis(g.basis, F, f);
    R area = __ldg(g.area + f);

    Cons<R> fv{R(0), v3(R(0), R(0), R(0)), R(0)};
    Cons<R> fc{R(0), v3(R(0), R(0), R(0)), R(0)};

    if (ORDER == 1) {
        if (FK != FK_NONE) {
            fc = convective_flux<FK>(ql, qr, gamma, b);
        }
    }
    else {
        R gl[15], gr[15];
        load_grad(grad, C, c.x, gl);
        if (!boundary) {
            load_grad(grad, C, c.y, gr);
        }
        if (NS) {
            // face average corrected along the centre-to-centre direction (derivative.c:71-89)
            R qlv[5] = {ql.rho, ql.u.x, ql.u.y, ql.u.z, ql.p};
            R qrv[5] = {qr.rho, qr.u.x, qr.u.y, qr.u.z, qr.p};
            R qm[5], gm[15];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                qm[v] = (qlv[v] + qrv[v]) / R(2);
            }
#pragma unroll
            for (int k = 0; k < 15; k++) {
                gm[k] = boundary ? gl[k] : (gl[k] + gr[k]) / R(2);
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
            fv = viscous_central(prim_from(qm), gg, gamma, mu, prandtl, b);
        }
        if (FK != FK_NONE) {
            // reconstruct with the limited gradient (derivative.c:158-164, :191-224)
            V3<R> ol = load_v3(g.offl, F, f);
            R pl[5], pr[5];
            R ps[5];
            if (!FOLD) {
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    ps[v] = __ldg(psi + v * C + c.x);
                }
            }
            R qlv[5] = {ql.rho, ql.u.x, ql.u.y, ql.u.z, ql.p};
#pragma unroll
            for (int v = 0; v < 5; v++) {
                V3<R> gv = v3(gl[3 * v], gl[3 * v + 1], gl[3 * v + 2]);
                if (!FOLD) {
                    gv = v3(gv.x * ps[v], gv.y * ps[v], gv.z * ps[v]);
                }
                pl[v] = qlv[v] + dot(gv, ol);
            }
            R qrv[5] = {qr.rho, qr.u.x, qr.u.y, qr.u.z, qr.p};
            if (boundary) {
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    pr[v] = qrv[v];
                }
            }
            else {
                V3<R> orr = load_v3(g.offr, F, f);
                if (!FOLD) {
#pragma unroll
                    for (int v = 0; v < 5; v++) {
                        ps[v] = __ldg(psi + v * C + c.y);
                    }
                }
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    V3<R> gv = v3(gr[3 * v], gr[3 * v + 1], gr[3 * v + 2]);
                    if (!FOLD) {
                        gv = v3(gv.x * ps[v], gv.y * ps[v], gv.z * ps[v]);
                    }
                    pr[v] = qrv[v] + dot(gv, orr);
                }
            }
            fc = convective_flux<FK>(prim_from(pl), prim_from(pr), gamma, b);
        }
    }

    G[f] = (fc.rho * area) - (fv.rho * area);
    G[F + f] = (fc.m.x * area) - (fv.m.x * area);
    G[2 * F + f] = (fc.m.y * area) - (fv.m.y * area);
    G[3 * F + f] = (fc.m.z * area) - (fv.m.z * area);
    G[4 * F + f] = (fc.e * area) - (fv.e * area);
}

}  // namespace tg
