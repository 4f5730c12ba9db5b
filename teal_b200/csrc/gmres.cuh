// Kernels of the implicit Euler step with a Jacobian-free Newton-GMRES solve
// (src/simulation/advance.c:119-195, src/simulation/gmres.c:12-149). Vectors are the conserved
// state of the inner cells, [5][C] flattened to n = 5C; dot products and norms are deterministic
// block-partial reductions; Arnoldi, Givens rotations and back substitution run on the device.
#pragma once

#include "kernels.cuh"

namespace tg {

// scalar slots of the device scalar array
enum GmresScalar {
    GS_NORM = 0,      // Newton residual norm
    GS_CONS_NORM = 1, // norm of the conserved state
    GS_FD_SCALE = 2,  // finite-difference scale
    GS_VNORM = 3,     // norm of the Krylov vector being multiplied
    GS_STEP = 4,      // time step
    GS_KTOL = 5,      // Krylov tolerance * norm
    GS_DONE = 6,      // Arnoldi stopped early
    GS_DOT = 7,       // last dot product
    GS_HEAD = 16      // H [(dim+1) x dim], cs [dim], sn [dim], rhs [dim+1], coef [dim]
};

__device__ __forceinline__ double *gm_H(double *sc, int dim, int i, int k)
{
    return sc + GS_HEAD + i * dim + k;
}

// partial sums of x . y over n elements
__global__ void __launch_bounds__(BLOCK) k_dot_part(long n, const double *__restrict__ x,
                                                    const double *__restrict__ y, double *__restrict__ part)
{
    __shared__ double sh[BLOCK / 32];
    double t = 0;
    for (long i = blockIdx.x * (long)BLOCK + threadIdx.x; i < n; i += (long)gridDim.x * BLOCK) {
        t += x[i] * y[i];
    }
    double s = block_sum<BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
    }
}

// dst = sum of partials (optionally its square root)
__global__ void __launch_bounds__(REDUCE_BLOCK) k_reduce_scalar(const double *__restrict__ part, int nparts,
                                                                double *dst, int take_sqrt)
{
    __shared__ double sh[REDUCE_BLOCK / 32];
    double t = 0;
    for (int i = threadIdx.x; i < nparts; i += REDUCE_BLOCK) {
        t += part[i];
    }
    double s = block_sum<REDUCE_BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        *dst = take_sqrt ? sqrt(s) : s;
    }
}

// r = -R * step (advance.c:148-153)
__global__ void k_newton_init(long n, const double *__restrict__ R, const double *__restrict__ sc,
                              double *__restrict__ r)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) {
        r[i] = -R[i] * sc[GS_STEP];
    }
}

// r = U - U0 - R * step (advance.c:176-181)
__global__ void k_newton_residual(long n, const double *__restrict__ U, const double *__restrict__ U0,
                                  const double *__restrict__ R, const double *__restrict__ sc,
                                  double *__restrict__ r)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) {
        r[i] = (U[i] - U0[i]) - (R[i] * sc[GS_STEP]);
    }
}

// fd_scale = 1e-6 * max(1, |U|) / max(1, |r|) (advance.c:155-159)
__global__ void k_fd_scale(double *sc)
{
    sc[GS_FD_SCALE] = 1e-6 * fmax(1.0, sc[GS_CONS_NORM]) / fmax(1.0, sc[GS_NORM]);
}

// start of a GMRES cycle (gmres.c:68-83): V0 = -r / norm, rhs = (norm, 0, ...), delta = 0
__global__ void k_gmres_start(long n, int dim, const double *__restrict__ r, double *__restrict__ V0,
                              double *__restrict__ delta, double *sc, double krylov_tol)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    double norm = sc[GS_NORM];
    if (i < n) {
        V0[i] = -r[i] / norm;
        delta[i] = 0.0;
    }
    if (i == 0) {
        double *rhs = sc + GS_HEAD + (dim + 1) * dim + 2 * dim;
        for (int k = 0; k <= dim; k++) {
            rhs[k] = 0.0;
        }
        rhs[0] = norm;
        sc[GS_KTOL] = krylov_tol * norm;
        sc[GS_DONE] = 0.0;
    }
}

// perturbed primitive state q1 = prim(U + eps * v), eps = fd_scale / |v| (gmres.c:26-36)
__global__ void k_perturb(int C, int N, const double *__restrict__ U, const double *__restrict__ v,
                          const double *__restrict__ sc, double gamma, double *__restrict__ q1)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    double eps = sc[GS_FD_SCALE] / sc[GS_VNORM];
    Cons<double> u;
    u.rho = U[c] + (eps * v[c]);
    u.m.x = U[C + c] + (eps * v[C + c]);
    u.m.y = U[2 * C + c] + (eps * v[2 * C + c]);
    u.m.z = U[3 * C + c] + (eps * v[3 * C + c]);
    u.e = U[4 * C + c] + (eps * v[4 * C + c]);
    Prim<double> p = cons_to_prim(u, gamma);
    q1[c] = p.rho;
    q1[N + c] = p.u.x;
    q1[2 * N + c] = p.u.y;
    q1[3 * N + c] = p.u.z;
    q1[4 * N + c] = p.p;
}

// w = v - step * (R1 - R) / eps (gmres.c:41-46)
__global__ void k_matvec_finish(long n, const double *__restrict__ v, const double *__restrict__ R1,
                                const double *__restrict__ R, const double *__restrict__ sc,
                                double *__restrict__ w)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) {
        double eps = sc[GS_FD_SCALE] / sc[GS_VNORM];
        w[i] = v[i] - ((sc[GS_STEP] * (R1[i] - R[i])) / eps);
    }
}

// store a dot product into H[i][k]
__global__ void k_store_h(double *sc, int dim, int i, int k)
{
    *gm_H(sc, dim, i, k) = sc[GS_DOT];
}

// modified Gram-Schmidt update w -= H[i][k] * V_i (gmres.c:92-99)
__global__ void k_mgs_axpy(long n, const double *__restrict__ Vi, const double *__restrict__ sc, int dim,
                           int i, int k, double *__restrict__ w)
{
    long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (j < n) {
        double h = sc[GS_HEAD + i * dim + k];
        w[j] -= h * Vi[j];
    }
}

// Givens rotations of column k, new rotation, right-hand side, convergence test (gmres.c:102-119)
__global__ void k_givens(double *sc, int dim, int k)
{
    double *cs = sc + GS_HEAD + (dim + 1) * dim;
    double *sn = cs + dim;
    double *rhs = sn + dim;
    for (int i = 0; i < k; i++) {
        double hik = *gm_H(sc, dim, i, k), hi1k = *gm_H(sc, dim, i + 1, k);
        double tmp = (cs[i] * hik) + (sn[i] * hi1k);
        *gm_H(sc, dim, i + 1, k) = (-sn[i] * hik) + (cs[i] * hi1k);
        *gm_H(sc, dim, i, k) = tmp;
    }
    double hkk = *gm_H(sc, dim, k, k), hk1k = *gm_H(sc, dim, k + 1, k);
    double rot = sqrt((hkk * hkk) + (hk1k * hk1k));
    cs[k] = hkk / rot;
    sn[k] = hk1k / rot;
    *gm_H(sc, dim, k, k) = rot;
    rhs[k + 1] = -sn[k] * rhs[k];
    rhs[k] = cs[k] * rhs[k];
    sc[GS_DONE] = (fabs(rhs[k + 1]) < sc[GS_KTOL]) ? 1.0 : 0.0;
}

// V_{k+1} = w / H[k+1][k] (gmres.c:121-125)
__global__ void k_normalize(long n, const double *__restrict__ w, const double *__restrict__ sc, int dim,
                            int k, double *__restrict__ Vk1)
{
    long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (j < n) {
        Vk1[j] = w[j] / sc[GS_HEAD + (k + 1) * dim + k];
    }
}

// back substitution coefficients for m Krylov vectors (gmres.c:128-136)
__global__ void k_backsolve(double *sc, int dim, int m)
{
    double *rhs = sc + GS_HEAD + (dim + 1) * dim + 2 * dim;
    double *coef = rhs + dim + 1;
    for (int i = m - 1; i >= 0; i--) {
        double ci = rhs[i];
        for (int j = i + 1; j < m; j++) {
            ci -= *gm_H(sc, dim, i, j) * coef[j];
        }
        coef[i] = ci / *gm_H(sc, dim, i, i);
    }
}

// delta += coef[i] * V_i, i from m-1 down to 0 in one pass (gmres.c:137-141)
__global__ void k_accumulate(long n, const double *__restrict__ V, const double *__restrict__ sc, int dim,
                             int m, double *__restrict__ delta)
{
    long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (j >= n) {
        return;
    }
    const double *coef = sc + GS_HEAD + (dim + 1) * dim + 2 * dim + dim + 1;
    double d = delta[j];
    for (int i = m - 1; i >= 0; i--) {
        d += coef[i] * V[(long)i * n + j];
    }
    delta[j] = d;
}

// U += delta, q = prim(U) (advance.c:168-173)
__global__ void k_newton_update(int C, int N, double *__restrict__ U, const double *__restrict__ delta,
                                double gamma, double *__restrict__ q)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    Cons<double> u;
    u.rho = U[c] += delta[c];
    u.m.x = U[C + c] += delta[C + c];
    u.m.y = U[2 * C + c] += delta[2 * C + c];
    u.m.z = U[3 * C + c] += delta[3 * C + c];
    u.e = U[4 * C + c] += delta[4 * C + c];
    Prim<double> p = cons_to_prim(u, gamma);
    q[c] = p.rho;
    q[N + c] = p.u.x;
    q[2 * N + c] = p.u.y;
    q[3 * N + c] = p.u.z;
    q[4 * N + c] = p.p;
}

}  // namespace tg
