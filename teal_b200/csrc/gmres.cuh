// Kernels of the implicit Euler step with a Jacobian-free Newton-GMRES solve
// (src/simulation/advance.c:119-195, src/simulation/gmres.c:12-149), for every instance of an
// arena at once. Vectors are the conserved state of the inner cells, [5][C] over the arena; each
// instance has its own scalars (norms, step, finite-difference scale, Hessenberg matrix, Givens
// rotations, right-hand side, coefficients) and its own Newton / Arnoldi progress, so instances
// converge independently: a finished instance is masked out of the vector updates. Dot products
// and norms are per-piece partial sums, then per-instance sums in piece order: deterministic, and
// the same bits for an instance alone or in a batch.
#pragma once

#include "kernels.cuh"

namespace tg {

// scalar slots of an instance's block in the device scalar array
enum GmresScalar {
    GS_NORM = 0,       // Newton residual norm
    GS_CONS_NORM = 1,  // norm of the conserved state
    GS_FD_SCALE = 2,   // finite-difference scale
    GS_VNORM = 3,      // norm of the Krylov vector being multiplied
    GS_STEP = 4,       // time step
    GS_KTOL = 5,       // Krylov tolerance * norm
    GS_TOL_NORM = 6,   // Newton tolerance * first norm
    GS_HEAD = 8        // H [(dim+1) x dim], cs [dim], sn [dim], rhs [dim+1], coef [dim]
};

// per-instance flags: Newton iterating, Arnoldi iterating, Krylov vectors used, Newton iterations
enum GmresFlag { GF_NEWTON = 0, GF_ARNOLDI = 1, GF_M = 2, GF_ITER = 3, GF_COUNT = 4 };

// device loop counters of the graph-driven solve: the Arnoldi column k, the Gram-Schmidt row i and
// the Newton iterations of the current step
enum GmresControl { GC_K = 0, GC_I = 1, GC_N = 2, GC_COUNT = 3 };

// Newton iterations one implicit step may take on the device before it stops with ERR_LOOP_LIMIT
// (teal's own bound, 128 (cells + 1) per instance, advance.c:162, stays in force below it); the
// bound keeps every device loop of the step graph finite
constexpr int NEWTON_LOOP_LIMIT = 1000;

struct GmresBatch {
    int dim;    // Krylov dimension
    int scn;    // doubles per instance block of `sc`
    int ninst;
    const int *__restrict__ cell_inst;
    double *sc;  // [ninst][scn]
    int *flag;   // [GF_COUNT][ninst]
    int *count;  // [2] instances still iterating (Newton, Arnoldi)
    int *ctl;    // [GC_COUNT] loop counters read by the kernels of one Arnoldi iteration

    __device__ __forceinline__ double *s(int i) const { return sc + (size_t)i * scn; }
    __device__ __forceinline__ double *H(int i, int r, int k) const { return s(i) + GS_HEAD + r * dim + k; }
    __device__ __forceinline__ double *cs(int i) const { return s(i) + GS_HEAD + (dim + 1) * dim; }
    __device__ __forceinline__ double *sn(int i) const { return cs(i) + dim; }
    __device__ __forceinline__ double *rhs(int i) const { return sn(i) + dim; }
    __device__ __forceinline__ double *coef(int i) const { return rhs(i) + dim + 1; }
    __device__ __forceinline__ int &newton(int i) const { return flag[GF_NEWTON * ninst + i]; }
    __device__ __forceinline__ int &arnoldi(int i) const { return flag[GF_ARNOLDI * ninst + i]; }
    __device__ __forceinline__ int &m(int i) const { return flag[GF_M * ninst + i]; }
    __device__ __forceinline__ int &iter(int i) const { return flag[GF_ITER * ninst + i]; }
};

__host__ __device__ inline int gmres_scn(int dim)
{
    return GS_HEAD + (dim + 1) * dim + 4 * dim + 2;
}

// per-piece partial sums of x . y over the 5 variables of the piece's cells; pieces of instances
// whose flag `which` is off are skipped (their sums are not read)
__global__ void __launch_bounds__(BLOCK) k_piece_dot(Segments seg, int C, const double *__restrict__ x,
                                                     const double *__restrict__ y, GmresBatch gb, int which,
                                                     double *__restrict__ part)
{
    __shared__ double sh[BLOCK / 32];
    const int beg = seg.piece_beg[blockIdx.x], end = seg.piece_beg[blockIdx.x + 1];
    if (!gb.flag[which * gb.ninst + gb.cell_inst[beg]]) {
        return;
    }
    double t = 0;
    for (int c = beg + threadIdx.x; c < end; c += BLOCK) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
            t += x[(size_t)v * C + c] * y[(size_t)v * C + c];
        }
    }
    double sum = block_sum<BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sum;
    }
}

constexpr int GM_INST_BLOCK = 128;

// sc[inst][slot] = sum of the instance's piece partials (or its square root), for instances whose
// flag `which` is set
__global__ void __launch_bounds__(GM_INST_BLOCK) k_inst_dot(Segments seg, const double *__restrict__ part,
                                                           GmresBatch gb, int which, int slot, int take_sqrt)
{
    __shared__ double sh[GM_INST_BLOCK / 32];
    const int i = blockIdx.x;
    if (!gb.flag[which * gb.ninst + i]) {
        return;
    }
    double t = 0;
    for (int p = seg.inst_piece_off[i] + threadIdx.x; p < seg.inst_piece_off[i + 1]; p += GM_INST_BLOCK) {
        t += part[p];
    }
    double sum = block_sum<GM_INST_BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        gb.s(i)[slot] = take_sqrt ? sqrt(sum) : sum;
    }
}

// start of a step for every instance: Newton flag on for the active ones, step copied
__global__ void k_newton_begin(GmresBatch gb, Steps st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gb.ninst) {
        return;
    }
    const int on = st.active[i] != 0;
    gb.newton(i) = on;
    gb.arnoldi(i) = 0;
    gb.m(i) = 0;
    gb.iter(i) = 0;
    if (on) {
        gb.s(i)[GS_STEP] = st.step[i];
    }
}

// r = -R * step (advance.c:148-153)
__global__ void k_newton_init(int C, const double *__restrict__ R, GmresBatch gb, double *__restrict__ r)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.newton(i)) {
        return;
    }
    const double step = gb.s(i)[GS_STEP];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        r[(size_t)v * C + c] = -R[(size_t)v * C + c] * step;
    }
}

// r = U - U0 - R * step (advance.c:176-181)
__global__ void k_newton_residual(int C, const double *__restrict__ U, const double *__restrict__ U0,
                                  const double *__restrict__ R, GmresBatch gb, double *__restrict__ r)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.newton(i)) {
        return;
    }
    const double step = gb.s(i)[GS_STEP];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        size_t k = (size_t)v * C + c;
        r[k] = (U[k] - U0[k]) - (R[k] * step);
    }
}

// fd_scale = fd_rel * max(1, |U|) / max(1, |r|) (advance.c:155-159, fd_rel = 1e-6 there); on the
// first call of a step also the Newton target tol * |r|
__global__ void k_fd_scale(GmresBatch gb, double fd_rel, double newton_tol, int first)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gb.ninst || !gb.newton(i)) {
        return;
    }
    double *s = gb.s(i);
    s[GS_FD_SCALE] = fd_rel * fmax(1.0, s[GS_CONS_NORM]) / fmax(1.0, s[GS_NORM]);
    if (first) {
        s[GS_TOL_NORM] = newton_tol * s[GS_NORM];
    }
}

// Newton loop test per instance (advance.c:162-165): keep iterating while |r| > tol * |r0| and
// within 128 (cells + 1) iterations; a non-finite norm marks the instance failed. count[0] = instances
// that go on.
__global__ void k_newton_check(GmresBatch gb, Segments seg, Steps st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gb.ninst || !gb.newton(i)) {
        return;
    }
    const double norm = gb.s(i)[GS_NORM];
    if (!isfinite(norm)) {  // the instance stops (its residual follows as non-finite); the others go on
        atomicOr(st.error, ERR_NONFINITE);
        st.fail[i] = 1;
        gb.newton(i) = 0;
        return;
    }
    const long max_iter = 128L * (seg.inst_cell_off[i + 1] - seg.inst_cell_off[i] + 1);
    const long it = gb.iter(i);
    if (!(norm > gb.s(i)[GS_TOL_NORM]) || it >= max_iter) {
        gb.newton(i) = 0;
        return;
    }
    atomicAdd(&gb.count[0], 1);
}

// start of a GMRES cycle (gmres.c:68-83) per Newton instance: rhs = (norm, 0, ...), Arnoldi on
// unless the residual is already zero
__global__ void k_gmres_begin(GmresBatch gb, double krylov_tol)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gb.ninst) {
        return;
    }
    gb.arnoldi(i) = 0;
    gb.m(i) = 0;
    if (!gb.newton(i)) {
        return;
    }
    double *s = gb.s(i);
    const double norm = s[GS_NORM];
    double *rhs = gb.rhs(i);
    for (int k = 0; k <= gb.dim; k++) {
        rhs[k] = 0.0;
    }
    rhs[0] = norm;
    s[GS_KTOL] = krylov_tol * norm;
    gb.arnoldi(i) = norm > 0;
    gb.iter(i) += 1;
}

// V0 = -r / norm and delta = 0 for every Newton instance (delta stays 0 when the norm is 0)
__global__ void k_gmres_start(int C, const double *__restrict__ r, GmresBatch gb, double *__restrict__ V0,
                              double *__restrict__ delta)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.newton(i)) {
        return;
    }
    const double norm = gb.s(i)[GS_NORM];
    const bool on = gb.arnoldi(i) != 0;
#pragma unroll
    for (int v = 0; v < 5; v++) {
        size_t k = (size_t)v * C + c;
        if (on) {
            V0[k] = -r[k] / norm;
        }
        delta[k] = 0.0;
    }
}

// back substitution coefficients for the instance's m Krylov vectors (gmres.c:128-136)
__global__ void k_backsolve(GmresBatch gb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gb.ninst || !gb.newton(i)) {
        return;
    }
    const int m = gb.m(i);
    double *rhs = gb.rhs(i), *coef = gb.coef(i);
    for (int r = m - 1; r >= 0; r--) {
        double cr = rhs[r];
        for (int j = r + 1; j < m; j++) {
            cr -= *gb.H(i, r, j) * coef[j];
        }
        coef[r] = cr / *gb.H(i, r, r);
    }
}

// delta += coef[r] * V_r, r from m-1 down to 0 in one pass (gmres.c:137-141)
__global__ void k_accumulate(int C, const double *__restrict__ V, GmresBatch gb, double *__restrict__ delta)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.newton(i)) {
        return;
    }
    const int m = gb.m(i);
    const double *coef = gb.coef(i);
    const size_t n = 5 * (size_t)C;
#pragma unroll
    for (int v = 0; v < 5; v++) {
        size_t j = (size_t)v * C + c;
        double d = delta[j];
        for (int r = m - 1; r >= 0; r--) {
            d += coef[r] * V[(size_t)r * n + j];
        }
        delta[j] = d;
    }
}

// U += delta, q = prim(U) (advance.c:168-173)
__global__ void k_newton_update(int C, int N, double *__restrict__ U, const double *__restrict__ delta,
                                GmresBatch gb, double gamma, double *__restrict__ q)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    if (!gb.newton(gb.cell_inst[c])) {
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

// ---- device-driven loops ------------------------------------------------------------------------
//
// The implicit step runs from one CUDA graph whose Newton, Arnoldi and Gram-Schmidt loops are
// conditional WHILE nodes: the kernels below read the loop counters (GmresBatch::ctl) from device
// memory instead of taking them as launch arguments, and the last kernel of each loop body sets
// the loop's condition, so no iteration waits for the host. Each kernel does the same arithmetic
// in the same order as the host-driven sequence it replaces, so the results keep their bits.

// Newton loop condition: go on while some instance iterates (count[0], set by k_newton_check) and
// the step's iterations stay below NEWTON_LOOP_LIMIT; `enter` starts the count of the step
__global__ void k_newton_next(GmresBatch gb, cudaGraphConditionalHandle h, int enter, int *err)
{
    const int n = enter ? 0 : gb.ctl[GC_N] + 1;
    gb.ctl[GC_N] = n;
    const bool going = gb.count[0] > 0;
    if (going && n >= NEWTON_LOOP_LIMIT) {
        atomicOr(err, ERR_LOOP_LIMIT);
    }
    cudaGraphSetConditional(h, (going && n < NEWTON_LOOP_LIMIT) ? 1u : 0u);
}

// start of an Arnoldi loop: k = 0; count[1] = instances whose Arnoldi flag is set; the loop's
// condition from it
__global__ void k_arnoldi_enter(GmresBatch gb, cudaGraphConditionalHandle h)
{
    __shared__ int n;
    if (threadIdx.x == 0) {
        n = 0;
        gb.ctl[GC_K] = 0;
    }
    __syncthreads();
    int t = 0;
    for (int i = threadIdx.x; i < gb.ninst; i += blockDim.x) {
        t += gb.arnoldi(i) != 0;
    }
    atomicAdd(&n, t);
    __syncthreads();
    if (threadIdx.x == 0) {
        cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
    }
}

// start of the Gram-Schmidt loop of column k: i = 0, condition on (the body runs at least once)
__global__ void k_mgs_enter(GmresBatch gb, cudaGraphConditionalHandle h)
{
    gb.ctl[GC_I] = 0;
    cudaGraphSetConditional(h, 1u);
}

// per-piece partials of V_k . V_k (the norm of the vector being multiplied, gmres.c:26)
__global__ void __launch_bounds__(BLOCK) k_piece_vnorm(Segments seg, int C, const double *__restrict__ V,
                                                       GmresBatch gb, double *__restrict__ part)
{
    __shared__ double sh[BLOCK / 32];
    const double *x = V + (size_t)gb.ctl[GC_K] * 5 * (size_t)C;
    const int beg = seg.piece_beg[blockIdx.x], end = seg.piece_beg[blockIdx.x + 1];
    if (!gb.arnoldi(gb.cell_inst[beg])) {  // the instance left its Arnoldi loop
        return;
    }
    double t = 0;
    for (int c = beg + threadIdx.x; c < end; c += BLOCK) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
            t += x[(size_t)v * C + c] * x[(size_t)v * C + c];
        }
    }
    double sum = block_sum<BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sum;
    }
}

// One Gram-Schmidt row fused with the update of the row before it (gmres.c:92-99): with i > 0,
// w -= H[i-1][k] V_{i-1} for the cells of Arnoldi instances, then the per-piece partials of
// V_i . w; after the last row (`last`), w -= H[k][k] V_k and the partials of w . w.
__global__ void __launch_bounds__(BLOCK) k_mgs_piece(Segments seg, int C, const double *__restrict__ V,
                                                     GmresBatch gb, int last, double *__restrict__ w,
                                                     double *__restrict__ part)
{
    __shared__ double sh[BLOCK / 32];
    const size_t n = 5 * (size_t)C;
    const int k = gb.ctl[GC_K];
    const int i = last ? k + 1 : gb.ctl[GC_I];
    const int beg = seg.piece_beg[blockIdx.x], end = seg.piece_beg[blockIdx.x + 1];
    const int inst = gb.cell_inst[beg];  // a piece lies in one instance
    if (!gb.arnoldi(inst)) {  // the instance left its Arnoldi loop: nothing to update or sum
        return;
    }
    const bool update = i > 0;
    const double h = update ? *gb.H(inst, i - 1, k) : 0.0;
    const double *Vp = V + (size_t)(i > 0 ? i - 1 : 0) * n;
    const double *x = last ? w : V + (size_t)i * n;
    double t = 0;
    for (int c = beg + threadIdx.x; c < end; c += BLOCK) {
        if (update) {
#pragma unroll
            for (int v = 0; v < 5; v++) {
                size_t j = (size_t)v * C + c;
                w[j] -= h * Vp[j];
            }
        }
#pragma unroll
        for (int v = 0; v < 5; v++) {
            size_t j = (size_t)v * C + c;
            t += x[j] * w[j];
        }
    }
    double sum = block_sum<BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sum;
    }
}

// instance sums of the piece partials into H[row][k] (row: i, or k + 1 with the square root) or the
// vector norm slot, for the Arnoldi instances; slot kinds: 0 = H[i][k], 1 = H[k+1][k] = sqrt, 2 =
// GS_VNORM = sqrt
__global__ void __launch_bounds__(GM_INST_BLOCK) k_inst_dot_at(Segments seg, const double *__restrict__ part,
                                                              GmresBatch gb, int kind)
{
    __shared__ double sh[GM_INST_BLOCK / 32];
    const int i = blockIdx.x;
    if (!gb.arnoldi(i)) {
        return;
    }
    double t = 0;
    for (int p = seg.inst_piece_off[i] + threadIdx.x; p < seg.inst_piece_off[i + 1]; p += GM_INST_BLOCK) {
        t += part[p];
    }
    double sum = block_sum<GM_INST_BLOCK>(t, sh);
    if (threadIdx.x == 0) {
        const int k = gb.ctl[GC_K];
        if (kind == 0) {
            *gb.H(i, gb.ctl[GC_I], k) = sum;
        }
        else if (kind == 1) {
            *gb.H(i, k + 1, k) = sqrt(sum);
        }
        else {
            gb.s(i)[GS_VNORM] = sqrt(sum);
        }
    }
}

// next Gram-Schmidt row: i += 1; go on while i <= k
__global__ void k_mgs_next(GmresBatch gb, cudaGraphConditionalHandle h)
{
    const int i = gb.ctl[GC_I] + 1;
    gb.ctl[GC_I] = i;
    cudaGraphSetConditional(h, (i <= gb.ctl[GC_K] && i < gb.dim) ? 1u : 0u);
}

// next Arnoldi column: k += 1; go on while some instance iterates (count[1], set by k_givens_at),
// at most `dim` columns (k_givens_at already stops every instance there)
__global__ void k_arnoldi_next(GmresBatch gb, cudaGraphConditionalHandle h)
{
    const int k = gb.ctl[GC_K] + 1;
    gb.ctl[GC_K] = k;
    cudaGraphSetConditional(h, (gb.count[1] > 0 && k < gb.dim) ? 1u : 0u);
}

// The matvec, Givens and normalisation steps of Arnoldi column k (k read from the device):
// perturbed primitive state q1 = prim(U + eps V_k), eps = fd_scale / |V_k| (gmres.c:26-36)
__global__ void k_perturb_at(int C, int N, const double *__restrict__ U, const double *__restrict__ V,
                             GmresBatch gb, double gamma, double *__restrict__ q1)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.arnoldi(i)) {
        return;
    }
    const double *v = V + (size_t)gb.ctl[GC_K] * 5 * (size_t)C;
    const double eps = gb.s(i)[GS_FD_SCALE] / gb.s(i)[GS_VNORM];
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

// w = V_k - step (R1 - R) / eps (gmres.c:41-46)
__global__ void k_matvec_finish_at(int C, const double *__restrict__ V, const double *__restrict__ R1,
                                   const double *__restrict__ R, GmresBatch gb, double *__restrict__ w)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.arnoldi(i)) {
        return;
    }
    const double *v = V + (size_t)gb.ctl[GC_K] * 5 * (size_t)C;
    const double *s = gb.s(i);
    const double eps = s[GS_FD_SCALE] / s[GS_VNORM];
    const double step = s[GS_STEP];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        size_t j = (size_t)k * C + c;
        w[j] = v[j] - ((step * (R1[j] - R[j])) / eps);
    }
}

// Givens rotations of column k, new rotation, right-hand side and convergence test per Arnoldi
// instance (gmres.c:102-119); an instance that converged (or filled the basis) stops with m = k + 1;
// count[1] = instances that go on
__global__ void k_givens_at(GmresBatch gb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = gb.ctl[GC_K];
    if (i >= gb.ninst || !gb.arnoldi(i)) {
        return;
    }
    double *cs = gb.cs(i), *sn = gb.sn(i), *rhs = gb.rhs(i);
    for (int r = 0; r < k; r++) {
        double hrk = *gb.H(i, r, k), hr1k = *gb.H(i, r + 1, k);
        double tmp = (cs[r] * hrk) + (sn[r] * hr1k);
        *gb.H(i, r + 1, k) = (-sn[r] * hrk) + (cs[r] * hr1k);
        *gb.H(i, r, k) = tmp;
    }
    double hkk = *gb.H(i, k, k), hk1k = *gb.H(i, k + 1, k);
    double rot = sqrt((hkk * hkk) + (hk1k * hk1k));
    cs[k] = hkk / rot;
    sn[k] = hk1k / rot;
    *gb.H(i, k, k) = rot;
    rhs[k + 1] = -sn[k] * rhs[k];
    rhs[k] = cs[k] * rhs[k];
    gb.m(i) = k + 1;
    if (fabs(rhs[k + 1]) < gb.s(i)[GS_KTOL] || k + 1 >= gb.dim) {
        gb.arnoldi(i) = 0;
        return;
    }
    atomicAdd(&gb.count[1], 1);
}

// V_{k+1} = w / H[k+1][k] (gmres.c:121-125)
__global__ void k_normalize_at(int C, const double *__restrict__ w, GmresBatch gb, double *__restrict__ V)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) {
        return;
    }
    const int i = gb.cell_inst[c];
    if (!gb.arnoldi(i)) {
        return;
    }
    const int k = gb.ctl[GC_K];
    double *Vk1 = V + (size_t)(k + 1) * 5 * (size_t)C;
    const double h = *gb.H(i, k + 1, k);
#pragma unroll
    for (int v = 0; v < 5; v++) {
        size_t j = (size_t)v * C + c;
        Vk1[j] = w[j] / h;
    }
}

}  // namespace tg
