// Stage kernels (boundary, gradient + limiter, cell gather + RK stage, preparation) with teal's
// exact FP64 arithmetic: compiled with TG_EXACT_TU=1 and -fmad=false (see physics.cuh). Together
// with face_*_exact.cu they make the TG_PRECISION_FP64_EXACT form, which reproduces teal's
// explicit residuals and steps bit for bit.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace tg {

static_assert(kExact, "stage_exact.cu is compiled with TG_EXACT_TU=1");

template <bool MIXED>
static void gradient_m(const GradientLaunch &a, cudaStream_t st)
{
    if (a.s.hi <= a.s.lo) return;
    dim3 grid((a.s.hi - a.s.lo + GRAD_CELLS - 1) / GRAD_CELLS);
    switch (a.limiter) {
        case 0: k_gradient<double, 0, true, MIXED, true><<<grid, GRAD_THREADS, 0, st>>>(a.s, a.g, a.eps2, a.q, a.rec, a.err, a.polls); break;
        case 1:
            if (a.fold)
                k_gradient<double, 1, true, MIXED, true><<<grid, GRAD_THREADS, 0, st>>>(a.s, a.g, a.eps2, a.q, a.rec, a.err, a.polls);
            else
                k_gradient<double, 1, false, MIXED, true><<<grid, GRAD_THREADS, 0, st>>>(a.s, a.g, a.eps2, a.q, a.rec, a.err, a.polls);
            break;
        default:
            if (a.fold)
                k_gradient<double, 2, true, MIXED, true><<<grid, GRAD_THREADS, 0, st>>>(a.s, a.g, a.eps2, a.q, a.rec, a.err, a.polls);
            else
                k_gradient<double, 2, false, MIXED, true><<<grid, GRAD_THREADS, 0, st>>>(a.s, a.g, a.eps2, a.q, a.rec, a.err, a.polls);
            break;
    }
}

cudaError_t launch_gradient_exact(const GradientLaunch &a, cudaStream_t st)
{
    if (a.mixed)
        gradient_m<true>(a, st);
    else
        gradient_m<false>(a, st);
    return cudaGetLastError();
}

template <int MODE, bool NS, int SRC>
static void cell_s(const CellLaunch &a, cudaStream_t st)
{
    if (a.s.hi <= a.s.lo) return;
    k_cell<MODE, NS, double, SRC, true><<<(a.s.hi - a.s.lo + CELL_BLOCK - 1) / CELL_BLOCK, CELL_BLOCK, 0, st>>>(
        a.s, a.slot_face, a.slot_cnt, a.cd, a.G, a.U0, a.q, a.Rout, a.seg, a.st, a.alpha, a.last, a.prop, a.dtc,
        a.src, a.two);
}

template <int MODE, bool NS>
static void cell_n(const CellLaunch &a, cudaStream_t st)
{
    switch (a.source) {
        case 1: cell_s<MODE, NS, 1>(a, st); break;
        case 2: cell_s<MODE, NS, 2>(a, st); break;
        case 3: cell_s<MODE, NS, 3>(a, st); break;
        default: cell_s<MODE, NS, 0>(a, st); break;
    }
}

cudaError_t launch_cell_exact(const CellLaunch &a, cudaStream_t st)
{
    if (a.mode == 0) {
        if (a.ns)
            cell_n<0, true>(a, st);
        else
            cell_n<0, false>(a, st);
    }
    else {
        if (a.ns)
            cell_n<1, true>(a, st);
        else
            cell_n<1, false>(a, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_prepare_exact(bool ns, Sizes s, CellData cd, const double *q, double *U0, Props prop, double *dtc,
                                 cudaStream_t st)
{
    const int grid = (s.C + BLOCK - 1) / BLOCK;
    if (ns)
        k_prepare<true, true><<<grid, BLOCK, 0, st>>>(s, cd, q, U0, prop, dtc);
    else
        k_prepare<false, true><<<grid, BLOCK, 0, st>>>(s, cd, q, U0, prop, dtc);
    return cudaGetLastError();
}

cudaError_t launch_boundary_exact(const BoundaryLaunch &a, cudaStream_t st)
{
    const int nbf = a.s.F_bd - a.s.F_in;
    k_boundary<true><<<(nbf + BLOCK - 1) / BLOCK, BLOCK, 0, st>>>(a.s, a.lr, a.basis, a.bface_ent, a.bkind, a.bctx,
                                                                  a.q, a.gamma, a.cell_inst, a.active);
    return cudaGetLastError();
}

}  // namespace tg
