// Kernel launchers shared by the translation units. Face-flux kernels are instantiated per flux
// scheme in face_*.cu so the many template variants compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "face.cuh"

namespace tg {

struct FaceLaunch {
    Sizes s;
    const void *geom;  // Geometry<R>*
    const double *q;
    const void *rec;
    double gamma, mu, prandtl;
    void *G;
    int *err;  // device error word (bounded waits that give up set ERR_TIMEOUT)
    PressureRef pr_ref;  // FP32-flux form: reference pressure per instance
    int polls;           // limit of the staged kernel's first wait (MBAR_POLLS unless a test lowers it)
};

// The launchers below are local to each translation unit (unnamed namespace): the exact and the plain
// face translation units instantiate them with the same template arguments, and one shared
// definition would launch the other arithmetic's kernels.
namespace {

template <typename R, int FK, bool NS, int ORDER, bool FOLD>
inline void launch_face_v(bool staged, const FaceLaunch &a, const Geometry<R> &g, const R *rec, R *G, cudaStream_t st)
{
    constexpr bool X = kExact;
    if (a.s.hi <= a.s.lo) {
        return;
    }
    dim3 grid((a.s.hi - a.s.lo + FACE_BLOCK - 1) / FACE_BLOCK);
    R gm = R(a.gamma), mu = R(a.mu), pr = R(a.prandtl);
    PressureRefOf<R> pref{};
    if constexpr (sizeof(R) == sizeof(float)) {
        pref = a.pr_ref;
    }
    if (staged) {
        k_face_staged<R, FK, NS, ORDER, FOLD, X>
            <<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G, a.err, pref, a.polls);
    }
    else {
        k_face<R, FK, NS, ORDER, FOLD, X><<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G, pref);
    }
}

// staged geometry (bulk copies into shared memory) or thread loads, per physics (tuned.h)
template <int FK, typename R>
inline cudaError_t launch_face_r(bool ns, int order, bool fold, const FaceLaunch &a, cudaStream_t st)
{
    const Geometry<R> &g = *static_cast<const Geometry<R> *>(a.geom);
    const R *rec = static_cast<const R *>(a.rec);
    R *G = static_cast<R *>(a.G);
    const bool staged = ns ? (TG_FACE_STAGED_NS != 0) : (TG_FACE_STAGED_EULER != 0);
    if (order == 1) {
        launch_face_v<R, FK, false, 1, true>(staged, a, g, rec, G, st);
    }
    else if (!ns) {
        launch_face_v<R, FK, false, 2, true>(staged, a, g, rec, G, st);
    }
    else if (fold) {
        launch_face_v<R, FK, true, 2, true>(staged, a, g, rec, G, st);
    }
    else {
        launch_face_v<R, FK, true, 2, false>(staged, a, g, rec, G, st);
    }
    return cudaGetLastError();
}

}  // namespace

// precision: 0 = FP64, 1 = FP32 flux path
template <int FK>
cudaError_t launch_face(int precision, bool ns, int order, bool fold, const FaceLaunch &a,
                        cudaStream_t st);

// FP64 with teal's exact arithmetic (face_*_exact.cu); with a viscous flux, `a.G` holds 2 x 5 F
// values (convective and viscous records)
template <int FK>
cudaError_t launch_face_exact(bool ns, int order, bool fold, const FaceLaunch &a, cudaStream_t st);

#define TG_INSTANTIATE_FACE(FK)                                                                 \
    template <>                                                                                 \
    cudaError_t launch_face<FK>(int precision, bool ns, int order, bool fold, const FaceLaunch &a, \
                                cudaStream_t st)                                                \
    {                                                                                           \
        if (precision == 0) {                                                                   \
            return launch_face_r<FK, double>(ns, order, fold, a, st);                           \
        }                                                                                       \
        return launch_face_r<FK, float>(ns, order, fold, a, st);                                \
    }

#define TG_INSTANTIATE_FACE_EXACT(FK)                                                              \
    static_assert(kExact, "face_*_exact.cu is compiled with TG_EXACT_TU=1");                       \
    template <>                                                                                 \
    cudaError_t launch_face_exact<FK>(bool ns, int order, bool fold, const FaceLaunch &a, cudaStream_t st) \
    {                                                                                           \
        return launch_face_r<FK, double>(ns, order, fold, a, st);                               \
    }

}  // namespace tg
