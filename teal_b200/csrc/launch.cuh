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
};

template <int FK, typename R>
inline cudaError_t launch_face_r(bool ns, int order, bool fold, const FaceLaunch &a, cudaStream_t st)
{
    const Geometry<R> &g = *static_cast<const Geometry<R> *>(a.geom);
    const R *rec = static_cast<const R *>(a.rec);
    R *G = static_cast<R *>(a.G);
    dim3 grid((a.s.F + FACE_BLOCK - 1) / FACE_BLOCK);
    R gm = R(a.gamma), mu = R(a.mu), pr = R(a.prandtl);
    if (order == 1) {
        k_face<R, FK, false, 1, true><<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G);
    }
    else if (!ns) {
        k_face<R, FK, false, 2, true><<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G);
    }
    else if (fold) {
        k_face<R, FK, true, 2, true><<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G);
    }
    else {
        k_face<R, FK, true, 2, false><<<grid, FACE_BLOCK, 0, st>>>(a.s, g, a.q, rec, gm, mu, pr, G);
    }
    return cudaGetLastError();
}

// precision: 0 = FP64, 1 = FP32 flux path
template <int FK>
cudaError_t launch_face(int precision, bool ns, int order, bool fold, const FaceLaunch &a,
                        cudaStream_t st);

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

}  // namespace tg
