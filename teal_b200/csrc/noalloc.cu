// Residual norm of a device-resident derivative that allocates no device memory.
//
// tg_residual goes through a context (tg_ctx), whose creation allocates the state, the geometry and
// the partial-sum scratch with cudaMalloc. Some callers cannot allocate while they solve: a serving
// process that committed its whole HBM budget to state arenas up front, or a host loop that must not
// stall the device (cudaMalloc and cudaFree can synchronise it). tg_residual_noalloc serves them: the
// derivative, the volumes and the result are the caller's device buffers, and the partial sums go to
// a fixed array compiled into this library (one copy per device).
//
// The reduction is the same as the context path's (per piece of PIECE cells, one block sums
// volume * r^2 per variable; one block of INST_BLOCK threads sums the pieces and takes
// sqrt(sum / sum_volume)), with the same loop order, so both give the same bits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/teal_b200.h"
#include "common.cuh"

using namespace tg;

int tg_record_error(int code, const char *msg);  // sets tg_last_error (context.cu)

namespace {

constexpr int NA_BLOCK = BLOCK;         // threads per piece, as k_piece_reduce
constexpr int NA_FINISH_BLOCK = 128;    // threads of the finishing block, as k_inst_end
constexpr long NA_MAX_PIECES = (long)TG_NOALLOC_MAX_CELLS / PIECE;
constexpr int NA_MAX_DEVICES = 64;

static_assert((long)TG_NOALLOC_MAX_CELLS % PIECE == 0, "the cell limit is a whole number of pieces");

}  // namespace

// partial sums, [piece][5]: 16384 pieces x 5 doubles = 640 KiB per device. Every slot the finishing
// kernel reads is written by the partial kernel of the same call, so nothing has to start at zero.
static __device__ __align__(256) double g_noalloc_partials[5 * NA_MAX_PIECES];

// one block per piece of PIECE cells: partials[p][k] = sum over the piece of volume * r_k^2
__global__ void __launch_bounds__(NA_BLOCK) k_noalloc_residual_pieces(int C, const double *__restrict__ deriv,
                                                                      const double *__restrict__ volume,
                                                                      double *__restrict__ partials)
{
    __shared__ double sh[NA_BLOCK / 32];
    const int beg = blockIdx.x * PIECE;
    const int end = min(C, beg + PIECE);
    double t[5] = {0, 0, 0, 0, 0};
    for (int c = beg + threadIdx.x; c < end; c += NA_BLOCK) {
        double v = volume[c];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            double r = deriv[(size_t)c * 5 + k];
            t[k] += v * (r * r);
        }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        double sum = block_sum<NA_BLOCK>(t[k], sh);
        if (threadIdx.x == 0) {
            partials[5 * blockIdx.x + k] = sum;
        }
    }
}

// one block: residual[k] = sqrt(sum over pieces / sum_volume)
__global__ void __launch_bounds__(NA_FINISH_BLOCK) k_noalloc_residual_finish(int npieces,
                                                                             const double *__restrict__ partials,
                                                                             double sum_volume,
                                                                             double *__restrict__ residual)
{
    __shared__ double sh[NA_FINISH_BLOCK / 32];
    double res[5];
    for (int k = 0; k < 5; k++) {
        double t = 0;
        for (int p = threadIdx.x; p < npieces; p += NA_FINISH_BLOCK) {
            t += partials[5 * p + k];
        }
        res[k] = block_sum<NA_FINISH_BLOCK>(t, sh);
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 5; k++) {
            residual[k] = sqrt(res[k] / sum_volume);
        }
    }
}

// Address of this device's scratch array, looked up once per device (with that device current)
// and kept for the life of the process. A cudaDeviceReset after that first lookup unloads the module
// holding the array, and the kept address would then be stale: resetting a device on which
// tg_residual_noalloc has run is not supported. Returns null after recording the error.
static double *noalloc_scratch(int *status)
{
    static std::mutex lock;
    static double *addr[NA_MAX_DEVICES] = {};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *status = tg_record_error(TG_ERR_NO_DEVICE, cudaGetErrorString(e));
        return nullptr;
    }
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        *status = tg_record_error(TG_ERR_INVALID, "tg_residual_noalloc: device ordinal out of range");
        return nullptr;
    }
    std::lock_guard<std::mutex> g(lock);
    if (!addr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            *status = tg_record_error(TG_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e)
                                                                     : "tg_residual_noalloc: null scratch address");
            return nullptr;
        }
        addr[dev] = p;
    }
    return addr[dev];
}

// a buffer the kernels may read or write: managed memory, or device memory of device `dev` (the
// current one: memory of another GPU would be a peer access the kernels are not set up for), 8-byte
// aligned
static bool device_buffer(const void *p, int dev)
{
    if (!p || ((uintptr_t)p & 7u)) {
        return false;
    }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) {
        return true;
    }
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

extern "C" int tg_residual_noalloc(const double *derivative, const double *volume, int num_cells, double sum_volume,
                                   double *residual, void *stream)
{
    if (num_cells < 0 || num_cells > TG_NOALLOC_MAX_CELLS) {
        return tg_record_error(TG_ERR_INVALID,
                               "tg_residual_noalloc: num_cells must be in [0, TG_NOALLOC_MAX_CELLS = 67108864]; "
                               "use tg_residual through a context for larger meshes");
    }
    if (!(sum_volume > 0.0) || !std::isfinite(sum_volume)) {
        return tg_record_error(TG_ERR_INVALID, "tg_residual_noalloc: sum_volume must be finite and positive");
    }
    int dev = -1;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess) {
        return tg_record_error(TG_ERR_NO_DEVICE, cudaGetErrorString(de));
    }
    if (!device_buffer(residual, dev) ||
        (num_cells > 0 && (!device_buffer(derivative, dev) || !device_buffer(volume, dev)))) {
        return tg_record_error(TG_ERR_INVALID,
                               "tg_residual_noalloc: derivative, volume and residual must be 8-byte aligned "
                               "memory of the current device (or managed memory)");
    }
    int status = TG_OK;
    double *partials = noalloc_scratch(&status);
    if (!partials) {
        return status;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int npieces = (num_cells + PIECE - 1) / PIECE;
    if (npieces > 0) {
        k_noalloc_residual_pieces<<<npieces, NA_BLOCK, 0, s>>>(num_cells, derivative, volume, partials);
    }
    k_noalloc_residual_finish<<<1, NA_FINISH_BLOCK, 0, s>>>(npieces, partials, sum_volume, residual);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return tg_record_error(TG_ERR_CUDA, cudaGetErrorString(e));
    }
    return TG_OK;
}
