// Device helpers shared by all kernels: state / geometry loads, teal's is_close, and fixed-shape
// (deterministic) block reductions.
#pragma once

#include <cfloat>
#include <type_traits>

#include "device.cuh"
#include "tuned.h"

namespace tg {

// bits of the device error word (Steps::error)
enum DeviceError { ERR_NONFINITE = 1, ERR_TIMEOUT = 2, ERR_LOOP_LIMIT = 4 };

constexpr int BLOCK = 256;
constexpr int FACE_BLOCK = TG_FACE_BLOCK;
constexpr int FACE_MINB = TG_FACE_MINB;
constexpr int FACE_MINB_EULER = TG_FACE_MINB_EULER;
constexpr int FACE_MINB_FP32 = TG_FACE_MINB_FP32;
// resident face blocks per SM: FP64 Navier-Stokes (more registers: the viscous flux), FP64 Euler,
// or the FP32-flux form
template <typename R>
__host__ __device__ constexpr int face_minb(bool ns)
{
    return sizeof(R) == sizeof(float) ? FACE_MINB_FP32 : ns ? FACE_MINB : FACE_MINB_EULER;
}
constexpr int CELL_BLOCK = TG_CELL_BLOCK;
constexpr int CELL_MINB = TG_CELL_MINB;
constexpr int GRAD_MINB = TG_GRAD_MINB;
constexpr int REDUCE_BLOCK = 1024;

// ---- small helpers ---------------------------------------------------------------------------

template <typename R>
__device__ __forceinline__ Prim<R> load_prim(const double *__restrict__ q, int ld, int i)
{
    Prim<R> p;
    p.rho = R(__ldg(q + i));
    p.u.x = R(__ldg(q + ld + i));
    p.u.y = R(__ldg(q + 2 * ld + i));
    p.u.z = R(__ldg(q + 3 * ld + i));
    p.p = R(__ldg(q + 4 * ld + i));
    return p;
}

__device__ __forceinline__ void store_prim(double *__restrict__ q, int ld, int i, const Prim<double> &p)
{
    q[i] = p.rho;
    q[ld + i] = p.u.x;
    q[2 * ld + i] = p.u.y;
    q[3 * ld + i] = p.u.z;
    q[4 * ld + i] = p.p;
}

// The state of cell i with the pressure taken relative to pref (in FP64, then converted)
template <typename R>
__device__ __forceinline__ Prim<R> load_prim_rel(const double *__restrict__ q, int ld, int i, double pref)
{
    Prim<R> p;
    p.rho = R(__ldg(q + i));
    p.u = v3(R(__ldg(q + ld + i)), R(__ldg(q + 2 * ld + i)), R(__ldg(q + 3 * ld + i)));
    p.p = R(__ldg(q + 4 * ld + i) - pref);
    return p;
}

// no reference pressure (FP64 kernels)
struct NoPressureRef {
};

// Reference pressure of the FP32-flux form, per instance (null: none)
struct PressureRef {
    const double *pref;     // [ninst]
    const int *cell_inst;   // [C]
    __device__ __forceinline__ double of(int c) const { return pref ? __ldg(pref + __ldg(cell_inst + c)) : 0.0; }
};

// the reference-pressure argument of a face kernel in precision R
template <typename R>
using PressureRefOf = typename std::conditional<sizeof(R) == sizeof(float), PressureRef, NoPressureRef>::type;

template <typename R>
__device__ __forceinline__ Basis<R> load_basis(const R *__restrict__ b, int ld, int f)
{
    Basis<R> m;
    m.x = v3(__ldg(b + f), __ldg(b + ld + f), __ldg(b + 2 * ld + f));
    m.y = v3(__ldg(b + 3 * ld + f), __ldg(b + 4 * ld + f), __ldg(b + 5 * ld + f));
    m.z = v3(__ldg(b + 6 * ld + f), __ldg(b + 7 * ld + f), __ldg(b + 8 * ld + f));
    return m;
}

template <typename R>
__device__ __forceinline__ V3<R> load_v3(const R *__restrict__ a, int ld, int i)
{
    return v3(__ldg(a + i), __ldg(a + ld + i), __ldg(a + 2 * ld + i));
}

template <typename R>
__device__ __forceinline__ R prim_get(const Prim<R> &p, int v)
{
    return v == 0 ? p.rho : v == 1 ? p.u.x : v == 2 ? p.u.y : v == 3 ? p.u.z : p.p;
}

template <typename R>
__device__ __forceinline__ Prim<R> prim_from(const R *a)
{
    return Prim<R>{a[0], v3(a[1], a[2], a[3]), a[4]};
}

// Re-read of a value another part of the kernel already loaded: a volatile read-only load, so the
// compiler neither merges it with the first load nor keeps the first value live in a register
// across the code in between (the line is still in L1)
__device__ __forceinline__ double reload(const double *p)
{
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float reload(const float *p)
{
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

template <typename R>
__device__ __forceinline__ Basis<R> reload_basis(const R *__restrict__ b, int ld, int f)
{
    Basis<R> m;
    m.x = v3(reload(b + f), reload(b + ld + f), reload(b + 2 * ld + f));
    m.y = v3(reload(b + 3 * ld + f), reload(b + 4 * ld + f), reload(b + 5 * ld + f));
    m.z = v3(reload(b + 6 * ld + f), reload(b + 7 * ld + f), reload(b + 8 * ld + f));
    return m;
}

template <typename R>
__device__ __forceinline__ Prim<R> reload_prim(const double *__restrict__ q, int ld, int i)
{
    Prim<R> p;
    p.rho = R(reload(q + i));
    p.u.x = R(reload(q + ld + i));
    p.u.y = R(reload(q + 2 * ld + i));
    p.u.z = R(reload(q + 3 * ld + i));
    p.p = R(reload(q + 4 * ld + i));
    return p;
}

// Per-cell gradient record: (gx, gy, gz, psi) for each of the 5 variables, 20 values per cell;
// each variable's 4 values are one aligned 32-byte access in FP64, a single 256-bit load or store,
// so that a record gather costs one instruction per variable (TGV 128^3 face kernel 0.493 -> 0.479
// ms, gradient kernel 0.264 -> 0.246 ms against two 16-byte accesses). (A
// compact 16-value layout for folded records, one cache line per cell, was measured slower: the
// per-variable writers leave partially written sectors.)
template <typename R>
struct Vec2;
template <>
struct Vec2<double> {
    using T = double2;
};
template <>
struct Vec2<float> {
    using T = float2;
};

__device__ __forceinline__ void grad_rec_store(double *rec, int c, int v, double gx, double gy, double gz,
                                               double psi)
{
    double *p = rec + ((size_t)c * 5 + v) * 4;
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(gx), "d"(gy), "d"(gz), "d"(psi)
                 : "memory");
}
__device__ __forceinline__ void grad_rec_store(float *rec, int c, int v, float gx, float gy, float gz, float psi)
{
    float2 *p = reinterpret_cast<float2 *>(rec + ((size_t)c * 5 + v) * 4);
    p[0] = make_float2(gx, gy);
    p[1] = make_float2(gz, psi);
}

// read-only loads: the records are written by an earlier launch
__device__ __forceinline__ void grad_rec_load(const double *rec, int c, int v, double &gx, double &gy, double &gz,
                                              double &psi)
{
    const double *p = rec + ((size_t)c * 5 + v) * 4;
    asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(gx), "=d"(gy), "=d"(gz), "=d"(psi) : "l"(p));
}
__device__ __forceinline__ void grad_rec_load(const float *rec, int c, int v, float &gx, float &gy, float &gz,
                                              float &psi)
{
    // two 8-byte loads: one 16-byte load was measured slower in the FP32 face kernel (0.371 vs
    // 0.326 ms, TGV 128^3)
    const float2 *p = reinterpret_cast<const float2 *>(rec + ((size_t)c * 5 + v) * 4);
    const float2 a = __ldg(p), b = __ldg(p + 1);
    gx = a.x, gy = a.y, gz = b.x, psi = b.y;
}

// Per-face flux records, 5 values per face without padding: components 0-3 as [F][4] (one 256-bit
// access in FP64, two 2-vector accesses in FP32), component 4 as [F] after them.
constexpr int FLUX_REC = 5;

// Element offset of a second set of flux records (the exact form's viscous records) behind the
// first: 5 F rounded up to a multiple of 4, so that its [F][4] part starts on a 32-byte boundary as
// the 256-bit record accesses require.
__host__ __device__ constexpr size_t flux_rec2_offset(int F)
{
    return ((size_t)FLUX_REC * (size_t)F + 3) & ~(size_t)3;
}

__device__ __forceinline__ void flux_rec_store(double *G, int F, int f, const double (&v)[5])
{
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(G + (size_t)f * 4), "d"(v[0]), "d"(v[1]),
                 "d"(v[2]), "d"(v[3])
                 : "memory");
    G[(size_t)4 * F + f] = v[4];
}

__device__ __forceinline__ void flux_rec_load(const double *G, int F, int f, double (&v)[5])
{
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
        : "l"(G + (size_t)f * 4));
    v[4] = __ldg(G + (size_t)4 * F + f);
}

template <typename R>
__device__ __forceinline__ void flux_rec_store(R *G, int F, int f, const R (&v)[5])
{
    using T2 = typename Vec2<R>::T;
    T2 *p = reinterpret_cast<T2 *>(G + (size_t)f * 4);
    p[0] = T2{v[0], v[1]};
    p[1] = T2{v[2], v[3]};
    G[(size_t)4 * F + f] = v[4];
}

template <typename R>
__device__ __forceinline__ void flux_rec_load(const R *G, int F, int f, double (&v)[5])
{
    using T2 = typename Vec2<R>::T;
    const T2 *p = reinterpret_cast<const T2 *>(G + (size_t)f * 4);
    T2 a = __ldg(p), b = __ldg(p + 1);
    v[0] = double(a.x), v[1] = double(a.y), v[2] = double(b.x), v[3] = double(b.y);
    v[4] = double(__ldg(G + (size_t)4 * F + f));
}

// is_close(x, 0) of src/core/utils.c:29-34 (absolute 1e-8, relative 1e-5)
template <typename R>
__device__ __forceinline__ bool is_close_zero(R x)
{
    // |x| <= max(1e-8, 1e-5 |x|) holds exactly when |x| <= 1e-8 or x is infinite
    const R a = fabs(x);
    return (a <= R(1e-8)) || (a == R(INFINITY));
}


// ---- block reductions (fixed shape => deterministic) -----------------------------------------

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, o);
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        sh[warp] = v;
    }
    __syncthreads();
    double r = 0;
    if (warp == 0) {
        r = (lane < NT / 32) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
        }
    }
    return r;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ double block_min(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        sh[warp] = v;
    }
    __syncthreads();
    double r = DBL_MAX;
    if (warp == 0) {
        r = (lane < NT / 32) ? sh[lane] : DBL_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r = fmin(r, __shfl_down_sync(0xffffffffu, r, o));
        }
    }
    return r;
}

}  // namespace tg
