// Bulk asynchronous copies (TMA, cp.async.bulk) from global into shared memory, completed on an
// mbarrier, for staging streamed SoA rows of a tile. One CTA, no clusters, no multicast.
#pragma once

#include <cstdint>

namespace tg {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async proxy that completes the copies
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// the calling thread's arrival, announcing `bytes` of copies that complete on the barrier
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy: both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// One try at the barrier's phase: the thread is suspended in hardware until the phase completes or
// about `hint_ns` nanoseconds pass (mbarrier.try_wait with a suspend-time hint), so a waiting warp
// issues one instruction per try instead of spinning on test_wait.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase, uint32_t hint_ns)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase), "r"(hint_ns)
        : "memory");
    return done != 0;
}

// tries of a bounded wait (each suspends up to about a microsecond): about a second
constexpr int MBAR_POLLS = 1 << 20;

// Wait for the barrier's phase with an iteration limit; false when it gave up (at once for 0).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, int polls)
{
    for (int it = 0; it < polls; it++) {
        if (mbar_try_wait(bar, phase, 1000u)) {
            return true;
        }
    }
    return false;
}

// Bulk copy of n elements starting at src into dst, where dst is 16-byte aligned and src need
// not be: the copy starts at src rounded down to 16 bytes and is rounded up to a multiple of 16
// bytes, so it reads up to 15 bytes before and after the elements (allocations carry slack for
// that). Returns the bytes copied; with issue == false only computes them and sets *shift, the
// elements before src in the copy.
template <typename T>
__device__ __forceinline__ uint32_t stage_span(T *dst, const T *src, int n, uint64_t *bar, bool issue,
                                               uint8_t *shift)
{
    uint32_t mis = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(src) & 15u);
    uint32_t bytes = (mis + static_cast<uint32_t>(n) * static_cast<uint32_t>(sizeof(T)) + 15u) & ~15u;
    if (issue) {
        bulk_g2s(dst, reinterpret_cast<const char *>(src) - mis, bytes, bar);
    }
    else {
        *shift = static_cast<uint8_t>(mis / sizeof(T));
    }
    return bytes;
}

}  // namespace tg
