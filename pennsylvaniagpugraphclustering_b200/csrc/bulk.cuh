// bulk.cuh -- staging a contiguous range of one or two 4-byte arrays from this
// GPU's global memory into a block's shared memory with TMA bulk copies
// (cp.async.bulk, non-multicast, completion on an mbarrier), used by the
// kernels that split one very long row across many blocks.
#pragma once
#include "common.cuh"

namespace pggc {

// bounded waits on a bulk copy's mbarrier (far above any copy's duration)
constexpr u32 BULK_WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// non-multicast bulk copy global -> this CTA's shared memory; both addresses
// 16-byte aligned and bytes a multiple of 16 (the caller's job)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, u32 bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Block-cooperative: copies a[j0, j1) (and b[j0, j1) when b is not null) into
// sa / sb, element j at index j - (j0 & ~3).  sa and sb are 16-byte aligned
// shared buffers of at least (j1 - j0) + 4 elements; `bar` is a shared 8-byte
// mbarrier word used once per call.  The 16-byte-aligned middle goes by bulk
// copy, the ragged tail by plain loads (the head below j0 is copied and not
// used); a global base that is not 16-byte aligned makes it all plain loads.
// Returns false (every thread) after latching DEV_ERR_WAIT in *err when the
// copy did not complete within the bounded wait.
template <class A, class B>
__device__ bool stage_rows(const A* a, const B* b, i64 j0, i64 j1, A* sa, B* sb, unsigned long long* bar,
                           int* err) {
    static_assert(sizeof(A) == 4 && sizeof(B) == 4, "4-byte elements");
    __shared__ int staged;
    const i64 lo16 = j0 & ~(i64)3, hi16 = j1 & ~(i64)3;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a) & 15) == 0) &&
                         (!b || (reinterpret_cast<uintptr_t>(b) & 15) == 0);
    const u32 bytes = (aligned && hi16 > lo16) ? (u32)((hi16 - lo16) * 4) : 0u;
    if (threadIdx.x == 0 && bytes) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && bytes) {
        mbar_expect_tx(bar, b ? 2 * bytes : bytes);
        bulk_g2s(sa, a + lo16, bytes, bar);
        if (b) bulk_g2s(sb, b + lo16, bytes, bar);
    }
    const i64 plain_from = bytes ? (hi16 > j0 ? hi16 : j0) : j0;
    for (i64 j = plain_from + threadIdx.x; j < j1; j += blockDim.x) {
        sa[j - lo16] = a[j];
        if (b) sb[j - lo16] = b[j];
    }
    // one thread waits (bounded) for the bulk copy and tells the block
    if (threadIdx.x == 0) {
        bool done = bytes == 0;
        for (u32 it = 0; it < BULK_WAIT_LIMIT && !done; it++) done = mbar_try_wait(bar, 0);
        if (!done) {
            // never expected: report, wait (bounded) for the copy that still
            // targets this block's shared memory, and give up the range
            atomicExch(err, (int)DEV_ERR_WAIT);
            for (u32 it = 0; it < BULK_WAIT_LIMIT && !done; it++) done = mbar_try_wait(bar, 0);
            done = false;
        }
        staged = done ? 1 : 0;
    }
    __syncthreads();
    return staged != 0;
}

}  // namespace pggc
