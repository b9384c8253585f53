// Device-side building blocks shared by the decode kernels (sm_100a).
//
//  * mbarrier + cp.async.bulk (the bulk-copy engine behind TMA) for staging a
//    chunk's compressed bytes into shared memory without register traffic;
//    every wait on an mbarrier is bounded and reports a timeout instead of
//    spinning forever.
//  * block-wide exclusive scans over 32- and 64-bit values.
#pragma once

#include <cstdint>

namespace cdb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
            smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait on one mbarrier phase. Returns false if the phase did not
// complete within the iteration budget (each try_wait itself suspends for a
// hardware-bounded interval), so a lost transfer becomes an error status, not
// a hung SM.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar,
                                                  uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    return false;
}

// Orders this thread's earlier generic-proxy shared-memory accesses before a
// following async-proxy (bulk copy) access to the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// cp.async.bulk global -> shared, completion signalled on `bar` as tx bytes.
// Both addresses 16-byte aligned and `bytes` a multiple of 16 (checked by the
// caller's arithmetic, see stage_window).
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gsrc,
                                         uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1], %2, [%3];" ::"r"(smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Block-wide exclusive scan. `warp_tmp` holds one slot per warp (plus one for
// the total). Contains two __syncthreads(); every thread must call it.
template <typename T, int kThreads>
__device__ __forceinline__ T block_exclusive_scan(T v, T* warp_tmp, T* total) {
    constexpr int kWarps = kThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) warp_tmp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kWarps ? warp_tmp[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T o = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += o;
        }
        if (lane < kWarps) warp_tmp[lane] = wi - w;
        if (lane == kWarps - 1) warp_tmp[kWarps] = wi;
    }
    __syncthreads();
    *total = warp_tmp[kWarps];
    return warp_tmp[warp] + incl - v;
}

}  // namespace cdb
