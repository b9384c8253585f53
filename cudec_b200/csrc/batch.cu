// C-ABI batch entries for the byte-oriented LZ formats (LZ4, raw Snappy):
// the CTA-per-chunk decoder (lz_cta_kernel.cuh), persistent over the batch.
//
// Contract (include/cudec.h): synchronous validation with no CUDA call on a
// reject, then the pending CUDA error is consumed, the kernel is submitted on
// the caller's stream, and the submission status is returned. Replaces
// iderex/cudec src/batch.cu:6-31 with validate_batch_args at
// src/lz4_decode.cuh:187-201 and the limit at src/batch_limits.h:28.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "cudec.h"
#include "launch.h"
#include "lz_cta_kernel.cuh"

namespace cdb {

cudec_status validate_batch(const void* const* src, const size_t* src_sizes,
                            void* const* dst, const size_t* caps, size_t n,
                            const cudec_chunk_result* results) {
    if (src == nullptr || src_sizes == nullptr || dst == nullptr ||
        caps == nullptr || results == nullptr ||
        reinterpret_cast<uintptr_t>(results) % 16 != 0 || n == 0 ||
        n > kMaxBatchChunks) {
        return CUDEC_ERR_INVALID_ARGUMENT;
    }
    return CUDEC_OK;
}

namespace {

constexpr int kMaxDevices = 64;
std::atomic<int> g_sm_count[kMaxDevices];

}  // namespace

int device_sm_count(int dev) {
    if (dev < 0 || dev >= kMaxDevices) return 0;
    int v = g_sm_count[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
        return 0;
    g_sm_count[dev].store(v, std::memory_order_relaxed);
    return v;
}

// The CTA-per-chunk kernel's resident CTAs per SM, once per device and
// format (its shared state exceeds 48 KB: opted into here).
template <class F>
cudaError_t prepare_cta(std::atomic<int>* ready, int dev, int* per_sm) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int v = ready[dev].load(std::memory_order_acquire);
    if (v > 0) {
        *per_sm = v;
        return cudaSuccess;
    }
    constexpr int kSmem = static_cast<int>(sizeof(lzc::Shm<F>));
    cudaError_t e = cudaFuncSetAttribute(lzc::lz_cta_kernel<F>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, lzc::lz_cta_kernel<F>, lzc::kThreads,
                                                      kSmem);
    if (e != cudaSuccess) return e;
    if (v <= 0) return cudaErrorInvalidConfiguration;
    ready[dev].store(v, std::memory_order_release);
    *per_sm = v;
    return cudaSuccess;
}

std::atomic<int> g_lz4_cta_ready[kMaxDevices];
std::atomic<int> g_snappy_cta_ready[kMaxDevices];

// One CTA per chunk at a time, persistent over the batch.
template <class F>
static cudec_status launch_lz_cta(std::atomic<int>* ready, const void* const* src,
                                  const size_t* src_sizes, void* const* dst, const size_t* caps,
                                  size_t n, cudec_chunk_result* results, cudaStream_t stream) {
    const cudec_status v = validate_batch(src, src_sizes, dst, caps, n, results);
    if (v != CUDEC_OK) return v;
    (void)cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CUDEC_ERR_CUDA;
    int per_sm = 0;
    if (prepare_cta<F>(ready, dev, &per_sm) != cudaSuccess) return CUDEC_ERR_CUDA;
    const int sms = device_sm_count(dev);
    if (sms <= 0) return CUDEC_ERR_CUDA;
    const size_t max_blocks = static_cast<size_t>(sms) * per_sm;
    const unsigned grid = static_cast<unsigned>(n < max_blocks ? n : max_blocks);
    lzc::lz_cta_kernel<F><<<grid, lzc::kThreads, sizeof(lzc::Shm<F>), stream>>>(
        src, src_sizes, dst, caps, n, results);
    return cudaGetLastError() == cudaSuccess ? CUDEC_OK : CUDEC_ERR_CUDA;
}

}  // namespace cdb

extern "C" {

cudec_status cudec_lz4_decompress_batch(const void* const* d_src_ptrs,
                                        const size_t* d_src_sizes,
                                        void* const* d_dst_ptrs,
                                        const size_t* d_dst_capacities,
                                        size_t chunk_count,
                                        cudec_chunk_result* d_results,
                                        cudec_stream_t stream) {
    return cdb::launch_lz_cta<cdb::lzc::Lz4F>(
        cdb::g_lz4_cta_ready, d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities,
        chunk_count, d_results, reinterpret_cast<cudaStream_t>(stream));
}

cudec_status cudec_snappy_decompress_batch(const void* const* d_src_ptrs,
                                           const size_t* d_src_sizes,
                                           void* const* d_dst_ptrs,
                                           const size_t* d_dst_capacities,
                                           size_t chunk_count,
                                           cudec_chunk_result* d_results,
                                           cudec_stream_t stream) {
    return cdb::launch_lz_cta<cdb::lzc::SnappyF>(
        cdb::g_snappy_cta_ready, d_src_ptrs, d_src_sizes, d_dst_ptrs,
        d_dst_capacities, chunk_count, d_results,
        reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"

#ifdef CDB_PHASE_TIMING
// Profiling builds only: the CTA decoder's phase cycles [0, 16) and event
// counts [16, 32) since the last call (then reset).
extern "C" int cudec_lzc_phase_counters(unsigned long long* out) {
    if (cudaMemcpyFromSymbol(out, cdb::lzc::lzc_cycles, 16 * sizeof(unsigned long long)) !=
            cudaSuccess ||
        cudaMemcpyFromSymbol(out + 16, cdb::lzc::lzc_events, 16 * sizeof(unsigned long long)) !=
            cudaSuccess)
        return 1;
    static const unsigned long long zero[16] = {};
    if (cudaMemcpyToSymbol(cdb::lzc::lzc_cycles, zero, sizeof(zero)) != cudaSuccess ||
        cudaMemcpyToSymbol(cdb::lzc::lzc_events, zero, sizeof(zero)) != cudaSuccess)
        return 1;
    return 0;
}
#endif
