// Zstd batch entry: one Zstd frame per chunk, device memory in and out.
// The table builders and bit readers are in zstd_kernel.cuh, the frame loop
// and sequence execution in zstd_frame.cuh; this file holds the batch kernel
// and the C ABI.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "cudec.h"
#include "launch.h"
#include "zstd_frame.cuh"

namespace cdb {
namespace zstd {

constexpr uint32_t kMaxSlots = 4096;  // frames decoded concurrently (workspace slots)

// Multi: a chunk is a sequence of frames (decode_frames) rather than one
// frame (decode_frame); a template parameter, so the one-frame kernel is
// compiled alone.
template <bool Multi>
__global__ void __launch_bounds__(kCtaThreads)
    zstd_decode_kernel(const void* const* src_ptrs, const size_t* src_sizes,
                       void* const* dst_ptrs, const size_t* dst_caps, size_t n,
                       cudec_chunk_result* results, uint8_t* workspace) {
    __shared__ WarpSmem wsm[kWarpsPerCta];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t gw = static_cast<size_t>(blockIdx.x) * kWarpsPerCta + warp;
    const size_t total = static_cast<size_t>(gridDim.x) * kWarpsPerCta;
    uint8_t* litbuf = workspace + gw * kLitSlot;
    for (size_t c = gw; c < n; c += total) {
        uint64_t written = 0;
        const uint8_t* src = static_cast<const uint8_t*>(src_ptrs[c]);
        uint8_t* dst = static_cast<uint8_t*>(dst_ptrs[c]);
        int st;
        if constexpr (Multi)
            st = decode_frames(src, src_sizes[c], dst, dst_caps[c], wsm[warp], litbuf, lane,
                               &written);
        else
            st = decode_frame(src, src_sizes[c], dst, dst_caps[c], wsm[warp], litbuf, lane,
                              &written);
        __syncwarp();
        if (lane == 0) {
            results[c].status = st;
            results[c].reserved = 0;
            results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
    }
}

}  // namespace zstd
}  // namespace cdb

extern "C" {

size_t cudec_zstd_workspace_bytes(size_t chunk_count) {
    const size_t slots = chunk_count < cdb::zstd::kMaxSlots ? chunk_count : cdb::zstd::kMaxSlots;
    const size_t rounded = (slots + cdb::zstd::kWarpsPerCta - 1) / cdb::zstd::kWarpsPerCta *
                           cdb::zstd::kWarpsPerCta;
    return rounded * cdb::zstd::kLitSlot;
}

}  // extern "C"

namespace {

cudec_status launch_zstd(const void* const* d_src_ptrs, const size_t* d_src_sizes,
                         void* const* d_dst_ptrs, const size_t* d_dst_capacities,
                         size_t chunk_count, cudec_chunk_result* d_results, void* d_workspace,
                         size_t workspace_bytes, cudec_stream_t stream, bool multi) {
    const cudec_status v = cdb::validate_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                               d_dst_capacities, chunk_count, d_results);
    if (v != CUDEC_OK) return v;
    if (d_workspace == nullptr || workspace_bytes < cudec_zstd_workspace_bytes(chunk_count))
        return CUDEC_ERR_INVALID_ARGUMENT;
    (void)cudaGetLastError();
    const size_t slots = cudec_zstd_workspace_bytes(chunk_count) / cdb::zstd::kLitSlot;
    const unsigned grid = static_cast<unsigned>(slots / cdb::zstd::kWarpsPerCta);
    const auto kernel = multi ? cdb::zstd::zstd_decode_kernel<true>
                              : cdb::zstd::zstd_decode_kernel<false>;
    kernel<<<grid, cdb::zstd::kCtaThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, chunk_count, d_results,
        static_cast<uint8_t*>(d_workspace));
    return cudaGetLastError() == cudaSuccess ? CUDEC_OK : CUDEC_ERR_CUDA;
}

}  // namespace

extern "C" {

cudec_status cudec_zstd_decompress_batch(const void* const* d_src_ptrs,
                                         const size_t* d_src_sizes,
                                         void* const* d_dst_ptrs,
                                         const size_t* d_dst_capacities,
                                         size_t chunk_count,
                                         cudec_chunk_result* d_results,
                                         void* d_workspace, size_t workspace_bytes,
                                         cudec_stream_t stream) {
    return launch_zstd(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, chunk_count,
                       d_results, d_workspace, workspace_bytes, stream, false);
}

cudec_status cudec_zstd_decompress_batch_multi(const void* const* d_src_ptrs,
                                               const size_t* d_src_sizes,
                                               void* const* d_dst_ptrs,
                                               const size_t* d_dst_capacities,
                                               size_t chunk_count,
                                               cudec_chunk_result* d_results,
                                               void* d_workspace, size_t workspace_bytes,
                                               cudec_stream_t stream) {
    return launch_zstd(d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, chunk_count,
                       d_results, d_workspace, workspace_bytes, stream, true);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant: the same kernel, its literal slots taken from a
// file-scope device array instead of a caller workspace. One slot per frame,
// so a call takes at most kNoAllocChunks frames (8 MiB of slots). The array's
// address is looked up once per device. Nothing in it needs to start at zero:
// every literal byte a sequence reads was written by the same frame's
// Huffman decode first. Calls whose launches overlap in time on one device
// share the array and race; calls queued on one stream are ordered.
namespace cdb {
namespace zstd {

constexpr size_t kNoAllocChunks = CUDEC_ZSTD_NOALLOC_MAX_CHUNKS;
constexpr int kNoAllocMaxDevices = 256;
static_assert(kNoAllocChunks % kWarpsPerCta == 0, "whole CTAs of slots");

static __device__ __align__(256) uint8_t g_noalloc_slots[kNoAllocChunks * kLitSlot];

static std::atomic<uint8_t*> g_noalloc_addr[kNoAllocMaxDevices];

// Device address of the slot array on the current device (nullptr on error).
static uint8_t* noalloc_slots(cudaError_t* err) {
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    uint8_t* p = g_noalloc_addr[dev].load(std::memory_order_acquire);
    if (p != nullptr) return p;
    void* a = nullptr;
    *err = cudaGetSymbolAddress(&a, g_noalloc_slots);
    if (*err != cudaSuccess || a == nullptr) {
        if (*err == cudaSuccess) *err = cudaErrorInvalidSymbol;
        return nullptr;
    }
    g_noalloc_addr[dev].store(static_cast<uint8_t*>(a), std::memory_order_release);
    return static_cast<uint8_t*>(a);
}

}  // namespace zstd
}  // namespace cdb

extern "C" cudec_status cudec_zstd_decompress_batch_noalloc(
    const void* const* d_src_ptrs, const size_t* d_src_sizes, void* const* d_dst_ptrs,
    const size_t* d_dst_capacities, size_t chunk_count, cudec_chunk_result* d_results,
    cudec_stream_t stream) {
    const cudec_status v = cdb::validate_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                               d_dst_capacities, chunk_count, d_results);
    if (v != CUDEC_OK) return v;
    if (chunk_count > cdb::zstd::kNoAllocChunks) return CUDEC_ERR_INVALID_ARGUMENT;
    (void)cudaGetLastError();
    cudaError_t err = cudaSuccess;
    uint8_t* slots = cdb::zstd::noalloc_slots(&err);
    if (slots == nullptr) {
        (void)cudaGetLastError();
        return CUDEC_ERR_CUDA;
    }
    const unsigned grid = static_cast<unsigned>(
        (chunk_count + cdb::zstd::kWarpsPerCta - 1) / cdb::zstd::kWarpsPerCta);
    cdb::zstd::zstd_decode_kernel<false><<<grid, cdb::zstd::kCtaThreads, 0,
                                           reinterpret_cast<cudaStream_t>(stream)>>>(
        d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, chunk_count, d_results, slots);
    return cudaGetLastError() == cudaSuccess ? CUDEC_OK : CUDEC_ERR_CUDA;
}
