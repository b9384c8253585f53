// GDeflate entries: the page batch (one 64 KiB page per chunk, device memory
// in and out) and the TileStream container (host parse of the envelope, then
// every tile in one page-batch launch).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cudec.h"
#include "gdeflate_page.cuh"
#include "host_util.h"
#include "launch.h"

namespace cdb {
namespace gdf {

constexpr uint32_t kWarps = 4;
constexpr int kSmem = static_cast<int>(kWarps * sizeof(Tables));

__global__ void __launch_bounds__(32 * kWarps)
    gdeflate_kernel(const void* const* src_ptrs, const size_t* src_sizes, void* const* dst_ptrs,
                    const size_t* dst_caps, size_t n, cudec_chunk_result* results) {
    extern __shared__ __align__(16) uint8_t gdf_smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Tables& tb = reinterpret_cast<Tables*>(gdf_smem)[warp];
    const size_t total = static_cast<size_t>(gridDim.x) * kWarps;
    for (size_t c = static_cast<size_t>(blockIdx.x) * kWarps + warp; c < n; c += total) {
        uint64_t written = 0;
        const int st = decode_page(static_cast<const uint8_t*>(src_ptrs[c]), src_sizes[c],
                                   static_cast<uint8_t*>(dst_ptrs[c]), dst_caps[c], tb, lane,
                                   &written);
        __syncwarp();
        if (lane == 0) {
            results[c].status = st;
            results[c].reserved = 0;
            results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
    }
}

constexpr int kMaxDevices = 64;
std::atomic<int> g_ready[kMaxDevices];

cudaError_t prepare(int dev, int* per_sm) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int v = g_ready[dev].load(std::memory_order_acquire);
    if (v > 0) {
        *per_sm = v;
        return cudaSuccess;
    }
    cudaError_t e = cudaFuncSetAttribute(gdeflate_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, gdeflate_kernel, 32 * kWarps, kSmem);
    if (e != cudaSuccess) return e;
    if (v <= 0) return cudaErrorInvalidConfiguration;
    g_ready[dev].store(v, std::memory_order_release);
    *per_sm = v;
    return cudaSuccess;
}

// TileStream envelope (mirrors iderex/cudec src/tilestream.h:117-261).
uint32_t rd32(const uint8_t* p) {
    return static_cast<uint32_t>(p[0]) | (static_cast<uint32_t>(p[1]) << 8) |
           (static_cast<uint32_t>(p[2]) << 16) | (static_cast<uint32_t>(p[3]) << 24);
}

cudec_status parse(const uint8_t* st, uint64_t size, cudec_tile* tiles, uint64_t cap,
                   uint64_t* count, uint64_t* total) {
    if (st == nullptr || tiles == nullptr || count == nullptr || total == nullptr)
        return CUDEC_ERR_INVALID_ARGUMENT;
    if (size < 8) return CUDEC_ERR_CORRUPT_INPUT;
    if (st[0] != static_cast<uint8_t>(st[1] ^ 0xFFu)) return CUDEC_ERR_CORRUPT_INPUT;
    const uint64_t n = static_cast<uint64_t>(st[2]) | (static_cast<uint64_t>(st[3]) << 8);
    if (n == 0) return CUDEC_ERR_CORRUPT_INPUT;
    const uint32_t packed = rd32(st + 4);
    const uint64_t last = (packed >> 2) & 0x3FFFFu;
    if ((packed & 3u) != 1u || ((packed >> 20) & 0xFFFu) != 0 || last >= 65536)
        return CUDEC_ERR_CORRUPT_INPUT;
    if (cap < n) return CUDEC_ERR_INVALID_ARGUMENT;
    const uint64_t toc_end = 8 + 4 * n;
    if (size < toc_end) return CUDEC_ERR_CORRUPT_INPUT;
    const uint64_t last_src = rd32(st + 8);
    if (last_src == 0) return CUDEC_ERR_CORRUPT_INPUT;
    uint64_t prev = toc_end;
    for (uint64_t i = 1; i < n; ++i) {
        const uint64_t off = rd32(st + 8 + 4 * i);
        if (off <= prev) return CUDEC_ERR_CORRUPT_INPUT;
        tiles[i].src_offset = off;
        prev = off;
    }
    tiles[0].src_offset = toc_end;
    for (uint64_t i = 0; i + 1 < n; ++i)
        tiles[i].src_size = tiles[i + 1].src_offset - tiles[i].src_offset;
    tiles[n - 1].src_size = last_src;
    if (tiles[n - 1].src_offset + last_src > size) return CUDEC_ERR_CORRUPT_INPUT;
    for (uint64_t i = 0; i + 1 < n; ++i) tiles[i].dst_size = 65536;
    tiles[n - 1].dst_size = last == 0 ? 65536 : last;
    *count = n;
    *total = n * 65536 - (last == 0 ? 0 : 65536 - last);
    return CUDEC_OK;
}

}  // namespace gdf
}  // namespace cdb

extern "C" {

cudec_status cudec_gdeflate_decompress_batch(const void* const* d_src_ptrs,
                                             const size_t* d_src_sizes,
                                             void* const* d_dst_ptrs,
                                             const size_t* d_dst_capacities,
                                             size_t chunk_count,
                                             cudec_chunk_result* d_results,
                                             cudec_stream_t stream) {
    const cudec_status v = cdb::validate_batch(d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                               d_dst_capacities, chunk_count, d_results);
    if (v != CUDEC_OK) return v;
    (void)cudaGetLastError();
    int dev = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CUDEC_ERR_CUDA;
    if (cdb::gdf::prepare(dev, &per_sm) != cudaSuccess) return CUDEC_ERR_CUDA;
    const int sms = cdb::device_sm_count(dev);
    if (sms <= 0) return CUDEC_ERR_CUDA;
    const size_t max_blocks = static_cast<size_t>(sms) * per_sm;
    const size_t want = (chunk_count + cdb::gdf::kWarps - 1) / cdb::gdf::kWarps;
    const unsigned grid = static_cast<unsigned>(want < max_blocks ? want : max_blocks);
    cdb::gdf::gdeflate_kernel<<<grid, 32 * cdb::gdf::kWarps, cdb::gdf::kSmem,
                                reinterpret_cast<cudaStream_t>(stream)>>>(
        d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, chunk_count, d_results);
    return cudaGetLastError() == cudaSuccess ? CUDEC_OK : CUDEC_ERR_CUDA;
}

cudec_status cudec_gdeflate_tilestream_parse(const void* h_stream, size_t stream_size,
                                             cudec_tile* tiles, size_t tiles_capacity,
                                             size_t* out_tile_count, size_t* out_total) {
    uint64_t count = 0, total = 0;
    const cudec_status st = cdb::gdf::parse(static_cast<const uint8_t*>(h_stream), stream_size,
                                            tiles, tiles_capacity, &count, &total);
    if (st != CUDEC_OK) return st;
    if (out_tile_count) *out_tile_count = count;
    if (out_total) *out_total = total;
    return CUDEC_OK;
}

cudec_status cudec_gdeflate_tilestream_decompress(const void* h_stream, size_t stream_size,
                                                  void* dst, size_t dst_capacity,
                                                  cudec_mem_space dst_space,
                                                  size_t* out_written) {
    if (out_written == nullptr || dst == nullptr ||
        (dst_space != CUDEC_MEM_HOST && dst_space != CUDEC_MEM_DEVICE))
        return CUDEC_ERR_INVALID_ARGUMENT;
    *out_written = 0;
    if (h_stream == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    std::vector<cudec_tile> tiles(65535);
    uint64_t count = 0, total = 0;
    cudec_status st = cdb::gdf::parse(static_cast<const uint8_t*>(h_stream), stream_size,
                                      tiles.data(), tiles.size(), &count, &total);
    if (st != CUDEC_OK) return st;
    if (total > dst_capacity) return CUDEC_ERR_OUTPUT_TOO_SMALL;
    (void)cudaGetLastError();
    cdb::StreamOwner s;
    if (s.create() != cudaSuccess) return CUDEC_ERR_CUDA;
    // Device block: tables (5 x 8 bytes per tile), results, the stream body,
    // and (for host destinations) the output.
    const size_t n = count;
    const size_t tab = 48 * n;
    const size_t out_bytes = dst_space == CUDEC_MEM_HOST ? total : 0;
    cdb::AsyncBuf dev;
    if (dev.alloc(tab + stream_size + out_bytes + 64, s.s) != cudaSuccess) return CUDEC_ERR_CUDA;
    uint8_t* d = static_cast<uint8_t*>(dev.p);
    uint8_t* d_in = d + tab;
    uint8_t* d_out = dst_space == CUDEC_MEM_HOST ? d_in + stream_size : static_cast<uint8_t*>(dst);
    cdb::PinnedBuf hb;
    if (hb.ensure(tab) != cudaSuccess) return CUDEC_ERR_CUDA;
    auto* h = static_cast<uint64_t*>(hb.p);
    uint64_t at = 0;
    for (size_t i = 0; i < n; ++i) {
        h[i] = reinterpret_cast<uint64_t>(d_in + tiles[i].src_offset);
        h[n + i] = tiles[i].src_size;
        h[2 * n + i] = reinterpret_cast<uint64_t>(d_out + at);
        h[3 * n + i] = tiles[i].dst_size;
        at += tiles[i].dst_size;
    }
    auto* d_res = reinterpret_cast<cudec_chunk_result*>(d + 32 * n);
    bool ok = cudaMemcpyAsync(d, h, 32 * n, cudaMemcpyHostToDevice, s.s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_in, h_stream, stream_size, cudaMemcpyHostToDevice, s.s) ==
                   cudaSuccess;
    if (!ok) return CUDEC_ERR_CUDA;
    st = cudec_gdeflate_decompress_batch(
        reinterpret_cast<const void* const*>(d), reinterpret_cast<const size_t*>(d + 8 * n),
        reinterpret_cast<void* const*>(d + 16 * n), reinterpret_cast<const size_t*>(d + 24 * n),
        n, d_res, reinterpret_cast<cudec_stream_t>(s.s));
    if (st != CUDEC_OK) return st;
    std::vector<cudec_chunk_result> res(n);
    ok = cudaMemcpyAsync(res.data(), d_res, 16 * n, cudaMemcpyDeviceToHost, s.s) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s.s) == cudaSuccess;
    if (!ok) return CUDEC_ERR_CUDA;
    // the first failing tile decides; a tile must produce exactly its size
    for (size_t i = 0; i < n; ++i) {
        if (res[i].status != CUDEC_OK) return static_cast<cudec_status>(res[i].status);
        if (res[i].bytes_written != tiles[i].dst_size) return CUDEC_ERR_CORRUPT_INPUT;
    }
    if (dst_space == CUDEC_MEM_HOST) {
        if (cudaMemcpyAsync(dst, d_out, total, cudaMemcpyDeviceToHost, s.s) != cudaSuccess ||
            cudaStreamSynchronize(s.s) != cudaSuccess)
            return CUDEC_ERR_CUDA;
    }
    *out_written = total;
    return CUDEC_OK;
}

}  // extern "C"
