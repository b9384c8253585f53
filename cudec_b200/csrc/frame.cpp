// cudec_lz4f_decompress: one .lz4 frame, host memory in, host memory out.
//
// Replaces iderex/cudec src/frame.cpp:53-422 with the same accept/reject
// ladder (header, block table, checksums, content size) and the same
// statuses, on a different data path: the frame's compressed blocks go to the
// device in ONE copy straight out of the caller's frame (no host gather), the
// block table goes up in one packed copy, all blocks decode in one batch
// launch on a private stream into block_max-strided slots, and the decoded
// bytes come back in as few copies as the layout allows (runs of full blocks
// are contiguous on both sides). Device memory comes from a cached
// stream-ordered pool, so repeated frames do not pay driver allocations.
//
// Frame format: the public LZ4 frame format specification (magic 0x184D2204,
// FLG/BD descriptor, optional content size, header checksum, size-prefixed
// blocks with the uncompressed flag in bit 31, optional block checksums, end
// mark, optional content checksum), XXH32 with seed 0 throughout.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <functional>
#include <new>
#include <thread>
#include <vector>

#include "cudec.h"
#include "host_util.h"
#include "launch.h"
#include "xxhash32.h"

namespace {

using cdb::xxh32;

constexpr uint32_t kFrameMagic = 0x184D2204u;

uint32_t rd32(const unsigned char* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
uint64_t rd64(const unsigned char* p) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
}

struct Block {
    size_t off;
    size_t len;
    bool raw;  // stored uncompressed
};

// Block checksums of a frame, verified on host threads while the device
// decodes the blocks: every block is independent, and any mismatch is the
// same CORRUPT_INPUT that the walk would have returned at that block, so the
// order of the checks does not show. Frames with less than kParallelBytes of
// blocks are verified by the calling thread.
class BlockSums {
  public:
    static constexpr size_t kParallelBytes = size_t{4} << 20;

    BlockSums(const unsigned char* f, const std::vector<Block>& blocks, bool present)
        : f_(f), blocks_(blocks) {
        if (!present || blocks.empty()) return;
        size_t bytes = 0;
        for (const Block& b : blocks) bytes += b.len;
        unsigned hw = std::thread::hardware_concurrency();
        const size_t nt = std::min<size_t>({hw ? hw : 1u, 16u, blocks.size()});
        if (bytes < kParallelBytes || nt < 2) {
            ok_ = check(0, 1);
            return;
        }
        try {
            for (size_t t = 0; t < nt; ++t)
                threads_.emplace_back([this, t, nt] {
                    if (!check(t, nt)) bad_.store(true, std::memory_order_relaxed);
                });
        } catch (...) {  // no thread to be had: the rest on this one
            const size_t started = threads_.size();
            for (size_t t = started; t < nt; ++t)
                if (!check(t, nt)) bad_.store(true, std::memory_order_relaxed);
        }
    }
    ~BlockSums() { join(); }
    BlockSums(const BlockSums&) = delete;
    BlockSums& operator=(const BlockSums&) = delete;

    // Whether every block checksum matched (waits for the threads).
    bool ok() {
        join();
        return ok_ && !bad_.load(std::memory_order_relaxed);
    }

  private:
    // Blocks t, t + nt, ...: the 4-byte checksum follows each block.
    bool check(size_t t, size_t nt) const {
        for (size_t i = t; i < blocks_.size(); i += nt) {
            const Block& b = blocks_[i];
            if (xxh32(f_ + b.off, b.len) != rd32(f_ + b.off + b.len)) return false;
        }
        return true;
    }
    void join() {
        for (std::thread& th : threads_)
            if (th.joinable()) th.join();
    }

    const unsigned char* f_;
    const std::vector<Block>& blocks_;
    std::vector<std::thread> threads_;
    std::atomic<bool> bad_{false};
    bool ok_ = true;
};

#define FCUDA(call)                                   \
    do {                                              \
        if ((call) != cudaSuccess) {                  \
            (void)cudaGetLastError();                 \
            return CUDEC_ERR_CUDA;                    \
        }                                             \
    } while (0)

// Decode the compressed blocks and place every block's bytes in `out`
// (follows src/frame.cpp:53-278 for the statuses: any block reject is
// CORRUPT_INPUT, the caller's capacity is checked before the first byte is
// written, OUTPUT_TOO_SMALL otherwise).
// `sums_ok` runs once the device results are in and before anything is
// checked against the caller's capacity or copied to the caller: false (a
// block checksum mismatch) is CORRUPT_INPUT with the output untouched, as
// when the walk itself rejects the block.
cudec_status decode_blocks(const unsigned char* f, const std::vector<Block>& blocks,
                           size_t block_max, unsigned char* out, size_t cap,
                           size_t* total_out, const std::function<bool()>& sums_ok) {
    std::vector<size_t> comp;
    for (size_t i = 0; i < blocks.size(); ++i)
        if (!blocks[i].raw) comp.push_back(i);
    const size_t n = comp.size();
    std::vector<size_t> dec_len(blocks.size(), 0);

    cdb::StreamOwner stream;
    cdb::AsyncBuf d_src, d_dst, d_meta, d_res;
    if (n != 0) {
        if (block_max != 0 && n > SIZE_MAX / block_max) return CUDEC_ERR_CORRUPT_INPUT;
        if (n > SIZE_MAX / (4 * sizeof(void*))) return CUDEC_ERR_CORRUPT_INPUT;
        FCUDA(stream.create());
        // One copy of the frame span holding every compressed block.
        const size_t lo = blocks[comp.front()].off;
        const size_t hi = blocks[comp.back()].off + blocks[comp.back()].len;
        FCUDA(d_src.alloc(hi - lo, stream.s));
        FCUDA(d_dst.alloc(n * block_max, stream.s));
        FCUDA(d_meta.alloc(4 * n * sizeof(void*), stream.s));
        FCUDA(d_res.alloc(n * sizeof(cudec_chunk_result), stream.s));
        FCUDA(cudaMemcpyAsync(d_src.p, f + lo, hi - lo, cudaMemcpyHostToDevice, stream.s));
        std::vector<uint64_t> meta(4 * n);
        unsigned char* ds = static_cast<unsigned char*>(d_src.p);
        unsigned char* dd = static_cast<unsigned char*>(d_dst.p);
        for (size_t k = 0; k < n; ++k) {
            const Block& b = blocks[comp[k]];
            meta[k] = reinterpret_cast<uint64_t>(ds + (b.off - lo));
            meta[n + k] = b.len;
            meta[2 * n + k] = reinterpret_cast<uint64_t>(dd + k * block_max);
            meta[3 * n + k] = block_max;
        }
        FCUDA(cudaMemcpyAsync(d_meta.p, meta.data(), meta.size() * 8,
                              cudaMemcpyHostToDevice, stream.s));
        const uint64_t* dm = static_cast<const uint64_t*>(d_meta.p);
        const cudec_status launched = cudec_lz4_decompress_batch(
            reinterpret_cast<const void* const*>(dm), reinterpret_cast<const size_t*>(dm + n),
            reinterpret_cast<void* const*>(dm + 2 * n), reinterpret_cast<const size_t*>(dm + 3 * n),
            n, static_cast<cudec_chunk_result*>(d_res.p), stream.s);
        if (launched != CUDEC_OK) return launched;
        std::vector<cudec_chunk_result> res(n);
        FCUDA(cudaMemcpyAsync(res.data(), d_res.p, n * sizeof(cudec_chunk_result),
                              cudaMemcpyDeviceToHost, stream.s));
        FCUDA(cudaStreamSynchronize(stream.s));
        if (!sums_ok()) return CUDEC_ERR_CORRUPT_INPUT;
        for (size_t k = 0; k < n; ++k) {
            // The per-block capacity is ours (block_max), never the caller's:
            // every block-level reject is a corrupt frame.
            if (res[k].status != CUDEC_OK || res[k].bytes_written > block_max)
                return CUDEC_ERR_CORRUPT_INPUT;
            dec_len[comp[k]] = static_cast<size_t>(res[k].bytes_written);
        }
    }
    if (n == 0 && !sums_ok()) return CUDEC_ERR_CORRUPT_INPUT;
    size_t total = 0;
    for (size_t i = 0; i < blocks.size(); ++i) {
        const size_t len = blocks[i].raw ? blocks[i].len : dec_len[i];
        if (len > cap - total) return CUDEC_ERR_OUTPUT_TOO_SMALL;
        total += len;
    }
    // Place blocks; merge device runs that are contiguous on both sides.
    size_t run_dev = 0, run_out = 0, run_len = 0, off = 0, k = 0;
    for (size_t i = 0; i < blocks.size(); ++i) {
        if (blocks[i].raw) {
            if (blocks[i].len) std::memcpy(out + off, f + blocks[i].off, blocks[i].len);
            off += blocks[i].len;
            continue;
        }
        const size_t len = dec_len[i], dev = k * block_max;
        if (run_len != 0 && run_dev + run_len == dev && run_out + run_len == off) {
            run_len += len;
        } else {
            if (run_len)
                FCUDA(cudaMemcpyAsync(out + run_out, static_cast<unsigned char*>(d_dst.p) + run_dev,
                                      run_len, cudaMemcpyDeviceToHost, stream.s));
            run_dev = dev;
            run_out = off;
            run_len = len;
        }
        off += len;
        ++k;
    }
    if (run_len)
        FCUDA(cudaMemcpyAsync(out + run_out, static_cast<unsigned char*>(d_dst.p) + run_dev,
                              run_len, cudaMemcpyDeviceToHost, stream.s));
    if (n) FCUDA(cudaStreamSynchronize(stream.s));
    *total_out = total;
    return CUDEC_OK;
}

// The frame ladder, in the order of src/frame.cpp:282-397.
cudec_status decode_frame(const unsigned char* f, size_t size, unsigned char* out,
                          size_t cap, size_t* written) {
    if (size < 7 || rd32(f) != kFrameMagic) return CUDEC_ERR_CORRUPT_INPUT;
    const unsigned flg = f[4], bd = f[5];
    if (((flg >> 6) & 3) != 1 || (flg & 2) != 0) return CUDEC_ERR_CORRUPT_INPUT;
    const bool independent = (flg >> 5) & 1;
    const bool block_sum = (flg >> 4) & 1;
    const bool has_size = (flg >> 3) & 1;
    const bool content_sum = (flg >> 2) & 1;
    const bool dict = flg & 1;
    if ((bd & 0x8F) != 0) return CUDEC_ERR_CORRUPT_INPUT;
    const unsigned bmax = (bd >> 4) & 7;
    if (bmax < 4 || bmax > 7) return CUDEC_ERR_CORRUPT_INPUT;
    const size_t block_max = size_t{65536} << ((bmax - 4) * 2);
    if (!independent || dict) return CUDEC_ERR_UNSUPPORTED;
    size_t pos = 6;
    uint64_t declared = 0;
    if (has_size) {
        if (size < pos + 8) return CUDEC_ERR_CORRUPT_INPUT;
        declared = rd64(f + pos);
        pos += 8;
    }
    if (size < pos + 1) return CUDEC_ERR_CORRUPT_INPUT;
    if (((xxh32(f + 4, pos - 4) >> 8) & 0xFF) != f[pos]) return CUDEC_ERR_CORRUPT_INPUT;
    pos += 1;

    std::vector<Block> blocks;
    bool end = false;
    // Every step consumes at least 4 bytes; the bound is unreachable for a
    // frame the checks admit and turns a bounds bug into a reject.
    for (uint64_t fuel = size / 4 + 1; fuel != 0; --fuel) {
        if (size < pos + 4) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t bs = rd32(f + pos);
        pos += 4;
        if (bs == 0) {
            end = true;
            break;
        }
        const bool raw = (bs >> 31) & 1;
        const size_t blen = bs & 0x7FFFFFFFu;
        if (blen == 0 || blen > block_max || size < pos + blen) return CUDEC_ERR_CORRUPT_INPUT;
        if (block_sum && size < pos + blen + 4) return CUDEC_ERR_CORRUPT_INPUT;
        blocks.push_back({pos, blen, raw});
        pos += blen + (block_sum ? 4 : 0);
    }
    if (!end) return CUDEC_ERR_CORRUPT_INPUT;
    size_t total = 0;
    // the checksum values are verified while the blocks decode
    BlockSums sums(f, blocks, block_sum);
    const cudec_status st =
        decode_blocks(f, blocks, block_max, out, cap, &total, [&sums] { return sums.ok(); });
    // a checksum mismatch outranks whatever the device path met (the walk
    // would have stopped before any CUDA call)
    if (st != CUDEC_OK) return sums.ok() ? st : CUDEC_ERR_CORRUPT_INPUT;
    if (has_size && declared != total) return CUDEC_ERR_CORRUPT_INPUT;
    if (content_sum) {
        if (size < pos + 4) return CUDEC_ERR_CORRUPT_INPUT;
        if (xxh32(out, total) != rd32(f + pos)) return CUDEC_ERR_CORRUPT_INPUT;
    }
    *written = total;
    return CUDEC_OK;
}

}  // namespace

extern "C" cudec_status cudec_lz4f_decompress(const void* frame, size_t frame_size,
                                              void* dst, size_t dst_capacity,
                                              size_t* bytes_written) {
    if (bytes_written != nullptr) *bytes_written = 0;
    if (frame == nullptr || bytes_written == nullptr || (dst == nullptr && dst_capacity != 0))
        return CUDEC_ERR_INVALID_ARGUMENT;
    try {
        return decode_frame(static_cast<const unsigned char*>(frame), frame_size,
                            static_cast<unsigned char*>(dst), dst_capacity, bytes_written);
    } catch (...) {
        // A host allocation failed: a defined resource error, never a throw
        // across the ABI.
        *bytes_written = 0;
        return CUDEC_ERR_CUDA;
    }
}
