// Pinned streaming decode context: host-resident compressed chunks in,
// device- or host-resident output, synchronous.
//
// Replaces iderex/cudec src/stream.cpp:42-593 with the same contract
// (argument rules, wave sizing by a staging budget and a chunk ceiling,
// grow-only staging, per-chunk records always defined, aggregate status = CUDA
// fault first, else the first non-OK chunk in index order, poison latch on a
// CUDA fault). The data path differs: the staging is double-buffered, so the
// host copies wave w+1's chunks into pinned memory while the device uploads,
// decodes and reads back wave w; host-side output comes back as one copy of
// the wave's staging into pinned memory and is scattered to the caller's
// buffers (exactly bytes_written each) while the next wave is on the device.
// When every compressed chunk of a call lies in page-locked host memory mapped
// for the device, no staging happens at all: the decode kernel reads the
// chunks over the host link itself, so the transfer overlaps the decode.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "cudec.h"
#include "host_util.h"
#include "launch.h"

namespace {

// Staging per wave: compressed bytes (+ host-output destination bytes) are
// charged at the largest chunk of the call, as the reference's sizer does
// (src/stream.cpp:58-105); two waves are staged at a time.
constexpr size_t kWaveBudget = size_t{192} << 20;
constexpr size_t kWaveChunksMax = 4096;

size_t choose_wave(const size_t* sizes, const size_t* caps, size_t n, bool host_out) {
    size_t per = 1;
    for (size_t i = 0; i < n; ++i) {
        size_t b = sizes[i];
        if (host_out) b = (SIZE_MAX - b < caps[i]) ? SIZE_MAX : b + caps[i];
        if (b > per) per = b;
    }
    size_t w = kWaveBudget / per;
    if (w == 0) w = 1;
    if (w > kWaveChunksMax) w = kWaveChunksMax;
    if (w > n) w = n;
    return w;
}

void stamp(cudec_chunk_result* r, size_t n, cudec_status st) {
    for (size_t i = 0; i < n; ++i) {
        r[i].status = static_cast<int32_t>(st);
        r[i].reserved = 0;
        r[i].bytes_written = 0;
    }
}

// Same rules as src/stream.cpp:182-201; no CUDA call.
cudec_status validate(const void* const* src, const size_t* sizes, void* const* dst,
                      const size_t* caps, size_t n, cudec_mem_space space,
                      const cudec_chunk_result* res) {
    if (src == nullptr || sizes == nullptr || dst == nullptr || caps == nullptr ||
        res == nullptr || n == 0 || n > cdb::kMaxBatchChunks ||
        (space != CUDEC_MEM_HOST && space != CUDEC_MEM_DEVICE))
        return CUDEC_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < n; ++i)
        if ((src[i] == nullptr && sizes[i] != 0) || (dst[i] == nullptr && caps[i] != 0))
            return CUDEC_ERR_INVALID_ARGUMENT;
    return CUDEC_OK;
}

// cuPointerGetAttribute through the runtime's driver entry point (the library
// does not link libcuda); null when the driver does not offer it.
using PtrAttrFn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);

PtrAttrFn ptr_attr() {
    static const PtrAttrFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            return static_cast<PtrAttrFn>(nullptr);
        }
        return reinterpret_cast<PtrAttrFn>(f);
    }();
    return fn;
}

// The page-locked host allocation holding `p`, when it is mapped into the
// current context at the same address (unified addressing): [lo, hi).
bool pinned_range(const void* p, uintptr_t* lo, uintptr_t* hi) {
    const PtrAttrFn get = ptr_attr();
    if (get == nullptr) return false;
    const CUdeviceptr a = reinterpret_cast<CUdeviceptr>(p);
    unsigned int type = 0;
    CUdeviceptr dev = 0, start = 0;
    size_t span = 0;
    if (get(&type, CU_POINTER_ATTRIBUTE_MEMORY_TYPE, a) != CUDA_SUCCESS ||
        type != CU_MEMORYTYPE_HOST ||
        get(&dev, CU_POINTER_ATTRIBUTE_DEVICE_POINTER, a) != CUDA_SUCCESS || dev != a ||
        get(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, a) != CUDA_SUCCESS ||
        get(&span, CU_POINTER_ATTRIBUTE_RANGE_SIZE, a) != CUDA_SUCCESS || span == 0 ||
        start > a || a - start >= span)
        return false;
    *lo = static_cast<uintptr_t>(start);
    *hi = static_cast<uintptr_t>(start) + span;
    return true;
}

// True when the device can read every chunk in place: each [src, src+size)
// inside one mapped page-locked allocation. One driver query per allocation
// met (the last range is remembered), so a packed batch costs one query.
// The decode kernel's window fill reads whole aligned 16-byte blocks around
// a chunk; such a block shares its page with the chunk byte it holds, and
// page-locked allocations are locked and mapped in whole pages.
bool device_readable(const void* const* src, const size_t* sizes, size_t n) {
    uintptr_t lo = 0, hi = 0;
    for (size_t i = 0; i < n; ++i) {
        if (sizes[i] == 0) continue;
        const uintptr_t a = reinterpret_cast<uintptr_t>(src[i]);
        if (a < lo || a >= hi) {
            if (!pinned_range(src[i], &lo, &hi)) return false;
        }
        if (sizes[i] > hi - a) return false;
    }
    return true;
}

}  // namespace

struct cudec_stream_ctx {
    cdb::StreamOwner stream;
    cdb::EventOwner drained[2];  // slot b's wave is done (staging reusable)
    cdb::PinnedBuf p_src[2], p_meta[2], p_out[2];
    cdb::DevBuf d_src[2], d_meta[2], d_out[2];
    cdb::DevBuf d_results;
    cdb::PinnedBuf p_results;
    bool poisoned = false;
};

namespace {

// Copy one drained host-output wave from pinned staging to the caller:
// exactly bytes_written per chunk, bounded by the chunk's capacity (a longer
// device-reported length is a device fault: the chunk is stamped CUDA and
// the wave fails, as src/stream.cpp:163-184 does).
// Host copies of a wave: kParallelCopy bytes or more are split into ranges
// of consecutive chunks of about equal bytes over up to 16 host threads (the
// calling thread takes the first range); fewer go on the calling thread.
// bytes(j) is chunk j's share; copy(j0, j1, k) copies chunks [j0, j1), k
// being the range's index (its starting offsets are the caller's to keep).
constexpr size_t kParallelCopy = size_t{4} << 20;

template <class Bytes, class Copy>
void parallel_copy(size_t wn, size_t total, Bytes bytes, Copy copy) {
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nt = std::min<size_t>({hw ? hw : 1u, 16u, wn});
    if (total < kParallelCopy || nt < 2) {
        copy(size_t{0}, wn);
        return;
    }
    std::vector<size_t> jb(1, 0);
    size_t acc = 0;
    for (size_t j = 0; j < wn; ++j) {
        acc += bytes(j);
        if (jb.size() < nt && acc >= total / nt * jb.size() && j + 1 < wn) jb.push_back(j + 1);
    }
    jb.push_back(wn);
    std::vector<std::thread> threads;
    size_t r = 1;
    try {
        for (; r + 1 < jb.size(); ++r) threads.emplace_back(copy, jb[r], jb[r + 1]);
    } catch (...) {  // no thread to be had: the rest on this one
        for (; r + 1 < jb.size(); ++r) copy(jb[r], jb[r + 1]);
    }
    copy(jb[0], jb[1]);
    for (std::thread& th : threads) th.join();
}

// Every record is checked before any byte moves.
cudec_status scatter_wave(cudec_chunk_result* wr, const unsigned char* staged,
                          void* const* dst, const size_t* caps, size_t begin, size_t wn) {
    size_t total = 0;
    for (size_t j = 0; j < wn; ++j) {
        const size_t i = begin + j;
        const size_t bw = static_cast<size_t>(wr[j].bytes_written);
        if (bw > caps[i]) {
            wr[j].status = CUDEC_ERR_CUDA;
            wr[j].reserved = 0;
            wr[j].bytes_written = 0;
            return CUDEC_ERR_CUDA;
        }
        total += bw;
    }
    // staging offsets: chunk j's slot starts at the sum of the earlier caps
    std::vector<size_t> at(wn + 1, 0);
    for (size_t j = 0; j < wn; ++j) at[j + 1] = at[j] + caps[begin + j];
    parallel_copy(
        wn, total, [&](size_t j) { return static_cast<size_t>(wr[j].bytes_written); },
        [&](size_t j0, size_t j1) {
            for (size_t j = j0; j < j1; ++j) {
                const size_t i = begin + j;
                const size_t bw = static_cast<size_t>(wr[j].bytes_written);
                if (bw != 0 && dst[i] != nullptr) std::memcpy(dst[i], staged + at[j], bw);
            }
        });
    return CUDEC_OK;
}

cudec_status decode(cudec_stream_ctx& ctx, const void* const* src, const size_t* sizes,
                    void* const* dst, const size_t* caps, size_t n, cudec_mem_space space,
                    cudec_chunk_result* results) {
    const bool host_out = space == CUDEC_MEM_HOST;
    const size_t wave = choose_wave(sizes, caps, n, host_out);
    const size_t waves = (n + wave - 1) / wave;
    stamp(results, n, CUDEC_ERR_CUDA);
    const bool in_place = device_readable(src, sizes, n);

    size_t max_src = 0, max_out = 0;
    for (size_t w = 0; w < waves; ++w) {
        const size_t b = w * wave, e = b + wave < n ? b + wave : n;
        size_t ws = 0, wo = 0;
        for (size_t i = b; i < e; ++i) {
            if (SIZE_MAX - ws < sizes[i]) return CUDEC_ERR_CORRUPT_INPUT;
            ws += sizes[i];
            if (host_out) {
                if (SIZE_MAX - wo < caps[i]) return CUDEC_ERR_CORRUPT_INPUT;
                wo += caps[i];
            }
        }
        if (ws > max_src) max_src = ws;
        if (wo > max_out) max_out = wo;
    }
    if (n > SIZE_MAX / sizeof(cudec_chunk_result)) return CUDEC_ERR_CORRUPT_INPUT;
    const size_t meta_bytes = 4 * wave * sizeof(uint64_t);
    const size_t res_bytes = n * sizeof(cudec_chunk_result);
#define GROW(call)                       \
    do {                                 \
        if ((call) != cudaSuccess) {     \
            (void)cudaGetLastError();    \
            ctx.poisoned = true;         \
            return CUDEC_ERR_CUDA;       \
        }                                \
    } while (0)
    const size_t slots = waves > 1 ? 2 : 1;
    for (size_t b = 0; b < slots; ++b) {
        if (!in_place) {
            GROW(ctx.p_src[b].ensure(max_src ? max_src : 1));
            GROW(ctx.d_src[b].ensure(max_src ? max_src : 1));
        }
        GROW(ctx.p_meta[b].ensure(meta_bytes));
        GROW(ctx.d_meta[b].ensure(meta_bytes));
        if (host_out) {
            GROW(ctx.d_out[b].ensure(max_out ? max_out : 1));
            GROW(ctx.p_out[b].ensure(max_out ? max_out : 1));
        }
    }
    GROW(ctx.d_results.ensure(res_bytes));
    GROW(ctx.p_results.ensure(res_bytes));
#undef GROW
    cudaStream_t s = ctx.stream.s;
    cudec_chunk_result* p_res = static_cast<cudec_chunk_result*>(ctx.p_results.p);
    stamp(p_res, n, CUDEC_ERR_CUDA);

    // Host output in one wave to destinations that sit back to back in index
    // order (one caller buffer): once every chunk is known to have filled
    // its capacity, the decoded wave goes to the caller in one copy, with no
    // staging pass; otherwise it takes the staged path below.
    bool direct = host_out && waves == 1 && dst[0] != nullptr;
    for (size_t i = 1; i < n && direct; ++i)
        if (static_cast<unsigned char*>(dst[i]) !=
            static_cast<unsigned char*>(dst[i - 1]) + caps[i - 1])
            direct = false;

    cudec_status fail = CUDEC_OK;
    bool slot_busy[2] = {false, false};
    size_t slot_begin[2] = {0, 0}, slot_n[2] = {0, 0};
    // Host-output: finish (scatter) the wave staged in `slot`.
    auto finish_slot = [&](int slot) -> cudec_status {
        if (!slot_busy[slot]) return CUDEC_OK;
        if (cudaEventSynchronize(ctx.drained[slot].e) != cudaSuccess) return CUDEC_ERR_CUDA;
        slot_busy[slot] = false;
        if (!host_out) return CUDEC_OK;
        return scatter_wave(p_res + slot_begin[slot],
                            static_cast<const unsigned char*>(ctx.p_out[slot].p), dst, caps,
                            slot_begin[slot], slot_n[slot]);
    };
    for (size_t w = 0; w < waves && fail == CUDEC_OK; ++w) {
        const int b = static_cast<int>(w & 1);
        const size_t begin = w * wave, end = begin + wave < n ? begin + wave : n;
        const size_t wn = end - begin;
        // The slot's previous wave must be fully out of its staging.
        if ((fail = finish_slot(b)) != CUDEC_OK) break;
        unsigned char* ps = static_cast<unsigned char*>(ctx.p_src[b].p);
        unsigned char* ds = static_cast<unsigned char*>(ctx.d_src[b].p);
        unsigned char* dout = static_cast<unsigned char*>(ctx.d_out[b].p);
        uint64_t* pm = static_cast<uint64_t*>(ctx.p_meta[b].p);
        // Sources laid out back to back (the usual packed batch) go up in one
        // copy straight from the caller's memory: a DMA when it is pinned, a
        // driver-staged copy otherwise (faster, measured, than packing them
        // into the pinned staging on host threads first); scattered sources
        // are packed into the staging.
        bool contiguous = !in_place;
        for (size_t j = 1; j < wn && contiguous; ++j) {
            const size_t i = begin + j;
            if (sizes[i] && static_cast<const unsigned char*>(src[i]) !=
                                static_cast<const unsigned char*>(src[i - 1]) + sizes[i - 1])
                contiguous = false;
        }
        size_t so = 0, oo = 0;
        for (size_t j = 0; j < wn; ++j) {
            const size_t i = begin + j;
            if (in_place) {
                pm[j] = reinterpret_cast<uint64_t>(src[i]);
            } else {
                if (sizes[i] && !contiguous) std::memcpy(ps + so, src[i], sizes[i]);
                pm[j] = reinterpret_cast<uint64_t>(ds + so);
            }
            pm[wave + j] = sizes[i];
            pm[2 * wave + j] = host_out ? reinterpret_cast<uint64_t>(dout + oo)
                                        : reinterpret_cast<uint64_t>(dst[i]);
            pm[3 * wave + j] = caps[i];
            so += sizes[i];
            if (host_out) oo += caps[i];
        }
        const void* up = contiguous ? src[begin] : static_cast<const void*>(ps);
        if (!in_place && so &&
            cudaMemcpyAsync(ds, up, so, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            fail = CUDEC_ERR_CUDA;
            break;
        }
        if (cudaMemcpyAsync(ctx.d_meta[b].p, pm, meta_bytes, cudaMemcpyHostToDevice, s) !=
            cudaSuccess) {
            fail = CUDEC_ERR_CUDA;
            break;
        }
        const uint64_t* dm = static_cast<const uint64_t*>(ctx.d_meta[b].p);
        cudec_chunk_result* d_res = static_cast<cudec_chunk_result*>(ctx.d_results.p) + begin;
        const cudec_status launched = cudec_lz4_decompress_batch(
            reinterpret_cast<const void* const*>(dm), reinterpret_cast<const size_t*>(dm + wave),
            reinterpret_cast<void* const*>(dm + 2 * wave),
            reinterpret_cast<const size_t*>(dm + 3 * wave), wn, d_res, s);
        if (launched != CUDEC_OK) {
            fail = launched;
            break;
        }
        if (cudaMemcpyAsync(p_res + begin, d_res, wn * sizeof(cudec_chunk_result),
                            cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            fail = CUDEC_ERR_CUDA;
            break;
        }
        if (host_out && oo && !direct &&
            cudaMemcpyAsync(ctx.p_out[b].p, dout, oo, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            fail = CUDEC_ERR_CUDA;
            break;
        }
        if (cudaEventRecord(ctx.drained[b].e, s) != cudaSuccess) {
            fail = CUDEC_ERR_CUDA;
            break;
        }
        slot_busy[b] = true;
        slot_begin[b] = begin;
        slot_n[b] = wn;
    }
    // Drain: no work outlives the call.
    cudec_status drain = fail;
    if (cudaStreamSynchronize(s) != cudaSuccess && drain == CUDEC_OK) drain = CUDEC_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess && drain == CUDEC_OK) drain = CUDEC_ERR_CUDA;
    if (drain == CUDEC_OK && direct && slot_busy[0]) {
        // the records are in: every chunk full means one copy to the caller
        size_t total = 0;
        bool full = true;
        for (size_t i = 0; i < n; ++i) {
            full = full && p_res[i].status == CUDEC_OK &&
                   static_cast<size_t>(p_res[i].bytes_written) == caps[i];
            total += caps[i];
        }
        const void* dout = ctx.d_out[0].p;
        void* to = full ? dst[0] : ctx.p_out[0].p;
        if (total && (cudaMemcpyAsync(to, dout, total, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess))
            drain = CUDEC_ERR_CUDA;
        else if (full)
            slot_busy[0] = false;  // delivered; otherwise scattered from staging below
    }
    if (drain == CUDEC_OK) {
        // finish in wave order (the older slot first)
        const int first = waves > 1 ? static_cast<int>((waves - 2) & 1) : 0;
        for (int k = 0; k < 2 && drain == CUDEC_OK; ++k) {
            const int slot = (first + k) & 1;
            drain = finish_slot(slot);
        }
    }
    if (drain != CUDEC_OK && host_out) {
        // Waves whose output never reached the caller are not decodes.
        for (int slot = 0; slot < 2; ++slot)
            if (slot_busy[slot]) stamp(p_res + slot_begin[slot], slot_n[slot], CUDEC_ERR_CUDA);
    }
    std::memcpy(results, p_res, res_bytes);
    if (drain != CUDEC_OK) {
        ctx.poisoned = true;
        return drain;
    }
    for (size_t i = 0; i < n; ++i)
        if (results[i].status != CUDEC_OK) return static_cast<cudec_status>(results[i].status);
    return CUDEC_OK;
}

}  // namespace

extern "C" {

// Library-internal probe (not part of the C ABI): 1 when the streaming
// context would let the device read these chunks in place.
__attribute__((visibility("default"))) int cdb_stream_reads_in_place(
    const void* const* src, const size_t* sizes, size_t n) {
    return (src != nullptr && sizes != nullptr && device_readable(src, sizes, n)) ? 1 : 0;
}

cudec_status cudec_stream_ctx_create(cudec_stream_ctx** out_ctx) {
    if (out_ctx == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    *out_ctx = nullptr;
    cudec_stream_ctx* ctx = new (std::nothrow) cudec_stream_ctx();
    if (ctx == nullptr) return CUDEC_ERR_CUDA;
    if (ctx->stream.create() != cudaSuccess || ctx->drained[0].create() != cudaSuccess ||
        ctx->drained[1].create() != cudaSuccess) {
        (void)cudaGetLastError();
        delete ctx;
        return CUDEC_ERR_CUDA;
    }
    *out_ctx = ctx;
    return CUDEC_OK;
}

cudec_status cudec_lz4_decompress_stream_ctx(cudec_stream_ctx* ctx,
                                             const void* const* h_src_ptrs,
                                             const size_t* h_src_sizes, void* const* dst_ptrs,
                                             const size_t* dst_caps, size_t chunk_count,
                                             cudec_mem_space dst_space,
                                             cudec_chunk_result* h_results) {
    if (ctx == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    const cudec_status a = validate(h_src_ptrs, h_src_sizes, dst_ptrs, dst_caps, chunk_count,
                                    dst_space, h_results);
    if (a != CUDEC_OK) return a;
    if (ctx->poisoned) {
        stamp(h_results, chunk_count, CUDEC_ERR_CUDA);
        return CUDEC_ERR_CUDA;
    }
    try {
        return decode(*ctx, h_src_ptrs, h_src_sizes, dst_ptrs, dst_caps, chunk_count, dst_space,
                      h_results);
    } catch (...) {
        ctx->poisoned = true;
        return CUDEC_ERR_CUDA;
    }
}

void cudec_stream_ctx_destroy(cudec_stream_ctx* ctx) {
    if (ctx == nullptr) return;
    if (ctx->stream.s != nullptr) (void)cudaStreamSynchronize(ctx->stream.s);
    delete ctx;
}

cudec_status cudec_lz4_decompress_stream(const void* const* h_src_ptrs,
                                         const size_t* h_src_sizes, void* const* dst_ptrs,
                                         const size_t* dst_caps, size_t chunk_count,
                                         cudec_mem_space dst_space,
                                         cudec_chunk_result* h_results) {
    const cudec_status a = validate(h_src_ptrs, h_src_sizes, dst_ptrs, dst_caps, chunk_count,
                                    dst_space, h_results);
    if (a != CUDEC_OK) return a;
    cudec_stream_ctx* ctx = nullptr;
    const cudec_status c = cudec_stream_ctx_create(&ctx);
    if (c != CUDEC_OK) return c;
    const cudec_status st = cudec_lz4_decompress_stream_ctx(
        ctx, h_src_ptrs, h_src_sizes, dst_ptrs, dst_caps, chunk_count, dst_space, h_results);
    cudec_stream_ctx_destroy(ctx);
    return st;
}

}  // extern "C"
