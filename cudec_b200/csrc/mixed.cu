// Persistent mixed-format batch decode.
//
// One launch decodes a batch whose chunks are LZ4 blocks, raw Snappy blocks,
// Zstd frames and GDeflate pages in any mix and of any sizes (a per-chunk
// format code). A
// plan owns everything the launch needs so the call allocates nothing:
//
//   * a largest-first order of the chunks (by output capacity), built on the
//     device by a counting sort over log2 size classes, so the longest
//     chunks start first and the tail of the launch is short chunks;
//   * a work counter: every warp of the persistent grid takes the next chunk
//     of that order with one atomic add (work stealing), whatever its format;
//   * warps per chunk by size bucket: LZ4 and Snappy chunks of the buckets
//     set to a whole CTA go first in the order (largest first among them)
//     and are taken, one chunk per CTA, by the CTA-per-chunk decoder
//     (lz_cta_kernel.cuh) in a second persistent grid that runs beside the
//     warp grid; the warp grid starts after them;
//   * per-warp Zstd literal slots;
//   * the decode shape per size bucket (warps per chunk; for one warp, the
//     parse window, input lookahead and ring batch) chosen by
//     cudec_mixed_plan_tune, which times candidate shapes on the caller's
//     own chunks, bucket by bucket, or set by the caller (a saved table);
//   * a CUDA graph of the whole sequence (counter reset, order kernels,
//     decode kernel), captured once per argument set and replayed.
//
// Per-chunk statuses and bytes are exactly those of the per-format entries
// (the same device decoders run); an unknown format code is
// CUDEC_ERR_UNSUPPORTED for that chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "cudec.h"
#include "host_util.h"
#include "launch.h"
#include "gdeflate_page.cuh"
#include "lz_cta_kernel.cuh"
#include "lz_warp_kernel.cuh"
#include "mixed.h"
#include "zstd_frame.cuh"

namespace cdb {
namespace mixed {

constexpr uint32_t kWarps = 4;
constexpr uint32_t kThreads = 32 * kWarps;
constexpr uint32_t kMaxOf(uint32_t a, uint32_t b) { return a > b ? a : b; }
constexpr uint32_t kWarpSmem =
    kMaxOf(kMaxOf(lzw::kWarpSmem, static_cast<uint32_t>(sizeof(zstd::WarpSmem))),
           static_cast<uint32_t>(sizeof(gdf::Tables)));
constexpr uint32_t kSmem = kWarps * kWarpSmem;
constexpr int kBuckets = CUDEC_MIXED_BUCKETS;
constexpr int kSizeClasses = 64;  // floor(log2(capacity)) classes for the order
constexpr int kClasses = 2 * kSizeClasses;  // CTA-decoded chunks: the upper half
constexpr uint32_t kCtaWarps = lzc::kWarps;  // warps per chunk of the CTA decoder
// Resident CTAs per SM of the CTA grid, at most: three leave room for the
// warp grid that decodes beside it (with four, which the shared memory
// allows, 30,000 uneven LZ4 + Snappy chunks took 7 % longer).
constexpr int kCtaPerSmMax = 3;
static_assert(kCtaWarps == CUDEC_MIXED_CTA_WARPS, "the ABI's whole-CTA warps value");
constexpr uint32_t kCtaSmem = kMaxOf(static_cast<uint32_t>(sizeof(lzc::Shm<lzc::Lz4F>)),
                                     static_cast<uint32_t>(sizeof(lzc::Shm<lzc::SnappyF>)));
static_assert(kWarpSmem % 16 == 0, "per-warp regions stay 16-byte aligned");

// Tuning buckets by output capacity: < 4 KiB, < 16 KiB, < 64 KiB, < 256 KiB,
// < 1 MiB, larger.
__host__ __device__ inline int size_bucket(uint64_t cap) {
    return cap < 4096 ? 0 : cap < 16384 ? 1 : cap < 65536 ? 2 : cap < 262144 ? 3
         : cap < 1048576 ? 4 : 5;
}

__device__ __forceinline__ int size_class(uint64_t cap) {
    return cap ? 63 - __clzll(static_cast<long long>(cap)) : 0;
}

// The order class of chunk i: its size class, in the upper half when its
// bucket decodes LZ4 / Snappy with a whole CTA (bit b of cta_buckets).
__device__ __forceinline__ int order_class(uint64_t cap, uint8_t fmt, uint32_t cta_buckets) {
    const bool cta = (fmt == CUDEC_FORMAT_LZ4 || fmt == CUDEC_FORMAT_SNAPPY) &&
                     ((cta_buckets >> size_bucket(cap)) & 1u);
    return size_class(cap) + (cta ? kSizeClasses : 0);
}

struct Args {
    const void* const* src;
    const size_t* sizes;
    void* const* dst;
    const size_t* caps;
    const uint8_t* formats;
    size_t n;
    cudec_chunk_result* results;
    const uint32_t* order;
    unsigned long long* counter;
    const unsigned long long* first;  // order index of the warp grid's first chunk
    uint8_t* zstd_slots;
    lzw::Tune tune[kBuckets];
};

// Control block in device memory: the warp grid's and the CTA grid's work
// counters, class counts and cursors, and the number of CTA-decoded chunks
// (they occupy order[0, ncta)).
struct Ctrl {
    unsigned long long counter;
    unsigned long long cta_counter;
    unsigned long long ncta;
    unsigned long long counts[kClasses];
    unsigned long long cursor[kClasses];
};

__global__ void order_count(const size_t* caps, const uint8_t* formats, size_t n,
                            uint32_t cta_buckets, Ctrl* ctrl) {
    __shared__ unsigned int h[kClasses];
    for (uint32_t i = threadIdx.x; i < kClasses; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        atomicAdd(&h[order_class(caps[i], formats[i], cta_buckets)], 1u);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kClasses; i += blockDim.x)
        if (h[i]) atomicAdd(&ctrl->counts[i], static_cast<unsigned long long>(h[i]));
}

// Start of each class in the order, largest class first, the CTA-decoded
// half before the rest (one thread).
__global__ void order_scan(Ctrl* ctrl) {
    if (threadIdx.x != 0) return;
    unsigned long long at = 0;
    for (int c = kClasses - 1; c >= 0; --c) {
        ctrl->cursor[c] = at;
        at += ctrl->counts[c];
        if (c == kSizeClasses) ctrl->ncta = at;
    }
}

__global__ void order_place(const size_t* caps, const uint8_t* formats, size_t n,
                            uint32_t cta_buckets, Ctrl* ctrl, uint32_t* order) {
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int c = order_class(caps[i], formats[i], cta_buckets);
        const unsigned long long at = atomicAdd(&ctrl->cursor[c], 1ull);
        order[at] = static_cast<uint32_t>(i);
    }
}

// The CTA grid: each CTA takes the next chunk of order[0, ncta) and decodes
// it with the CTA-per-chunk decoder of its format.
struct CtaArgs {
    const void* const* src;
    const size_t* sizes;
    void* const* dst;
    const size_t* caps;
    const uint8_t* formats;
    cudec_chunk_result* results;
    const uint32_t* order;
    Ctrl* ctrl;
};

__global__ void __launch_bounds__(lzc::kThreads, lzc::kCtasPerSm) mixed_cta_kernel(CtaArgs a) {
    extern __shared__ __align__(16) uint8_t cta_smem[];
    __shared__ unsigned long long claim;
    const unsigned long long ncta = a.ctrl->ncta;
    for (;;) {
        if (threadIdx.x == 0) claim = atomicAdd(&a.ctrl->cta_counter, 1ull);
        __syncthreads();
        const unsigned long long idx = claim;
        __syncthreads();  // read by every thread before the next claim is written
        if (idx >= ncta) break;
        const uint32_t c = a.order[idx];
        const uint8_t* src = static_cast<const uint8_t*>(a.src[c]);
        uint8_t* dst = static_cast<uint8_t*>(a.dst[c]);
        uint64_t written = 0;
        int st;
        if (a.formats[c] == CUDEC_FORMAT_LZ4) {
            lzc::Chunk<lzc::Lz4F> ch{*reinterpret_cast<lzc::Shm<lzc::Lz4F>*>(cta_smem), src,
                                     a.sizes[c], dst, a.caps[c], 0};
            st = ch.run(&written);
        } else {
            lzc::Chunk<lzc::SnappyF> ch{*reinterpret_cast<lzc::Shm<lzc::SnappyF>*>(cta_smem),
                                        src, a.sizes[c], dst, a.caps[c], 0};
            st = ch.run(&written);
        }
        if (threadIdx.x == 0) {
            a.results[c].status = st;
            a.results[c].reserved = 0;
            a.results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
        __syncthreads();  // the next chunk reuses the shared state
    }
}

// Each format's path is an out-of-line call, compiled as in its own kernel:
// one decoder's register demand does not shape another's allocation.
template <class F>
__device__ __noinline__ int mixed_lz(const uint8_t* src, uint64_t S, uint8_t* dst, uint64_t cap,
                                     uint8_t* base, lzw::Tune tn, uint32_t lane,
                                     uint64_t* written) {
    return lzw::decode_chunk<F>(src, S, dst, cap, base, base + lzw::kRing, tn, lane, written);
}

__device__ __noinline__ int mixed_zstd(const uint8_t* src, uint64_t S, uint8_t* dst, uint64_t cap,
                                       uint8_t* base, uint8_t* litbuf, uint32_t lane,
                                       uint64_t* written) {
    return zstd::decode_frame(src, S, dst, cap, *reinterpret_cast<zstd::WarpSmem*>(base), litbuf,
                              lane, written);
}

__device__ __noinline__ int mixed_gdeflate(const uint8_t* src, uint64_t S, uint8_t* dst,
                                           uint64_t cap, uint8_t* base, uint32_t lane,
                                           uint64_t* written) {
    return gdf::decode_page(src, S, dst, cap, *reinterpret_cast<gdf::Tables*>(base), lane,
                            written);
}

__global__ void __launch_bounds__(kThreads, 2) mixed_kernel(Args a) {
    extern __shared__ __align__(16) uint8_t mixed_smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t* base = mixed_smem + warp * kWarpSmem;
    const size_t gw = static_cast<size_t>(blockIdx.x) * kWarps + warp;
    uint8_t* litbuf = a.zstd_slots + gw * zstd::kLitSlot;
    for (;;) {
        unsigned long long idx = 0;
        if (lane == 0) idx = *a.first + atomicAdd(a.counter, 1ull);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= a.n) break;
        const uint32_t c = a.order[idx];
        const uint8_t* src = static_cast<const uint8_t*>(a.src[c]);
        const uint64_t S = a.sizes[c], cap = a.caps[c];
        uint8_t* dst = static_cast<uint8_t*>(a.dst[c]);
        uint64_t written = 0;
        int st;
        switch (a.formats[c]) {
            case CUDEC_FORMAT_LZ4:
                st = mixed_lz<lzw::Lz4>(src, S, dst, cap, base, a.tune[size_bucket(cap)], lane,
                                        &written);
                break;
            case CUDEC_FORMAT_SNAPPY:
                st = mixed_lz<lzw::Snappy>(src, S, dst, cap, base, a.tune[size_bucket(cap)], lane,
                                           &written);
                break;
            case CUDEC_FORMAT_GDEFLATE:
                st = mixed_gdeflate(src, S, dst, cap, base, lane, &written);
                break;
            case CUDEC_FORMAT_ZSTD:
                st = mixed_zstd(src, S, dst, cap, base, litbuf, lane, &written);
                break;
            default:
                st = CUDEC_ERR_UNSUPPORTED;
                break;
        }
        __syncwarp();
        if (lane == 0) {
            a.results[c].status = st;
            a.results[c].reserved = 0;
            a.results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
    }
}

// Warps per LZ4 / Snappy chunk by bucket when the plan is created: one warp
// below 16 KiB, a whole CTA from 16 KiB up (what the tuner picks on B200
// over 100,000 uneven LZ4 + Snappy chunks, run after run: small chunks keep
// the warp grid busy beside the CTA grid, and the CTA decoder's parallel
// parse wins from 16 KiB up); Zstd and GDeflate chunks are one warp's.
constexpr uint32_t kDefaultWpc[kBuckets] = {1, 1, kCtaWarps, kCtaWarps, kCtaWarps, kCtaWarps};

struct Key {
    const void* const* src;
    const size_t* sizes;
    void* const* dst;
    const size_t* caps;
    const uint8_t* formats;
    size_t n;
    cudec_chunk_result* results;
    bool operator==(const Key& o) const {
        return src == o.src && sizes == o.sizes && dst == o.dst && caps == o.caps &&
               formats == o.formats && n == o.n && results == o.results;
    }
};

}  // namespace mixed
}  // namespace cdb

struct cudec_mixed_plan {
    int dev = -1;
    unsigned grid = 0;      // warp grid: resident CTAs x SMs
    unsigned cta_grid = 0;  // CTA grid: resident CTAs x SMs
    int sms = 0;
    cdb::DevBuf ctrl, order, slots;
    cudaStream_t s = nullptr, s2 = nullptr;  // s2: the CTA grid beside the warp grid
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, t0 = nullptr, t1 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cdb::mixed::Key key{};
    cdb::lzw::Tune tune[cdb::mixed::kBuckets];
    uint32_t wpc[cdb::mixed::kBuckets];  // warps per LZ4 / Snappy chunk: 1 or kCtaWarps

    uint32_t cta_buckets() const {
        uint32_t m = 0;
        for (int b = 0; b < cdb::mixed::kBuckets; ++b)
            if (wpc[b] > 1) m |= 1u << b;
        return m;
    }

    void drop_graph() {
        if (exec) (void)cudaGraphExecDestroy(exec);
        if (graph) (void)cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~cudec_mixed_plan() {
        if (s) (void)cudaStreamSynchronize(s);
        if (s2) (void)cudaStreamSynchronize(s2);
        drop_graph();
        for (cudaEvent_t e : {ev_in, ev_out, t0, t1, ev_fork, ev_join})
            if (e) (void)cudaEventDestroy(e);
        if (s) (void)cudaStreamDestroy(s);
        if (s2) (void)cudaStreamDestroy(s2);
    }
};

namespace {

using cdb::mixed::Args;
using cdb::mixed::Ctrl;
using cdb::mixed::Key;

cudec_status check_args(const cudec_mixed_plan* plan, const void* const* src,
                        const size_t* sizes, void* const* dst, const size_t* caps,
                        const uint8_t* formats, size_t n, const cudec_chunk_result* results) {
    if (plan == nullptr || formats == nullptr || n > 0xFFFFFFFFull)
        return CUDEC_ERR_INVALID_ARGUMENT;
    return cdb::validate_batch(src, sizes, dst, caps, n, results);
}

Args make_args(cudec_mixed_plan* p, const Key& k) {
    Args a{};
    a.src = k.src;
    a.sizes = k.sizes;
    a.dst = k.dst;
    a.caps = k.caps;
    a.formats = k.formats;
    a.n = k.n;
    a.results = k.results;
    a.order = static_cast<const uint32_t*>(p->order.p);
    a.counter = &static_cast<Ctrl*>(p->ctrl.p)->counter;
    a.first = &static_cast<Ctrl*>(p->ctrl.p)->ncta;
    a.zstd_slots = static_cast<uint8_t*>(p->slots.p);
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) a.tune[b] = p->tune[b];
    return a;
}

// The whole decode of one batch on stream s: order, then the persistent grid
// (no more CTAs than the batch has chunks for, so small batches leave SMs to
// other work on the device).
cdb::mixed::CtaArgs make_cta_args(cudec_mixed_plan* p, const Key& k) {
    return cdb::mixed::CtaArgs{k.src, k.sizes, k.dst, k.caps, k.formats, k.results,
                               static_cast<const uint32_t*>(p->order.p),
                               static_cast<Ctrl*>(p->ctrl.p)};
}

cudaError_t enqueue(cudec_mixed_plan* p, const Key& k, cudaStream_t s) {
    Ctrl* ctrl = static_cast<Ctrl*>(p->ctrl.p);
    cudaError_t e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), s);
    if (e != cudaSuccess) return e;
    const size_t want = (k.n + 255) / 256;
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>(want, 4u * p->sms));
    const uint32_t cb = p->cta_buckets();
    cdb::mixed::order_count<<<blocks, 256, 0, s>>>(k.caps, k.formats, k.n, cb, ctrl);
    cdb::mixed::order_scan<<<1, 32, 0, s>>>(ctrl);
    cdb::mixed::order_place<<<blocks, 256, 0, s>>>(k.caps, k.formats, k.n, cb, ctrl,
                                                    static_cast<uint32_t*>(p->order.p));
    if (cb) {
        // the CTA grid beside the warp grid: forked to the plan's second
        // stream after the order, joined back before the end
        e = cudaEventRecord(p->ev_fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s2, p->ev_fork, 0);
        if (e != cudaSuccess) return e;
        const unsigned cg = static_cast<unsigned>(std::min<size_t>(k.n, p->cta_grid));
        cdb::mixed::mixed_cta_kernel<<<cg, cdb::lzc::kThreads, cdb::mixed::kCtaSmem, p->s2>>>(
            make_cta_args(p, k));
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_join, p->s2);
        if (e != cudaSuccess) return e;
    }
    const size_t ctas = (k.n + cdb::mixed::kWarps - 1) / cdb::mixed::kWarps;
    const unsigned grid = static_cast<unsigned>(std::min<size_t>(ctas, p->grid));
    cdb::mixed::mixed_kernel<<<grid, cdb::mixed::kThreads, cdb::mixed::kSmem, s>>>(
        make_args(p, k));
    e = cudaGetLastError();
    if (e == cudaSuccess && cb) e = cudaStreamWaitEvent(s, p->ev_join, 0);
    return e;
}

cudec_status bind(cudec_mixed_plan* p, size_t n) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return CUDEC_ERR_CUDA;
    if (dev != p->dev) return CUDEC_ERR_INVALID_ARGUMENT;
    if (p->order.cap < n * sizeof(uint32_t)) {
        p->drop_graph();
        if (p->order.ensure(n * sizeof(uint32_t)) != cudaSuccess) return CUDEC_ERR_CUDA;
    }
    return CUDEC_OK;
}

}  // namespace

namespace cdb {

cudaError_t mixed_reserve(cudec_mixed_plan* plan, size_t max_chunks) {
    if (plan->order.cap >= max_chunks * sizeof(uint32_t)) return cudaSuccess;
    plan->drop_graph();
    return plan->order.ensure(max_chunks * sizeof(uint32_t));
}

cudaError_t mixed_launch(cudec_mixed_plan* plan, const void* const* d_src_ptrs,
                         const size_t* d_src_sizes, void* const* d_dst_ptrs,
                         const size_t* d_dst_capacities, const uint8_t* d_formats, size_t n,
                         cudec_chunk_result* d_results, cudaStream_t stream) {
    if (plan->order.cap < n * sizeof(uint32_t)) return cudaErrorInvalidValue;
    return enqueue(plan, Key{d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities, d_formats, n,
                             d_results},
                   stream);
}

}  // namespace cdb

extern "C" {

cudec_status cudec_mixed_plan_create(cudec_mixed_plan** out_plan) {
    if (out_plan == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    *out_plan = nullptr;
    (void)cudaGetLastError();
    cudec_mixed_plan* p = new (std::nothrow) cudec_mixed_plan();
    if (p == nullptr) return CUDEC_ERR_CUDA;
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) {
        p->tune[b] = cdb::lzw::kDefaultTune;
        p->wpc[b] = cdb::mixed::kDefaultWpc[b];
    }
    int per_sm = 0;
    bool ok = cudaGetDevice(&p->dev) == cudaSuccess;
    ok = ok && (p->sms = cdb::device_sm_count(p->dev)) > 0;
    ok = ok && cudaFuncSetAttribute(cdb::mixed::mixed_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(cdb::mixed::kSmem)) == cudaSuccess;
    ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cdb::mixed::mixed_kernel,
                                                             cdb::mixed::kThreads,
                                                             cdb::mixed::kSmem) == cudaSuccess;
    ok = ok && per_sm > 0;
    if (ok) p->grid = static_cast<unsigned>(p->sms * per_sm);
    int cta_per_sm = 0;
    ok = ok && cudaFuncSetAttribute(cdb::mixed::mixed_cta_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(cdb::mixed::kCtaSmem)) == cudaSuccess;
    ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &cta_per_sm, cdb::mixed::mixed_cta_kernel, cdb::lzc::kThreads,
                   cdb::mixed::kCtaSmem) == cudaSuccess;
    ok = ok && cta_per_sm > 0;
    if (cta_per_sm > cdb::mixed::kCtaPerSmMax) cta_per_sm = cdb::mixed::kCtaPerSmMax;
    if (ok) p->cta_grid = static_cast<unsigned>(p->sms * cta_per_sm);
    ok = ok && p->ctrl.ensure(sizeof(Ctrl)) == cudaSuccess;
    ok = ok && p->slots.ensure(static_cast<size_t>(p->grid) * cdb::mixed::kWarps *
                               cdb::zstd::kLitSlot) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&p->s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&p->s2, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t* e : {&p->ev_in, &p->ev_out, &p->ev_fork, &p->ev_join})
        ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
    for (cudaEvent_t* e : {&p->t0, &p->t1}) ok = ok && cudaEventCreate(e) == cudaSuccess;
    if (!ok) {
        delete p;
        (void)cudaGetLastError();
        return CUDEC_ERR_CUDA;
    }
    *out_plan = p;
    return CUDEC_OK;
}

cudec_status cudec_mixed_plan_destroy(cudec_mixed_plan* plan) {
    if (plan == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    delete plan;
    return CUDEC_OK;
}

cudec_status cudec_mixed_decompress(cudec_mixed_plan* plan, const void* const* d_src_ptrs,
                                    const size_t* d_src_sizes, void* const* d_dst_ptrs,
                                    const size_t* d_dst_capacities, const uint8_t* d_formats,
                                    size_t chunk_count, cudec_chunk_result* d_results,
                                    cudec_stream_t stream) {
    const cudec_status v = check_args(plan, d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                      d_dst_capacities, d_formats, chunk_count, d_results);
    if (v != CUDEC_OK) return v;
    (void)cudaGetLastError();
    const cudec_status b = bind(plan, chunk_count);
    if (b != CUDEC_OK) return b;
    const Key k{d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities,
                d_formats, chunk_count, d_results};
    if (plan->exec == nullptr || !(plan->key == k)) {
        plan->drop_graph();
        if (cudaStreamBeginCapture(plan->s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return CUDEC_ERR_CUDA;
        const cudaError_t ce = enqueue(plan, k, plan->s);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(plan->s, &g);
        if (ce != cudaSuccess || ee != cudaSuccess || g == nullptr) {
            if (g) (void)cudaGraphDestroy(g);
            (void)cudaGetLastError();
            return CUDEC_ERR_CUDA;
        }
        plan->graph = g;
        if (cudaGraphInstantiate(&plan->exec, g, 0) != cudaSuccess) {
            plan->drop_graph();
            (void)cudaGetLastError();
            return CUDEC_ERR_CUDA;
        }
        plan->key = k;
    }
    const cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    bool ok = cudaEventRecord(plan->ev_in, cs) == cudaSuccess;
    ok = ok && cudaStreamWaitEvent(plan->s, plan->ev_in, 0) == cudaSuccess;
    ok = ok && cudaGraphLaunch(plan->exec, plan->s) == cudaSuccess;
    ok = ok && cudaEventRecord(plan->ev_out, plan->s) == cudaSuccess;
    ok = ok && cudaStreamWaitEvent(cs, plan->ev_out, 0) == cudaSuccess;
    return ok ? CUDEC_OK : CUDEC_ERR_CUDA;
}

cudec_status cudec_mixed_plan_tune(cudec_mixed_plan* plan, const void* const* d_src_ptrs,
                                   const size_t* d_src_sizes, void* const* d_dst_ptrs,
                                   const size_t* d_dst_capacities, const uint8_t* d_formats,
                                   size_t chunk_count, cudec_chunk_result* d_results,
                                   cudec_stream_t stream) {
    const cudec_status v = check_args(plan, d_src_ptrs, d_src_sizes, d_dst_ptrs,
                                      d_dst_capacities, d_formats, chunk_count, d_results);
    if (v != CUDEC_OK) return v;
    (void)cudaGetLastError();
    const cudec_status b = bind(plan, chunk_count);
    if (b != CUDEC_OK) return b;
    const cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    if (cudaStreamSynchronize(cs) != cudaSuccess) return CUDEC_ERR_CUDA;
    std::vector<size_t> caps(chunk_count);
    std::vector<uint8_t> fmts(chunk_count);
    if (cudaMemcpy(caps.data(), d_dst_capacities, chunk_count * sizeof(size_t),
                   cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(fmts.data(), d_formats, chunk_count, cudaMemcpyDeviceToHost) != cudaSuccess)
        return CUDEC_ERR_CUDA;
    std::vector<std::vector<uint32_t>> members(cdb::mixed::kBuckets), lz(cdb::mixed::kBuckets);
    for (size_t i = 0; i < chunk_count; ++i) {
        const int bk = cdb::mixed::size_bucket(caps[i]);
        members[bk].push_back(static_cast<uint32_t>(i));
        if (fmts[i] == CUDEC_FORMAT_LZ4 || fmts[i] == CUDEC_FORMAT_SNAPPY)
            lz[bk].push_back(static_cast<uint32_t>(i));
    }
    std::vector<cdb::lzw::Tune> cands;
    for (uint32_t pw : {256u, 512u, 1024u})
        for (uint32_t ahead : {std::min(2 * pw + 64, cdb::lzw::kInAhead), cdb::lzw::kInAhead})
            for (uint32_t batch : {2048u, 4096u}) {
                const cdb::lzw::Tune t{pw, ahead, batch};
                bool dup = false;
                for (const auto& c : cands)
                    dup = dup || (c.pw == t.pw && c.ahead == t.ahead && c.batch == t.batch);
                if (!dup && cdb::lzw::tune_valid(t)) cands.push_back(t);
            }
    plan->drop_graph();
    const Key whole{d_src_ptrs, d_src_sizes, d_dst_ptrs, d_dst_capacities,
                    d_formats, chunk_count, d_results};
    Ctrl* ctrl = static_cast<Ctrl*>(plan->ctrl.p);
    constexpr size_t kCounters = 2 * sizeof(unsigned long long);  // counter, cta_counter
    // Best of two device-timed runs of `launch` on the plan's stream (after
    // resetting the work counters and publishing the CTA grid's chunk
    // count; every copy is on that stream, ordered with the launches).
    auto timed = [&](auto launch, unsigned long long ncta, float* out) -> bool {
        float ms_min = 0.f;
        for (int rep = 0; rep < 2; ++rep) {
            bool ok = cudaMemsetAsync(ctrl, 0, kCounters, plan->s) == cudaSuccess;
            const unsigned long long h_ncta = ncta;  // pageable: staged before the call returns
            ok = ok && cudaMemcpyAsync(&ctrl->ncta, &h_ncta, sizeof(h_ncta),
                                       cudaMemcpyHostToDevice, plan->s) == cudaSuccess;
            ok = ok && cudaEventRecord(plan->t0, plan->s) == cudaSuccess;
            launch();
            ok = ok && cudaGetLastError() == cudaSuccess;
            ok = ok && cudaEventRecord(plan->t1, plan->s) == cudaSuccess;
            ok = ok && cudaEventSynchronize(plan->t1) == cudaSuccess;
            float ms = 0.f;
            ok = ok && cudaEventElapsedTime(&ms, plan->t0, plan->t1) == cudaSuccess;
            if (!ok) return false;
            if (rep == 0 || ms < ms_min) ms_min = ms;
        }
        *out = ms_min;
        return true;
    };
    for (int bk = 0; bk < cdb::mixed::kBuckets; ++bk) {
        const std::vector<uint32_t>& m = members[bk];
        if (m.empty()) continue;
        if (cudaMemcpyAsync(plan->order.p, m.data(), m.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, plan->s) != cudaSuccess)
            return CUDEC_ERR_CUDA;
        // one warp per chunk: the fastest shape over the bucket's chunks
        float best = 0.f;
        cdb::lzw::Tune best_t = plan->tune[bk];
        for (const auto& t : cands) {
            Args a = make_args(plan, whole);
            a.n = m.size();
            for (int q = 0; q < cdb::mixed::kBuckets; ++q) a.tune[q] = t;
            float ms = 0.f;
            if (!timed([&] {
                    cdb::mixed::mixed_kernel<<<plan->grid, cdb::mixed::kThreads,
                                               cdb::mixed::kSmem, plan->s>>>(a);
                }, 0, &ms)) {
                (void)cudaGetLastError();
                return CUDEC_ERR_CUDA;
            }
            if (best == 0.f || ms < best) {
                best = ms;
                best_t = t;
            }
        }
        plan->tune[bk] = best_t;
        // warps per LZ4 / Snappy chunk: that shape against a whole CTA per
        // chunk, on the bucket's LZ4 and Snappy chunks
        const std::vector<uint32_t>& l = lz[bk];
        if (l.empty()) continue;
        if (cudaMemcpyAsync(plan->order.p, l.data(), l.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, plan->s) != cudaSuccess)
            return CUDEC_ERR_CUDA;
        Args a = make_args(plan, whole);
        a.n = l.size();
        for (int q = 0; q < cdb::mixed::kBuckets; ++q) a.tune[q] = best_t;
        float warp_ms = 0.f, cta_ms = 0.f;
        const unsigned cg = static_cast<unsigned>(std::min<size_t>(l.size(), plan->cta_grid));
        const bool ok =
            timed([&] {
                cdb::mixed::mixed_kernel<<<plan->grid, cdb::mixed::kThreads, cdb::mixed::kSmem,
                                           plan->s>>>(a);
            }, 0, &warp_ms) &&
            timed([&] {
                cdb::mixed::mixed_cta_kernel<<<cg, cdb::lzc::kThreads, cdb::mixed::kCtaSmem,
                                               plan->s>>>(make_cta_args(plan, whole));
            }, l.size(), &cta_ms);
        if (!ok) {
            (void)cudaGetLastError();
            return CUDEC_ERR_CUDA;
        }
        plan->wpc[bk] = cta_ms < warp_ms ? cdb::mixed::kCtaWarps : 1u;
    }
    return cudaStreamSynchronize(plan->s) == cudaSuccess ? CUDEC_OK : CUDEC_ERR_CUDA;
}

cudec_status cudec_mixed_plan_get_tuning(const cudec_mixed_plan* plan, uint32_t* out_params) {
    if (plan == nullptr || out_params == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) {
        out_params[3 * b] = plan->tune[b].pw;
        out_params[3 * b + 1] = plan->tune[b].ahead;
        out_params[3 * b + 2] = plan->tune[b].batch;
    }
    return CUDEC_OK;
}

cudec_status cudec_mixed_plan_get_shape(const cudec_mixed_plan* plan, uint32_t* out_shape) {
    if (plan == nullptr || out_shape == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) {
        out_shape[4 * b] = plan->wpc[b];
        out_shape[4 * b + 1] = plan->tune[b].pw;
        out_shape[4 * b + 2] = plan->tune[b].ahead;
        out_shape[4 * b + 3] = plan->tune[b].batch;
    }
    return CUDEC_OK;
}

cudec_status cudec_mixed_plan_set_shape(cudec_mixed_plan* plan, const uint32_t* shape) {
    if (plan == nullptr || shape == nullptr) return CUDEC_ERR_INVALID_ARGUMENT;
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) {
        const cdb::lzw::Tune t{shape[4 * b + 1], shape[4 * b + 2], shape[4 * b + 3]};
        if ((shape[4 * b] != 1 && shape[4 * b] != cdb::mixed::kCtaWarps) ||
            !cdb::lzw::tune_valid(t))
            return CUDEC_ERR_INVALID_ARGUMENT;
    }
    for (int b = 0; b < cdb::mixed::kBuckets; ++b) {
        plan->wpc[b] = shape[4 * b];
        plan->tune[b] = cdb::lzw::Tune{shape[4 * b + 1], shape[4 * b + 2], shape[4 * b + 3]};
    }
    plan->drop_graph();  // the graph holds the old shape
    return CUDEC_OK;
}

}  // extern "C"
