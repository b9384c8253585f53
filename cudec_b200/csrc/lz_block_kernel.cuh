// The block-per-chunk LZ decode kernel for LZ4 and raw Snappy (sm_100a).
//
// One CTA of kThreads decodes one chunk at a time and walks its chunks with a
// grid stride. A chunk is processed in input windows of kInWin bytes:
//
//  1. stage   — cp.async.bulk copies the window (plus a halo) of compressed
//               bytes from HBM into shared memory, 16-byte aligned.
//  2. chains  — kSegs threads each run the format's `step` from the start of
//               their kSegLen-byte segment ("speculative token chains") and
//               mark the positions they visit in a bitmap. A chain started at
//               a wrong position merges with the true token chain within a
//               few steps, so almost every segment's marks are the true
//               tokens from its entry point on.
//  3. resolve — for each segment, test whether the true chain's entry (the
//               previous segment's exit) is on the segment's chain; one
//               thread repairs the rare segments where it is not by walking
//               the true chain until it merges. The bitmap then holds exactly
//               the true token positions of the window.
//  4. batches — tokens are taken kBatch at a time in order: each thread
//               decodes one token's fields, a block scan gives every
//               sequence its output position, and each thread runs the full
//               reject ladder for its own sequence. The first failing (or
//               terminal) sequence decides the chunk's status exactly as the
//               serial decoder would.
//  5. execute — output is produced in sub-tiles of kSub bytes, one 16-byte
//               vector per thread, byte-parallel: each output byte finds its
//               sequence by binary search and reads its literal byte or its
//               match source. A match source inside the sub-tile being built
//               is resolved by following it back to a literal or to an
//               already-written byte. Bytes go to a shared-memory ring that
//               holds the last kRing output bytes (the LZ4 match window), and
//               each finished sub-tile is flushed to HBM with aligned 16-byte
//               stores; older match sources are read back from HBM.
//
// Nothing is written past a chunk's capacity: only sequences that passed the
// ladder are executed. Only a successful chunk reports bytes_written; a failed
// chunk's destination is unspecified (it may hold a validated prefix).
// Every loop is bounded by the input or output size; the one wait (the bulk
// copy's mbarrier) is bounded and reports CUDEC_ERR_CUDA on timeout.
#pragma once

#include <cstdint>

#include "cudec.h"
#include "device_util.cuh"
#include "lz_formats.cuh"

namespace cdb {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kInWin = 32768;
constexpr uint32_t kInHalo = 256;
constexpr uint32_t kInBuf = kInWin + kInHalo + 32;
constexpr int kSegs = 64;
constexpr uint32_t kSegLen = kInWin / kSegs;
constexpr uint32_t kBmWords = kInWin / 32;
constexpr uint32_t kWordsPerThread = kBmWords / kThreads;
constexpr uint32_t kRing = 65536;
constexpr uint32_t kSub = kThreads * 16;
constexpr int kBatch = kThreads;
constexpr uint32_t kNoEvent = 0xffffffffu;

static_assert(kSegLen % 32 == 0, "segments own whole bitmap words");
static_assert(kBmWords % kThreads == 0, "bitmap words split evenly");
static_assert((kRing & (kRing - 1)) == 0 && kRing >= 4 * kSub, "ring size");

enum : uint32_t { kModeChain = 0, kModeNone = 1, kModeFixed = 2 };

struct __align__(16) LzSmem {
    uint8_t ring[kRing];
    uint8_t in[kInBuf];
    uint32_t bm[kBmWords];
    uint64_t s_out[kBatch + 1];
    uint64_t s_lsrc[kBatch];
    uint64_t s_llen[kBatch];
    uint32_t s_off[kBatch];
    uint32_t s_pos[kBatch];
    uint64_t seg_exit[kSegs];
    uint64_t seg_entry[kSegs];
    uint32_t seg_mode[kSegs];
    uint32_t tok_prefix[kThreads];
    uint64_t scan64[kWarps + 1];
    uint32_t scan32[kWarps + 1];
    uint64_t bc[8];
    uint32_t fail_mask[2];
    uint32_t event;
    int32_t event_status;
    uint32_t event_done;
    uint64_t mbar;
};

constexpr size_t kLzSmemBytes = sizeof(LzSmem);
static_assert(kLzSmemBytes <= 115712, "two CTAs per SM must fit");

__device__ __forceinline__ bool bm_test(const uint32_t* bm, uint64_t r) {
    return (bm[r >> 5] >> (r & 31)) & 1u;
}

// Clear bitmap bits [a, b) (window-relative) — words wholly owned by caller.
__device__ __forceinline__ void bm_clear_range(uint32_t* bm, uint64_t a,
                                               uint64_t b) {
    while (a < b) {
        const uint32_t w = static_cast<uint32_t>(a >> 5), lo = a & 31;
        const uint64_t wend = (static_cast<uint64_t>(w) + 1) << 5;
        const uint64_t e = b < wend ? b : wend;
        const uint32_t n = static_cast<uint32_t>(e - a);
        const uint32_t mask = (n == 32 ? 0xffffffffu : ((1u << n) - 1u)) << lo;
        bm[w] &= ~mask;
        a = e;
    }
}

template <class Fmt>
struct LzChunk {
    LzSmem& sm;
    InView in;
    uint64_t S, cap, limit;
    uint8_t* gdst;
    uint32_t mis;       // gdst & 15: v-space position = x + mis
    uint64_t flush_v;   // first unflushed v (vector aligned)

    // Output byte x (< ready) from the ring or, when older than the ring's
    // intact range, from HBM where it was flushed.
    __device__ __forceinline__ uint32_t out_at(uint64_t x, int64_t ring_lo_v) const {
        const uint64_t v = x + mis;
        if (static_cast<int64_t>(v) >= ring_lo_v) return sm.ring[v & (kRing - 1)];
        return *(reinterpret_cast<volatile const uint8_t*>(gdst) + x);
    }

    // Index s with s_out[s] <= x < s_out[s + 1], searching [lo, hi).
    __device__ __forceinline__ uint32_t find_seq(uint64_t x, uint32_t lo,
                                                 uint32_t hi) const {
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.s_out[mid] <= x) lo = mid; else hi = mid;
        }
        return lo;
    }

    // Resolve output byte x in sequence s; `ready` is the first position not
    // yet written (sources below it are final).
    __device__ uint32_t resolve(uint64_t x, uint32_t s, uint64_t ready,
                                int64_t ring_lo_v) const {
        for (;;) {
            const uint64_t base = sm.s_out[s];
            const uint64_t rel = x - base;
            const uint64_t ll = sm.s_llen[s];
            if (rel < ll) return in.at(sm.s_lsrc[s] + rel);
            const uint64_t r = rel - ll;
            const uint32_t off = sm.s_off[s];
            const uint64_t src = base + ll - off + (r < off ? r : r % off);
            if (src < ready) return out_at(src, ring_lo_v);
            x = src;  // strictly smaller: follow it back within this sub-tile
            s = find_seq(x, 0, s + 1);
        }
    }

    // Produce output [o0, o1) for sequences 0..n-1 of the batch table.
    __device__ void execute(uint64_t o0, uint64_t o1, uint32_t n) {
        if (o1 <= o0) return;
        const uint64_t v_lo = (o0 + mis) & ~15ull;
        const uint64_t v_hi = (o1 + mis + 15) & ~15ull;
        const uint64_t v_done = (o1 + mis) & ~15ull;  // vectors below are complete
        for (uint64_t vb = v_lo; vb < v_hi; vb += kSub) {
            const int64_t ring_lo_v = static_cast<int64_t>(vb) + kSub - kRing;
            const uint64_t v = vb + 16ull * threadIdx.x;
            // Everything below `ready` is final: earlier batches and earlier
            // sub-tiles of this batch.
            const uint64_t sub_x0 = vb >= mis ? vb - mis : 0;
            const uint64_t ready = sub_x0 > o0 ? sub_x0 : o0;
            if (v < v_hi) {
                uint4 cur = *reinterpret_cast<const uint4*>(&sm.ring[v & (kRing - 1)]);
                uint32_t w[4] = {cur.x, cur.y, cur.z, cur.w};
                uint32_t s = 0xffffffffu;
#pragma unroll 1
                for (uint32_t j = 0; j < 16; ++j) {
                    const uint64_t vv = v + j;
                    if (vv < mis) continue;
                    const uint64_t x = vv - mis;
                    if (x < o0 || x >= o1) continue;
                    if (s == 0xffffffffu) s = find_seq(x, 0, n);
                    while (s + 1 < n && sm.s_out[s + 1] <= x) ++s;
                    const uint32_t b = resolve(x, s, ready, ring_lo_v);
                    const uint32_t sh = (j & 3) * 8;
                    w[j >> 2] = (w[j >> 2] & ~(0xffu << sh)) | (b << sh);
                }
                *reinterpret_cast<uint4*>(&sm.ring[v & (kRing - 1)]) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
            __syncthreads();
            // Flush this thread's vector if it is complete and not yet out.
            if (v < v_hi && v >= flush_v && v + 16 <= v_done) {
                const uint4 val = *reinterpret_cast<const uint4*>(&sm.ring[v & (kRing - 1)]);
                if (v >= mis) {
                    *reinterpret_cast<uint4*>(gdst - mis + v) = val;
                } else {
                    const uint32_t w[4] = {val.x, val.y, val.z, val.w};
                    for (uint32_t j = mis - static_cast<uint32_t>(v); j < 16; ++j)
                        gdst[v + j - mis] = static_cast<uint8_t>(w[j >> 2] >> ((j & 3) * 8));
                }
            }
        }
        if (v_done > flush_v) flush_v = v_done;
    }

    // Final partial vector of a successful chunk: bytes [flush_v - mis, end).
    __device__ void flush_tail(uint64_t end) {
        const uint64_t v_end = end + mis;
        if (threadIdx.x < 16) {
            const uint64_t v = flush_v + threadIdx.x;
            if (v < v_end && v >= mis) gdst[v - mis] = sm.ring[v & (kRing - 1)];
        }
    }
};

template <class Fmt>
__global__ void __launch_bounds__(kThreads, 2)
    lz_decode_kernel(const void* const* src_ptrs, const size_t* src_sizes,
                     void* const* dst_ptrs, const size_t* dst_caps,
                     size_t chunk_count, cudec_chunk_result* results) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    LzSmem& sm = *reinterpret_cast<LzSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    if (tid == 0) mbar_init(&sm.mbar, 1);
    __syncthreads();
    uint32_t phase = 0;
    bool aborted = false;  // uniform: decided by __syncthreads_or
    size_t chunk = blockIdx.x;

    for (; chunk < chunk_count; chunk += gridDim.x) {
        if (tid == 0) {
            sm.bc[0] = reinterpret_cast<uint64_t>(src_ptrs[chunk]);
            sm.bc[1] = src_sizes[chunk];
            sm.bc[2] = reinterpret_cast<uint64_t>(dst_ptrs[chunk]);
            sm.bc[3] = dst_caps[chunk];
            uint64_t first = 0, limit = 0;
            int st = Fmt::begin(reinterpret_cast<const uint8_t*>(sm.bc[0]),
                                sm.bc[1], sm.bc[3], &first, &limit);
            sm.bc[4] = first;
            sm.bc[5] = limit;
            sm.bc[6] = static_cast<uint64_t>(st);
        }
        __syncthreads();
        LzChunk<Fmt> c{sm, {}, 0, 0, 0, nullptr, 0, 0};
        const uint8_t* gsrc = reinterpret_cast<const uint8_t*>(sm.bc[0]);
        c.S = sm.bc[1];
        c.gdst = reinterpret_cast<uint8_t*>(sm.bc[2]);
        c.cap = sm.bc[3];
        c.limit = sm.bc[5];
        c.mis = static_cast<uint32_t>(sm.bc[2] & 15);
        c.flush_v = 0;
        c.in.g = gsrc;
        int status = static_cast<int>(sm.bc[6]);
        uint64_t E = sm.bc[4];   // true position of the next token
        uint64_t O = 0;          // output produced so far
        bool finished = status != CUDEC_OK;
        __syncthreads();  // everyone has read bc

        while (!finished) {
            if (E >= c.S) {
                status = Fmt::finish(E == c.S, O, c.limit);
                finished = true;
                break;
            }
            // ---- 1. stage the window -------------------------------------
            const uint64_t W0 = E;
            const uint64_t Wend = (c.S - W0 > kInWin) ? W0 + kInWin : c.S;
            const uint64_t Lend = (c.S - W0 > kInWin + kInHalo) ? W0 + kInWin + kInHalo : c.S;
            const uint64_t a0 = reinterpret_cast<uint64_t>(gsrc + W0) & ~15ull;
            const uint64_t a1 = (reinterpret_cast<uint64_t>(gsrc + Lend) + 15) & ~15ull;
            if (tid == 0) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&sm.mbar, static_cast<uint32_t>(a1 - a0));
                bulk_g2s(sm.in, reinterpret_cast<const void*>(a0),
                         static_cast<uint32_t>(a1 - a0), &sm.mbar);
            }
            for (uint32_t w = tid; w < kBmWords; w += kThreads) sm.bm[w] = 0;
            const bool ok = mbar_wait_bounded(&sm.mbar, phase);
            phase ^= 1;
            if (__syncthreads_or(!ok)) {
                status = CUDEC_ERR_CUDA;
                finished = true;
                aborted = true;
                break;
            }
            c.in.sm = sm.in + (reinterpret_cast<uint64_t>(gsrc + W0) - a0);
            c.in.lo = W0;
            c.in.len = Lend - W0;
            const uint32_t nseg = static_cast<uint32_t>((Wend - W0 + kSegLen - 1) / kSegLen);

            // ---- 2. speculative chains -------------------------------------
            if (tid < static_cast<uint32_t>(kSegs)) {
                const uint64_t ss = W0 + static_cast<uint64_t>(tid) * kSegLen;
                uint64_t pos = ss;
                if (tid < nseg) {
                    const uint64_t se = (Wend - ss > kSegLen) ? ss + kSegLen : Wend;
                    while (pos < se) {
                        const uint64_t r = pos - W0;
                        sm.bm[r >> 5] |= 1u << (r & 31);
                        pos = Fmt::step(c.in, c.S, pos);
                    }
                }
                sm.seg_exit[tid] = pos;
            }
            __syncthreads();
            // ---- 3. resolve -----------------------------------------------
            if (tid < static_cast<uint32_t>(kSegs)) {
                bool fail = false;
                if (tid > 0 && tid < nseg) {
                    const uint64_t ss = W0 + static_cast<uint64_t>(tid) * kSegLen;
                    const uint64_t se = (Wend - ss > kSegLen) ? ss + kSegLen : Wend;
                    const uint64_t e = sm.seg_exit[tid - 1];
                    fail = !(e >= ss && e < se && bm_test(sm.bm, e - W0));
                }
                sm.seg_entry[tid] = tid == 0 ? W0 : sm.seg_exit[tid - 1];
                sm.seg_mode[tid] = kModeChain;
                const uint32_t m = __ballot_sync(0xffffffffu, fail);
                if ((tid & 31) == 0) sm.fail_mask[tid >> 5] = m;
            }
            __syncthreads();
            if (tid == 0) {
                uint64_t fail = sm.fail_mask[0] | (static_cast<uint64_t>(sm.fail_mask[1]) << 32);
                uint64_t Eo;
                if (fail == 0) {
                    Eo = sm.seg_exit[nseg - 1];
                } else {
                    uint32_t k = __ffsll(static_cast<long long>(fail)) - 1;
                    uint64_t e = sm.seg_exit[k - 1];
                    while (k < nseg) {
                        const uint64_t ss = W0 + static_cast<uint64_t>(k) * kSegLen;
                        const uint64_t se = (Wend - ss > kSegLen) ? ss + kSegLen : Wend;
                        bool merged;
                        if (e >= se) {
                            sm.seg_mode[k] = kModeNone;
                            bm_clear_range(sm.bm, ss - W0, se - W0);
                            ++k;
                            continue;
                        }
                        if (bm_test(sm.bm, e - W0)) {
                            sm.seg_entry[k] = e;
                            sm.seg_mode[k] = kModeChain;
                            merged = true;
                        } else {
                            uint64_t pos = e;
                            while (pos < se && !bm_test(sm.bm, pos - W0))
                                pos = Fmt::step(c.in, c.S, pos);
                            const uint64_t stop = pos < se ? pos : se;
                            bm_clear_range(sm.bm, ss - W0, stop - W0);
                            for (uint64_t q = e; q < stop; q = Fmt::step(c.in, c.S, q)) {
                                const uint64_t r = q - W0;
                                sm.bm[r >> 5] |= 1u << (r & 31);
                            }
                            sm.seg_entry[k] = e;
                            sm.seg_mode[k] = kModeFixed;
                            merged = pos < se;
                            if (!merged) {
                                e = pos;
                                ++k;
                                continue;
                            }
                        }
                        // Merged: the segment's own exit is the true exit.
                        e = sm.seg_exit[k];
                        ++k;
                        const uint64_t rest = k < 64 ? (fail >> k) : 0;
                        if (rest == 0) {
                            e = sm.seg_exit[nseg - 1];
                            k = nseg;
                        } else {
                            const uint32_t k2 = k + __ffsll(static_cast<long long>(rest)) - 1;
                            if (k2 > k) e = sm.seg_exit[k2 - 1];
                            k = k2;
                        }
                    }
                    Eo = e;
                }
                sm.bc[7] = Eo;
            }
            __syncthreads();
            if (tid < nseg && sm.seg_mode[tid] == kModeChain) {
                const uint64_t ss = W0 + static_cast<uint64_t>(tid) * kSegLen;
                const uint64_t en = sm.seg_entry[tid];
                bm_clear_range(sm.bm, 0 + (ss - W0), en - W0);
            }
            __syncthreads();
            const uint64_t Wexit = sm.bc[7];

            // ---- 4/5. batches of true tokens -------------------------------
            uint32_t cnt = 0;
#pragma unroll
            for (uint32_t k = 0; k < kWordsPerThread; ++k)
                cnt += __popc(sm.bm[tid * kWordsPerThread + k]);
            uint32_t total = 0;
            const uint32_t pre = block_exclusive_scan<uint32_t, kThreads>(cnt, sm.scan32, &total);
            for (uint32_t b0 = 0; b0 < total && !finished; b0 += kBatch) {
                const uint32_t nb = total - b0 < static_cast<uint32_t>(kBatch) ? total - b0 : kBatch;
                if (pre < b0 + kBatch && pre + cnt > b0) {
                    uint32_t idx = pre;
                    for (uint32_t k = 0; k < kWordsPerThread && idx < b0 + kBatch; ++k) {
                        const uint32_t wi = tid * kWordsPerThread + k;
                        uint32_t word = sm.bm[wi];
                        while (word && idx < b0 + kBatch) {
                            const uint32_t bit = __ffs(word) - 1;
                            word &= word - 1;
                            if (idx >= b0) sm.s_pos[idx - b0] = wi * 32 + bit;
                            ++idx;
                        }
                    }
                }
                if (tid == 0) sm.event = kNoEvent;
                __syncthreads();
                Seq q{0, 0, 0, 1};
                uint64_t p = 0;
                int my_st = CUDEC_OK;
                bool my_done = false;
                if (tid < nb) {
                    p = W0 + sm.s_pos[tid];
                    Fmt::fields(c.in, c.S, p, &q);
                }
                const uint64_t len = tid < nb ? q.lit_len + q.match_len : 0;
                uint64_t btotal = 0;
                const uint64_t opre = block_exclusive_scan<uint64_t, kThreads>(len, sm.scan64, &btotal);
                const uint64_t d = O + opre;
                if (tid < nb) {
                    my_st = Fmt::check(c.in, c.S, c.limit, p, d, &my_done);
                    if (my_st != CUDEC_OK || my_done) atomicMin(&sm.event, tid);
                    sm.s_out[tid] = d;
                    sm.s_lsrc[tid] = q.lit_src;
                    sm.s_llen[tid] = q.lit_len;
                    sm.s_off[tid] = q.off;
                }
                __syncthreads();
                // The first event (lowest index) decides the chunk.
                const uint32_t ev = sm.event;
                if (ev != kNoEvent && tid == ev) {
                    sm.event_status = my_st;
                    sm.event_done = my_done ? 1u : 0u;
                }
                __syncthreads();
                uint32_t nexec = nb;
                if (ev != kNoEvent) {
                    const bool ok_done = sm.event_status == CUDEC_OK && sm.event_done;
                    nexec = ok_done ? ev + 1 : ev;
                    status = sm.event_status;
                    finished = true;
                }
                // End of the executed range: for an OK terminal run it is the
                // literal end; otherwise the next sequence's start.
                uint64_t o1;
                if (nexec == 0) {
                    o1 = O;
                } else if (ev != kNoEvent && nexec == ev + 1) {
                    o1 = sm.s_out[ev] + sm.s_llen[ev];
                } else if (nexec < nb) {
                    o1 = sm.s_out[nexec];
                } else {
                    o1 = O + btotal;
                }
                if (tid == 0) sm.s_out[nexec] = o1;
                __syncthreads();
                c.execute(O, o1, nexec);
                O = o1;
                __syncthreads();
            }
            if (!finished) E = Wexit;
        }
        if (aborted) break;
        if (status == CUDEC_OK) c.flush_tail(O);
        if (tid == 0) {
            results[chunk].status = status;
            results[chunk].reserved = 0;
            results[chunk].bytes_written = status == CUDEC_OK ? O : 0;
        }
        __syncthreads();
    }
    if (aborted) {
        // A staging copy never completed: report the chunk in flight and every
        // chunk this CTA still owned as a CUDA failure, not stale records.
        for (; chunk < chunk_count; chunk += gridDim.x) {
            if (tid == 0) {
                results[chunk].status = CUDEC_ERR_CUDA;
                results[chunk].reserved = 0;
                results[chunk].bytes_written = 0;
            }
        }
    }
}

}  // namespace cdb
