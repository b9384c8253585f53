// The block-per-chunk LZ decode kernel for LZ4 and raw Snappy (sm_100a).
//
// One CTA of kThreads decodes one chunk at a time and walks its chunks with a
// grid stride (two CTAs per SM overlap their phases). A chunk is processed in
// input windows of kInWin bytes:
//
//  1. stage   — cp.async.bulk copies the window (plus a halo) of compressed
//               bytes from HBM into shared memory, 16-byte aligned, while the
//               threads clear the token bitmap.
//  2. chains  — every thread runs the format's `step` from the start of its
//               kSegLen-byte segment ("speculative token chains") and marks
//               the positions it visits in a bitmap (one register word at a
//               time). A chain started at a wrong position merges with the
//               true token chain after a few steps.
//  3. resolve — every segment takes the previous segment's exit as its true
//               entry and follows the true chain from there until it lands on
//               one of its own chain's marks (merge) or leaves the segment; a
//               second parallel round redoes this from the previous
//               segment's corrected exit. One warp then walks the segments
//               with the true entry (skipping consistent runs by ballot),
//               following serially only where both guesses were wrong. The
//               bitmap is then rewritten to hold exactly the true tokens.
//  4. batches — tokens are taken kBatch at a time in order (two per thread):
//               fields, a block scan for output positions, and the full
//               reject ladder per sequence. The first failing (or terminal)
//               sequence decides the chunk's status exactly as the serial
//               decoder would; only sequences before it are executed.
//  5. execute — output is produced in sub-tiles of kSub bytes, one 16-byte
//               vector per thread. A scatter pass records which sequence
//               covers each vector's first byte. Phase A: each thread walks
//               the pieces (literal runs, match runs) of its vector and
//               copies them 4 bytes at a time with funnel shifts from the
//               staged input, the output ring or HBM. A vector with a match
//               source inside the sub-tile (or a period shorter than the
//               piece) is finished in phase B: rounds in which every byte
//               whose immediate source is final is produced, with per-vector
//               "final" masks double-buffered across rounds. Bytes go to a
//               shared-memory ring of the last kRing output bytes; finished
//               sub-tiles are flushed to HBM with aligned 16-byte stores and
//               older match sources are read back from HBM.
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
constexpr uint32_t kInWin = 40960;
constexpr uint32_t kInHalo = 1024;
constexpr uint32_t kInBuf = kInWin + kInHalo + 32;
constexpr int kSegs = kThreads;
constexpr uint32_t kSegLen = kInWin / kSegs;       // 160 bytes
constexpr uint32_t kBmWords = kInWin / 32;         // 1280
constexpr uint32_t kWordsPerThread = kBmWords / kThreads;  // 5
constexpr uint32_t kRing = 32768;
constexpr uint32_t kSub = kThreads * 16;           // 4096 output bytes
constexpr int kPerThread = 2;
constexpr int kBatch = kThreads * kPerThread;      // 512 sequences
constexpr uint32_t kNoEvent = 0xffffffffu;
constexpr uint32_t kRingWords = kRing / 4;

static_assert(kSegLen % 32 == 0, "segments own whole bitmap words");
static_assert(kBmWords % kThreads == 0, "bitmap words split evenly");
static_assert((kRing & (kRing - 1)) == 0 && kRing >= 4 * kSub, "ring size");

struct __align__(16) LzSmem {
    uint8_t ring[kRing];
    uint8_t in[kInBuf];
    uint32_t bm[kBmWords];
    uint64_t s_out[kBatch + 1];
    uint64_t s_lsrc[kBatch];
    uint64_t s_llen[kBatch];
    uint32_t s_off[kBatch];
    uint32_t s_pos[kBatch];
    uint64_t seg_exit[kSegs];     // speculative chain exits
    uint64_t seg_guess[kSegs];    // entry guess (previous speculative exit)
    uint64_t seg_out[kSegs];      // exit under that guess
    uint64_t seg_alt_out[kSegs];  // exit under the corrected guess (round 1)
    uint64_t seg_true[kSegs];     // true entry, from the warp walk
    uint16_t vec_seq[kSub / 16];  // sequence covering each vector's first byte
    uint8_t vec_done[2][kSub / 16];   // vector complete, by round parity
    uint64_t scan64[kWarps + 1];
    uint32_t scan32[kWarps + 1];
    uint64_t bc[8];
    uint32_t event;
    int32_t event_status;
    uint32_t event_done;
    uint64_t mbar;
};

constexpr size_t kLzSmemBytes = sizeof(LzSmem);
static_assert(kLzSmemBytes <= 115712, "two CTAs per SM must fit");

// Optional per-phase cycle accounting (compile with -DCDB_PHASE_TIMING):
// thread 0 of every CTA adds the clock cycles it spent in each phase to
// cdb_phase_cycles[] (0 stage, 1 chains, 2 resolve, 3 batch build, 4 execute,
// 5 whole chunk, 6 execute round 0, 7 later execute rounds). Off by default;
// costs nothing when off.
#ifdef CDB_PHASE_TIMING
__device__ unsigned long long cdb_phase_cycles[8];
#define CDB_T0(v) long long v = clock64()
#define CDB_ACC(i, v)                                                        \
    do {                                                                     \
        if (threadIdx.x == 0) {                                              \
            long long now_ = clock64();                                      \
            atomicAdd(&cdb_phase_cycles[i], (unsigned long long)(now_ - v)); \
            v = now_;                                                        \
        }                                                                    \
    } while (0)
#else
#define CDB_T0(v)
#define CDB_ACC(i, v) do { } while (0)
#endif

// Optional event counters (compile with -DCDB_EVENT_COUNTS): 0 execute rounds,
// 1 segments that did not merge, 2 HBM reads of old match sources, 3 chase
// steps, 4 sub-tiles, 5 produced bytes, 6 ring word reads, 7 vectors built
// byte by byte. Off by default.
#ifdef CDB_EVENT_COUNTS
__device__ unsigned long long cdb_event_counts[8];
#define CDB_COUNT(i, n) atomicAdd(&cdb_event_counts[i], (unsigned long long)(n))
#else
#define CDB_COUNT(i, n) do { } while (0)
#endif

__device__ __forceinline__ bool bm_test(const uint32_t* bm, uint64_t r) {
    return (bm[r >> 5] >> (r & 31)) & 1u;
}

// Clear bitmap bits [a, b) (window-relative); words owned by the caller.
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

// Segment outcome for an entry guess `a`: follow the true chain from `a`
// until it lands on a bit of this segment's speculative chain (merge) or
// leaves the segment. Returns the exit under that entry; *merge is the merge
// position (or `se` when none).
template <class Fmt>
__device__ __forceinline__ uint64_t follow_segment(const InView& in, uint64_t S,
                                                   const uint32_t* bm, uint64_t W0,
                                                   uint64_t se, uint64_t a,
                                                   uint64_t spec_exit,
                                                   uint64_t* merge) {
    if (a >= se) {
        *merge = se;
        return a;
    }
    uint64_t p = a;
    while (p < se && !bm_test(bm, p - W0)) p = Fmt::step(in, S, p);
    if (p < se) {
        *merge = p;
        return spec_exit;
    }
    *merge = se;
    return p;
}

template <class Fmt>
struct LzChunk {
    LzSmem& sm;
    InView in;
    uint64_t S, limit;
    uint8_t* gdst;
    uint32_t mis;       // gdst & 15: v-space position = x + mis
    uint64_t flush_v;   // first unflushed v (vector aligned)

    // Final output byte x from the ring or, when older than the ring's
    // intact range, from HBM where it was flushed.
    __device__ __forceinline__ uint32_t out_at(uint64_t x, int64_t ring_lo_v) const {
        const uint64_t v = x + mis;
        if (static_cast<int64_t>(v) >= ring_lo_v) return sm.ring[v & (kRing - 1)];
        CDB_COUNT(2, 1);
        return *(reinterpret_cast<volatile const uint8_t*>(gdst) + x);
    }

    // Four bytes starting at byte q of a word-addressed source, low byte first
    // (bytes past the wanted ones are whatever follows them).
    __device__ __forceinline__ static uint32_t funnel(uint32_t lo, uint32_t hi,
                                                      uint32_t q) {
        return __funnelshift_r(lo, hi, 8 * (q & 3));
    }
    __device__ __forceinline__ uint32_t ring4(uint64_t v) const {
        const uint32_t* rw = reinterpret_cast<const uint32_t*>(sm.ring);
        const uint32_t w = static_cast<uint32_t>(v >> 2);
        return funnel(rw[w & (kRingWords - 1)], rw[(w + 1) & (kRingWords - 1)],
                      static_cast<uint32_t>(v));
    }
    // Four bytes at global byte address a; only the aligned words holding the
    // `n` wanted bytes are read, so nothing outside them is touched.
    __device__ __forceinline__ static uint32_t global4(const uint8_t* a, uint32_t n,
                                                       bool stable) {
        const uintptr_t ad = reinterpret_cast<uintptr_t>(a);
        const uint32_t* w = reinterpret_cast<const uint32_t*>(ad & ~uintptr_t(3));
        const uint32_t lo = stable ? __ldg(w) : *reinterpret_cast<const volatile uint32_t*>(w);
        uint32_t hi = 0;
        if ((ad & 3) + n > 4) hi = stable ? __ldg(w + 1) : *reinterpret_cast<const volatile uint32_t*>(w + 1);
        return funnel(lo, hi, static_cast<uint32_t>(ad));
    }
    // Four input bytes at position q (n of them wanted).
    __device__ __forceinline__ uint32_t input4(uint64_t q, uint32_t n) const {
        const uint64_t r = q - in.lo;
        if (r < in.len && r + n <= in.len) {
            const uintptr_t a = reinterpret_cast<uintptr_t>(in.sm + r);
            const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
            const uint32_t hi = ((a & 3) + n > 4) ? w[1] : 0u;
            return funnel(w[0], hi, static_cast<uint32_t>(a));
        }
        return global4(in.g + q, n, true);
    }

    // Merge the bytes [j0, j1) of vector word k (bytes 4k..4k+3) from `val`,
    // whose low byte is vector byte max(4k, j0).
    __device__ __forceinline__ static void merge_word(uint32_t& w, uint32_t k,
                                                      uint32_t j0, uint32_t j1,
                                                      uint32_t val) {
        const uint32_t b0 = j0 > 4 * k ? j0 - 4 * k : 0;
        const uint32_t b1 = j1 < 4 * k + 4 ? j1 - 4 * k : 4;
        const uint32_t n = b1 - b0;
        const uint32_t m = (n >= 4 ? 0xffffffffu : ((1u << (8 * n)) - 1u)) << (8 * b0);
        w = (w & ~m) | ((val << (8 * b0)) & m);
    }

    // Byte at output position q for the byte path (periods shorter than a
    // vector): from this thread's own registers when q lies in its vector,
    // else from the ring/HBM when final. Returns false when not final yet.
    __device__ __forceinline__ bool byte_src(uint64_t q, uint64_t vx, uint64_t ready,
                                             uint64_t vb, int64_t ring_lo_v,
                                             const uint8_t* done, uint32_t w0,
                                             uint32_t w1, uint32_t w2, uint32_t w3,
                                             uint32_t* b) const {
        if (q - vx < 16) {  // modular: vx wraps below zero for the first vector
            const uint32_t sj = static_cast<uint32_t>(q - vx);
            const uint32_t ws = sj < 4 ? w0 : sj < 8 ? w1 : sj < 12 ? w2 : w3;
            *b = (ws >> ((sj & 3) * 8)) & 0xffu;
            return true;
        }
        if (q < ready) {
            *b = out_at(q, ring_lo_v);
            return true;
        }
        if (!done[(q + mis - vb) >> 4]) return false;
        *b = sm.ring[(q + mis) & (kRing - 1)];
        return true;
    }

    // Produce output [o0, o1) for sequences 0..n-1 of the batch table
    // (s_out[n] == o1).
    __device__ void execute(uint64_t o0, uint64_t o1, uint32_t n) {
        if (o1 <= o0) return;
        const uint32_t tid = threadIdx.x;
        const uint64_t v_lo = (o0 + mis) & ~15ull;
        const uint64_t v_hi = (o1 + mis + 15) & ~15ull;
        const uint64_t v_done = (o1 + mis) & ~15ull;  // vectors below are complete
        for (uint64_t vb = v_lo; vb < v_hi; vb += kSub) {
            const uint64_t vend = vb + kSub < v_hi ? vb + kSub : v_hi;
            // Map: the sequence covering the first byte (>= o0) of each vector.
            for (uint32_t k = 0; k < kPerThread; ++k) {
                const uint32_t s = tid * kPerThread + k;
                if (s < n) {
                    const uint64_t a = sm.s_out[s] + mis, b = sm.s_out[s + 1] + mis;
                    uint64_t f = s == 0 ? v_lo : ((a + 15) & ~15ull);
                    if (f < vb) f = vb;
                    const uint64_t e = b < vend ? b : vend;
                    for (; f < e; f += 16) sm.vec_seq[(f - vb) >> 4] = static_cast<uint16_t>(s);
                }
            }
            sm.vec_done[0][tid] = 0;
            __syncthreads();
            CDB_T0(tex);
            const int64_t ring_lo_v = static_cast<int64_t>(vb) + kSub - kRing;
            if (tid == 0) CDB_COUNT(4, 1);
            const uint64_t sub_x0 = vb >= mis ? vb - mis : 0;
            const uint64_t ready = sub_x0 > o0 ? sub_x0 : o0;
            const uint64_t v = vb + 16ull * tid;
            const bool mine = v < vend;
            // Bytes [jlo, jhi) of this vector belong to [o0, o1).
            uint32_t jlo = 0, jhi = 16;
            uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
            uint32_t s = 0;
            uint64_t base = 0, nxt = 0;
            if (mine) {
                if (v < o0 + mis) jlo = static_cast<uint32_t>(o0 + mis - v);
                if (v + 16 > o1 + mis) jhi = static_cast<uint32_t>(o1 + mis - v);
                if (jlo > 0 || jhi < 16) {
                    const uint4 cur = *reinterpret_cast<const uint4*>(&sm.ring[v & (kRing - 1)]);
                    w0 = cur.x; w1 = cur.y; w2 = cur.z; w3 = cur.w;
                }
                s = sm.vec_seq[tid];
                base = sm.s_out[s];
                nxt = sm.s_out[s + 1];
            }
            const uint64_t vx = v - mis;          // output position of vector byte 0
            const uint64_t jend_x = v + jhi - mis;
            uint32_t j = jlo;                     // next byte to produce
            // Rounds: round 0 takes only sources below `ready` (and literals);
            // later rounds also take sources in vectors completed in the
            // previous round. A thread resumes at its first unproduced byte.
            for (uint32_t round = 0; round <= kSub; ++round) {
                const uint8_t* done = sm.vec_done[round & 1];
                bool stalled = false;
                while (mine && j < jhi) {
                    const uint64_t x = vx + j;
                    while (x >= nxt) {
                        ++s;
                        base = nxt;
                        nxt = sm.s_out[s + 1];
                    }
                    const uint64_t ll = sm.s_llen[s];
                    const uint64_t rel = x - base;
                    uint32_t j1;
                    if (rel < ll) {
                        const uint64_t pend = base + ll < jend_x ? base + ll : jend_x;
                        j1 = static_cast<uint32_t>(pend - vx);
                        const uint64_t P = sm.s_lsrc[s] + rel;
#pragma unroll
                        for (uint32_t k = 0; k < 4; ++k) {
                            if (4 * k + 4 <= j || 4 * k >= j1) continue;
                            const uint32_t b0 = j > 4 * k ? j : 4 * k;
                            const uint32_t e1 = j1 < 4 * k + 4 ? j1 : 4 * k + 4;
                            const uint32_t val = input4(P + (b0 - j), e1 - b0);
                            if (k == 0) merge_word(w0, 0, j, j1, val);
                            else if (k == 1) merge_word(w1, 1, j, j1, val);
                            else if (k == 2) merge_word(w2, 2, j, j1, val);
                            else merge_word(w3, 3, j, j1, val);
                        }
                        j = j1;
                        continue;
                    }
                    const uint32_t off = sm.s_off[s];
                    const uint64_t r = rel - ll;
                    const uint64_t md = base + ll;
                    const uint64_t ph = r < off ? r : r % off;   // position in period
                    uint64_t pend = nxt < jend_x ? nxt : jend_x;
                    if (off < 16) {
                        // short period: byte path
                        uint64_t q = md - off + ph;
                        bool ok = true;
                        uint32_t jj = j;
                        const uint32_t jstop = static_cast<uint32_t>(pend - vx);
                        for (; jj < jstop; ++jj) {
                            uint32_t b;
                            if (!byte_src(q, vx, ready, vb, ring_lo_v, done, w0, w1, w2, w3, &b)) {
                                ok = false;
                                break;
                            }
                            const uint32_t sh = (jj & 3) * 8;
                            const uint32_t m = ~(0xffu << sh);
                            if (jj < 4) w0 = (w0 & m) | (b << sh);
                            else if (jj < 8) w1 = (w1 & m) | (b << sh);
                            else if (jj < 12) w2 = (w2 & m) | (b << sh);
                            else w3 = (w3 & m) | (b << sh);
                            if (++q == md) q = md - off;
                        }
                        j = jj;
                        if (!ok) { stalled = true; break; }
                        continue;
                    }
                    // contiguous sub-piece up to the period boundary
                    if (pend - x > off - ph) pend = x + (off - ph);
                    j1 = static_cast<uint32_t>(pend - vx);
                    const uint64_t P = md - off + ph;
                    const uint64_t len = pend - x;
                    bool in_ring;
                    if (P + len <= ready) {
                        const int64_t pv = static_cast<int64_t>(P + mis);
                        if (pv >= ring_lo_v) {
                            in_ring = true;
                        } else if (pv + static_cast<int64_t>(len) <= ring_lo_v) {
                            in_ring = false;
                        } else {
                            // straddles the ring's oldest byte: per byte, all final
                            for (uint32_t jj = j; jj < j1; ++jj) {
                                const uint32_t b = out_at(P + (jj - j), ring_lo_v);
                                const uint32_t sh = (jj & 3) * 8;
                                const uint32_t m = ~(0xffu << sh);
                                if (jj < 4) w0 = (w0 & m) | (b << sh);
                                else if (jj < 8) w1 = (w1 & m) | (b << sh);
                                else if (jj < 12) w2 = (w2 & m) | (b << sh);
                                else w3 = (w3 & m) | (b << sh);
                            }
                            j = j1;
                            continue;
                        }
                    } else {
                        // source inside this sub-tile: its vectors must be complete
                        const uint64_t a = P < ready ? ready : P;
                        const uint32_t va = static_cast<uint32_t>((a + mis - vb) >> 4);
                        const uint32_t vz = static_cast<uint32_t>((P + len - 1 + mis - vb) >> 4);
                        if (!done[va] || !done[vz]) { stalled = true; break; }
                        in_ring = true;
                    }
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k) {
                        if (4 * k + 4 <= j || 4 * k >= j1) continue;
                        const uint32_t b0 = j > 4 * k ? j : 4 * k;
                        const uint32_t e1 = j1 < 4 * k + 4 ? j1 : 4 * k + 4;
                        const uint64_t q = P + (b0 - j);
                        uint32_t val;
                        if (in_ring) { CDB_COUNT(6, 1); val = ring4(q + mis); }
                        else { CDB_COUNT(2, 1); val = global4(gdst + q, e1 - b0, false); }
                        if (k == 0) merge_word(w0, 0, j, j1, val);
                        else if (k == 1) merge_word(w1, 1, j, j1, val);
                        else if (k == 2) merge_word(w2, 2, j, j1, val);
                        else merge_word(w3, 3, j, j1, val);
                    }
                    j = j1;
                }
                const bool finished_now = mine && !stalled && j >= jhi;
                if (finished_now && j != 0xffffffffu) {
                    *reinterpret_cast<uint4*>(&sm.ring[v & (kRing - 1)]) = make_uint4(w0, w1, w2, w3);
                    j = 0xffffffffu;  // written
                }
                if (mine) sm.vec_done[(round + 1) & 1][tid] = j == 0xffffffffu ? 1 : 0;
                if (stalled) CDB_COUNT(3, 1);
                if (tid == 0) CDB_COUNT(0, 1);
                const bool more = __syncthreads_or(stalled);
                if (round == 0) CDB_ACC(6, tex); else CDB_ACC(7, tex);
                if (!more) break;
            }
            // Flush this thread's vector if it is complete and not yet out.
            if (mine && v >= flush_v && v + 16 <= v_done) {
                const uint4 val = *reinterpret_cast<const uint4*>(&sm.ring[v & (kRing - 1)]);
                if (v >= mis) {
                    *reinterpret_cast<uint4*>(gdst - mis + v) = val;
                } else {
                    const uint32_t w[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
                    for (uint32_t jj = 0; jj < 16; ++jj)
                        if (jj >= mis - static_cast<uint32_t>(v))
                            gdst[v + jj - mis] = static_cast<uint8_t>(w[jj >> 2] >> ((jj & 3) * 8));
                }
            }
            __syncthreads();
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
        LzChunk<Fmt> c{sm, {}, 0, 0, nullptr, 0, 0};
        const uint8_t* gsrc = reinterpret_cast<const uint8_t*>(sm.bc[0]);
        c.S = sm.bc[1];
        c.gdst = reinterpret_cast<uint8_t*>(sm.bc[2]);
        c.limit = sm.bc[5];
        c.mis = static_cast<uint32_t>(sm.bc[2] & 15);
        c.flush_v = 0;
        c.in.g = gsrc;
        int status = static_cast<int>(sm.bc[6]);
        uint64_t E = sm.bc[4];   // true position of the next token
        uint64_t O = 0;          // output produced so far
        bool finished = status != CUDEC_OK;
        __syncthreads();  // everyone has read bc
        CDB_T0(tchunk);

        while (!finished) {
            if (E >= c.S) {
                status = Fmt::finish(E == c.S, O, c.limit);
                finished = true;
                break;
            }
            // ---- 1. stage the window -------------------------------------
            CDB_T0(tph);
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
            CDB_ACC(0, tph);

            // ---- 2. speculative chains -------------------------------------
            const uint64_t ss = W0 + static_cast<uint64_t>(tid) * kSegLen;
            const uint64_t se = (tid < nseg) ? ((Wend - ss > kSegLen) ? ss + kSegLen : Wend) : ss;
            {
                uint64_t pos = ss;
                uint32_t cur_w = 0xffffffffu, acc = 0;
                while (pos < se) {
                    const uint64_t r = pos - W0;
                    const uint32_t w = static_cast<uint32_t>(r >> 5);
                    if (w != cur_w) {
                        if (cur_w != 0xffffffffu) sm.bm[cur_w] = acc;
                        cur_w = w;
                        acc = 0;
                    }
                    acc |= 1u << (r & 31);
                    pos = Fmt::step(c.in, c.S, pos);
                }
                if (cur_w != 0xffffffffu) sm.bm[cur_w] = acc;
                sm.seg_exit[tid] = pos;
            }
            __syncthreads();
            CDB_ACC(1, tph);

            // ---- 3. resolve ------------------------------------------------
            // Round 0: every segment assumes the previous speculative exit is
            // its true entry and follows the true chain from it to a merge.
            const uint64_t guess = tid == 0 ? W0 : sm.seg_exit[tid - 1];
            uint64_t merge = se, merge1 = se;
            if (tid < nseg) {
                sm.seg_guess[tid] = guess;
                sm.seg_out[tid] = follow_segment<Fmt>(c.in, c.S, sm.bm, W0, se, guess,
                                                     sm.seg_exit[tid], &merge);
            }
            __syncthreads();
            // Round 1: where the previous segment's round-0 exit differs from
            // this guess, redo the follow from that exit.
            const uint64_t alt = tid == 0 ? W0 : sm.seg_out[tid - 1];
            if (tid < nseg) {
                uint64_t ao = sm.seg_out[tid];
                merge1 = merge;
                if (alt != guess)
                    ao = follow_segment<Fmt>(c.in, c.S, sm.bm, W0, se, alt,
                                             sm.seg_exit[tid], &merge1);
                sm.seg_alt_out[tid] = ao;
            }
            __syncthreads();
            // One warp walks the segments with the true entry, skipping runs
            // whose guesses chain consistently; an entry matching neither
            // round is repaired by following the true chain (all lanes
            // redundantly, so the walk stays converged).
            if (tid < 32) {
                const uint32_t lane = tid;
                uint64_t E = W0;
                for (uint32_t g0 = 0; g0 < nseg; g0 += 32) {
                    const uint32_t k = g0 + lane;
                    const bool valid = k < nseg;
                    const uint64_t gk = valid ? sm.seg_guess[k] : 0;
                    const uint64_t ok_out = valid ? sm.seg_out[k] : 0;
                    const uint64_t ak = valid ? (k == 0 ? W0 : sm.seg_out[k - 1]) : 0;
                    const uint64_t ak_out = valid ? sm.seg_alt_out[k] : 0;
                    const uint64_t ssk = W0 + static_cast<uint64_t>(k) * kSegLen;
                    const uint64_t sek = valid ? ((Wend - ssk > kSegLen) ? ssk + kSegLen : Wend) : 0;
                    const uint64_t prev_out = __shfl_up_sync(0xffffffffu, ok_out, 1);
                    const bool cons = valid && lane > 0 && gk == prev_out && gk < sek;
                    const uint32_t cons_mask = __ballot_sync(0xffffffffu, cons);
                    uint64_t te = 0;
                    uint32_t l = 0;
                    while (l < 32 && g0 + l < nseg) {
                        const uint64_t gl = __shfl_sync(0xffffffffu, gk, l);
                        const uint64_t sel = __shfl_sync(0xffffffffu, sek, l);
                        const uint64_t al = __shfl_sync(0xffffffffu, ak, l);
                        const uint64_t alo = __shfl_sync(0xffffffffu, ak_out, l);
                        if (lane == l) te = E;
                        if (E >= sel) {
                            ++l;
                            continue;
                        }
                        if (E == gl) {
                            // lanes after l whose guess chains from l are right
                            const uint32_t rest = ~cons_mask & (0xfffffffeu << l);
                            const uint32_t nb = rest ? __ffs(rest) - 1 : 32;
                            if (lane > l && lane < nb) te = gk;
                            E = __shfl_sync(0xffffffffu, ok_out, nb - 1);
                            l = nb;
                            continue;
                        }
                        if (E == al) {
                            E = alo;
                        } else {
                            uint64_t mdummy;
                            E = follow_segment<Fmt>(c.in, c.S, sm.bm, W0, sel, E,
                                                    sm.seg_exit[g0 + l], &mdummy);
                        }
                        ++l;
                    }
                    if (valid) sm.seg_true[k] = te;
                }
                if (lane == 0) sm.bc[7] = E;
            }
            __syncthreads();
            // Rewrite this segment's bits: drop speculative marks before the
            // merge point, add the true chain from the true entry up to it.
            if (tid < nseg) {
                const uint64_t te = sm.seg_true[tid];
                if (te == alt && alt != guess)
                    merge = merge1;
                else if (te != guess)
                    follow_segment<Fmt>(c.in, c.S, sm.bm, W0, se, te, 0, &merge);
                const uint64_t stop = merge < se ? merge : se;
                // (reads of other segments' bits are finished: barrier above)
                bm_clear_range(sm.bm, ss - W0, stop - W0);
                for (uint64_t q = te; q < stop; q = Fmt::step(c.in, c.S, q)) {
                    const uint64_t r = q - W0;
                    sm.bm[r >> 5] |= 1u << (r & 31);
                }
            }
            const uint64_t Wexit = sm.bc[7];
            __syncthreads();
            CDB_ACC(2, tph);

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
                Seq q[kPerThread];
                uint64_t p[kPerThread];
                uint64_t mine = 0;
#pragma unroll
                for (int k = 0; k < kPerThread; ++k) {
                    const uint32_t j = tid * kPerThread + k;
                    q[k] = Seq{0, 0, 0, 1};
                    p[k] = 0;
                    if (j < nb) {
                        p[k] = W0 + sm.s_pos[j];
                        Fmt::fields(c.in, c.S, p[k], &q[k]);
                        mine += q[k].lit_len + q[k].match_len;
                    }
                }
                uint64_t btotal = 0;
                uint64_t d = O + block_exclusive_scan<uint64_t, kThreads>(mine, sm.scan64, &btotal);
                int my_st = CUDEC_OK;
                bool my_done = false;
                uint32_t my_ev = kNoEvent;
#pragma unroll
                for (int k = 0; k < kPerThread; ++k) {
                    const uint32_t j = tid * kPerThread + k;
                    if (j < nb) {
                        if (my_ev == kNoEvent && !Fmt::fast_ok(q[k], c.limit, d)) {
                            bool done = false;
                            const int st = Fmt::check(c.in, c.S, c.limit, p[k], d, &done);
                            if (st != CUDEC_OK || done) {
                                my_ev = j;
                                my_st = st;
                                my_done = done;
                            }
                        }
                        sm.s_out[j] = d;
                        sm.s_lsrc[j] = q[k].lit_src;
                        sm.s_llen[j] = q[k].lit_len;
                        sm.s_off[j] = q[k].off;
                        d += q[k].lit_len + q[k].match_len;
                    }
                }
                if (my_ev != kNoEvent) atomicMin(&sm.event, my_ev);
                __syncthreads();
                // The first event (lowest index) decides the chunk.
                const uint32_t ev = sm.event;
                if (ev != kNoEvent && my_ev == ev) {
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
                __syncthreads();
                if (tid == 0) sm.s_out[nexec] = o1;
                __syncthreads();
                CDB_ACC(3, tph);
                c.execute(O, o1, nexec);
                if (tid == 0) CDB_COUNT(5, o1 - O);
                O = o1;
                __syncthreads();
                CDB_ACC(4, tph);
            }
            if (!finished) E = Wexit;
        }
        if (aborted) break;
        CDB_ACC(5, tchunk);
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
