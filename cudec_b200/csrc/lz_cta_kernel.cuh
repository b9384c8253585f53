// CTA-per-chunk decoder for the byte-oriented LZ formats (LZ4 block, raw
// Snappy): the chunk's token chain is found in parallel by the whole CTA,
// and the tokens execute one per thread.
//
// A chunk is decoded tile by tile. A tile is the kTile input positions that
// start at a known token (the chunk's first, then each tile's exit). For a
// tile, with kThreads threads:
//
//   1. stage: the tile's input bytes (plus kLook bytes past it) land in
//      shared memory by cp.async, in aligned 16-byte blocks;
//   2. segment exits: thread t owns the kSeg positions of segment t and,
//      walking them backwards, computes for every position p the exit of
//      the chain that starts at p: the first chain position at or past the
//      segment's end (the format's step, its length extensions capped at
//      kExtCap bytes; a position the cap stops is "unknown");
//   3. candidate chase: warp w owns super-segment w (kSupSegs segments) and
//      lane k follows the chain from the super-segment's k-th position
//      through its segments by their exits, recording where it enters each
//      segment; the true entry into a super-segment lies within its first
//      kCand positions unless a token straddles its start by more;
//   4. tile chase: one thread follows the true chain through the tile's
//      super-segments, picking the lane whose start is the true entry (an
//      unknown exit, or an entry past the candidates, is resolved by
//      walking that super-segment exactly);
//   5. count: each thread walks its segment from its true entry (exact
//      steps), counting tokens and output bytes; a block scan gives every
//      token its index and output offset;
//   6. check: each thread walks its segment again and runs the format's
//      exact ladder (lz_ladder.cuh) on each token at its output offset; the
//      first failing or terminal token (a block-wide minimum) decides the
//      chunk exactly as the serial parser would, since the steps equal the
//      ladder's next position for every token the ladder accepts;
//   7. execute, in groups of consecutive tokens whose output fits kGroupOut:
//      the group's literal runs are copied into an output ring in shared
//      memory (indexed by destination address mod kRing, so ring blocks and
//      destination blocks share alignment), then its matches as data flow:
//      each thread copies each of its matches once none of the bytes its
//      source reads is the output of a match still pending in the group (a
//      bit per output byte), and clears the match's own bits after its bytes
//      land; the lowest pending match is always ready, so the group always
//      makes progress.
//      Completed aligned 16-byte blocks leave the ring as coalesced stores.
//      A token longer than kBig is copied by the whole CTA straight to the
//      destination. Sources older than the ring are read back from the
//      destination.
//
// Every phase is per-thread code between CTA barriers, driven through an
// executor: on the device each phase runs once per thread followed by
// __syncthreads(); the host executor runs the phases for every thread in
// turn, which emulates the CTA exactly (no phase reads what another thread
// writes in the same phase, except through atomics whose order does not
// change the result). The host emulation is what the CPU tests run.
//
// Statuses follow the reference ladders exactly: LZ4 iderex/cudec
// src/lz4_block.h:95-258, Snappy src/snappy_block.h:172-435.
#pragma once

#include <cstdint>
#include <cstring>

#include "cudec.h"
#include "lz_ladder.cuh"

namespace cdb {
namespace lzc {

constexpr uint32_t kThreads = 256;                 // threads per CTA
constexpr uint32_t kCtasPerSm = 4;                 // resident CTAs per SM the registers allow
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kSeg = 16;                      // positions per segment (one per thread)
constexpr uint32_t kTile = kThreads * kSeg;        // positions per tile
constexpr uint32_t kSupSegs = 32;                  // segments per super-segment (a warp)
constexpr uint32_t kSupers = kThreads / kSupSegs;  // super-segments per tile
constexpr uint32_t kSupPos = kSupSegs * kSeg;
constexpr uint32_t kCand = 32;                     // candidate entries per super-segment
constexpr uint32_t kLook = 512;                    // staged bytes past the tile
constexpr uint32_t kInBytes = kTile + kLook + 32;  // staged input (aligned blocks)
constexpr uint32_t kExIdx = kTile + kTile / 16;    // exits, one pad word per 16
constexpr uint32_t kRing = 16384;                  // output ring (bytes)
constexpr uint32_t kGroupOut = 4096;               // output bytes per execution group
constexpr uint32_t kPerThread = 2;                 // tokens per thread per group
constexpr uint32_t kGroupTok = kThreads * kPerThread;
constexpr uint32_t kBig = 256;                     // longer tokens: whole-CTA copies
constexpr uint32_t kExtCap = 16;                   // extension bytes a segment step reads
constexpr uint32_t kSpinCap = 1u << 22;            // passes a thread makes over its matches

static_assert(kSupers == kWarps, "one super-segment per warp");
static_assert(kGroupOut + 32 <= kRing, "a group and its clear margin fit the ring");
static_assert(kInBytes % 16 == 0, "staging in 16-byte blocks");

// Exit codes of the segment walk (relative positions otherwise).
constexpr uint32_t kUnknown = 0xFFFFFFFFu;  // a step the cap stopped: resolve exactly
constexpr uint32_t kEndMark = 0xFFFFFFFEu;  // the chain ends inside this segment
constexpr uint32_t kFarRel = 0xFFFFFFF0u;   // relative positions at or above: unknown

// Step results (absolute positions otherwise).
constexpr uint64_t kStepUnknown = ~0ull;
constexpr uint64_t kStepEnd = ~0ull - 1;
constexpr uint32_t kSlowRel = 0xFFFFFFFFu;  // a fast step declines: the generic step decides

// Entry codes of the candidate chase (offsets into a segment otherwise).
constexpr uint8_t kNoEntry = 0xFF;   // no chain token starts in the segment
constexpr uint8_t kCodeUnk = 0xFE;   // the chain became unknown before the segment
constexpr uint8_t kCodeEnd = 0xFD;   // the chain ended before the segment
constexpr uint8_t kChoseOvr = 0xFC;  // super-segment resolved by an exact walk

// The tile's first event (first failing or terminal token).
constexpr uint8_t kEvNone = 0;
constexpr uint8_t kEvDone = 1;  // terminal token accepted: the chunk ends after it
constexpr uint8_t kEvFail = 2;  // rejected: ev_status holds the status

// ---------------------------------------------------------------------------
// Portable primitives (device: the real thing; host: the sequential
// emulation's plain operations).
#if defined(__CUDA_ARCH__)
#define LZC_LDG(p) __ldg(p)
__device__ __forceinline__ void at_or(uint32_t* a, uint32_t v) { atomicOr(a, v); }
__device__ __forceinline__ void at_and(uint32_t* a, uint32_t v) { atomicAnd(a, v); }
__device__ __forceinline__ void at_min(uint32_t* a, uint32_t v) { atomicMin(a, v); }
#else
#define LZC_LDG(p) (*(p))
inline void at_or(uint32_t* a, uint32_t v) { *a |= v; }
inline void at_and(uint32_t* a, uint32_t v) { *a &= v; }
inline void at_min(uint32_t* a, uint32_t v) {
    if (v < *a) *a = v;
}
#endif

// Profiling builds (-DCDB_PHASE_TIMING) accumulate, from thread 0 of every
// CTA, the SM cycles of each phase and event counts over a launch. Cycles:
// 0 stage, 1 segment exits, 2 candidate chase, 3 tile chase, 4 count and
// scan, 5 check, 6 group clear and literals, 7 match rounds, 8 flush,
// 9 whole-CTA tokens, 10 group cut. Events: 0 tiles, 1 tokens, 2 rounds,
// 3 groups, 4 whole-CTA tokens, 5 exact walks.
#if defined(CDB_PHASE_TIMING) && defined(__CUDACC__)
__device__ unsigned long long lzc_cycles[16];
__device__ unsigned long long lzc_events[16];
#endif
#if defined(CDB_PHASE_TIMING) && defined(__CUDA_ARCH__)
#define LZC_PHASE(i)                                                                    \
    do {                                                                                \
        if (threadIdx.x == 0) {                                                         \
            const long long n_ = clock64();                                             \
            atomicAdd(&lzc_cycles[i], static_cast<unsigned long long>(n_ - tl));        \
            tl = n_;                                                                    \
        }                                                                               \
    } while (0)
#define LZC_EVENT(i, n)                                                                 \
    do {                                                                                \
        if (threadIdx.x == 0) atomicAdd(&lzc_events[i], static_cast<unsigned long long>(n)); \
    } while (0)
#define LZC_START() tl = clock64()
#else
#define LZC_PHASE(i) \
    do {             \
    } while (0)
#define LZC_EVENT(i, n) \
    do {                \
    } while (0)
#define LZC_START() \
    do {            \
    } while (0)
#endif

CDB_HD uint32_t fsr(uint32_t lo, uint32_t hi, uint32_t sh) {  // funnel shift right, sh < 32
    return sh ? (lo >> sh) | (hi << (32 - sh)) : lo;
}
CDB_HD uint32_t fsl(uint32_t lo, uint32_t hi, uint32_t sh) {  // (hi:lo) << sh, high word
    return sh ? (hi << sh) | (lo >> (32 - sh)) : hi;
}
CDB_HD uint32_t keep_low(uint32_t w, uint32_t bits) {  // low `bits` (0..32) bits of w
    return bits >= 32 ? w : (w & ((1u << bits) - 1u));
}

struct V16 {
    uint32_t w[4];
};

// ---------------------------------------------------------------------------
// Phases. each(fn): fn(tid) for every thread of the CTA, then a barrier (on
// the host: every thread in turn). each_or: the same, and whether any call
// returned true. The host forms emulate the CTA sequentially.
template <class Fn>
CDB_HD void each(Fn fn) {
#if defined(__CUDA_ARCH__)
    fn(threadIdx.x);
    __syncthreads();
#else
    for (uint32_t t = 0; t < kThreads; ++t) fn(t);
#endif
}

template <class Fn>
CDB_HD bool each_or(Fn fn) {
#if defined(__CUDA_ARCH__)
    return __syncthreads_or(fn(threadIdx.x)) != 0;
#else
    bool any = false;
    for (uint32_t t = 0; t < kThreads; ++t) any = fn(t) || any;
    return any;
#endif
}

// 16 bytes global -> shared (an aligned block); completed by land().
CDB_HD void copy16_async(uint8_t* d, const uint8_t* src) {
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(d))),
                 "l"(src)
                 : "memory");
#else
    std::memcpy(d, src, 16);
#endif
}
CDB_HD void land_async() {
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
#endif
}
CDB_HD void st16(uint8_t* d, const uint8_t* src) {  // both 16-byte aligned
#if defined(__CUDA_ARCH__)
    *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(src);
#else
    std::memcpy(d, src, 16);
#endif
}
CDB_HD void zero16(uint8_t* p) {  // 16-byte aligned
#if defined(__CUDA_ARCH__)
    *reinterpret_cast<uint4*>(p) = make_uint4(0, 0, 0, 0);
#else
    std::memset(p, 0, 16);
#endif
}

// The first m (1..16) bytes of v at global address p.
CDB_HD void put_global(uint8_t* p, const V16& v, uint32_t m) {
#if defined(__CUDA_ARCH__)
    if (m == 16 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        *reinterpret_cast<uint4*>(p) = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
        return;
    }
    for (uint32_t j = 0; j < m; ++j) p[j] = static_cast<uint8_t>(v.w[j >> 2] >> (8 * (j & 3)));
#else
    std::memcpy(p, v.w, m);
#endif
}

// ---------------------------------------------------------------------------
// Formats: the exact ladder plus the segment step.

// LZ4: next = the ladder's next position for every token it accepts as
// non-terminal; kStepEnd when the token can have no successor (the ladder
// then answers terminal or reject); kStepUnknown when an extension run is
// longer than `cap` bytes (cap 0: no limit).
struct Lz4F : lzl::Lz4Ladder {
    static constexpr uint32_t kMaxTok = kTile / 3 + 3;  // tokens with a successor span >= 3 bytes
    static constexpr bool kSnappy = false;

    template <class R>
    CDB_HD static uint64_t step(const R& in, uint64_t S, uint64_t P, uint32_t cap,
                                uint64_t* olen) {
        if (P >= S) return kStepEnd;
        const uint32_t tok = in.at(P);
        uint64_t q = P + 1;
        uint64_t lit = tok >> 4;
        uint32_t b;
        if (lit == 15) {
            uint32_t k = 0;
            do {
                if (q >= S) return kStepEnd;
                if (cap && k++ == cap) return kStepUnknown;
                b = in.at(q++);
                lit += b;
            } while (b == 255);
        }
        *olen = lit;
        if (lit > S - q || S - q - lit < kSrcSlack) return kStepEnd;
        q += lit + 2;
        uint64_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15) {
            uint32_t k = 0;
            do {
                if (q >= S) return kStepEnd;
                if (cap && k++ == cap) return kStepUnknown;
                b = in.at(q++);
                ml += b;
            } while (b == 255);
        }
        *olen = lit + ml;
        return q;
    }
    // Position of the literal run of the token at P with lit literal bytes.
    template <class R>
    CDB_HD static uint64_t lit_src(const R&, uint64_t P, uint64_t lit) {
        return P + 1 + (lit >= 15 ? (lit - 15) / 255 + 1 : 0);
    }

    // Fast forms over the staged bytes, for a token whose header (with at
    // most kExtCap extension bytes per length) lies well inside them and well
    // before the chunk's end: b[r] is the token, lim = min(staged bytes, S)
    // relative to b. kSlowRel: the generic forms decide.
    static constexpr uint32_t kMargin = 2 * kExtCap + 2 + kSrcSlack;
    CDB_HD static uint32_t ext_rel(const uint8_t* b, uint32_t* q, uint32_t* len) {
        for (uint32_t k = 0; k < kExtCap; ++k) {
            const uint32_t x = b[(*q)++];
            *len += x;
            if (x != 255) return 1;
        }
        return 0;
    }
    CDB_HD static uint32_t step_rel(const uint8_t* b, uint32_t r, uint32_t lim,
                                    uint32_t* olen) {
        if (r + kMargin > lim) return kSlowRel;
        const uint32_t tok = b[r];
        uint32_t q = r + 1, lit = tok >> 4;
        if (lit == 15 && !ext_rel(b, &q, &lit)) return kSlowRel;
        q += lit;
        if (q + 2 + kExtCap + kSrcSlack > lim) return kSlowRel;
        q += 2;
        uint32_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15 && !ext_rel(b, &q, &ml)) return kSlowRel;
        *olen = lit + ml;
        return q;
    }
    // The ladder's answer for such a token when it accepts it as
    // non-terminal: the ladder's conditions (src/lz4_block.h:139-258) on its
    // final lengths (the extension loops' running checks only fail when the
    // final values fail them); false: the full ladder decides.
    CDB_HD static bool accept_rel(const uint8_t* b, uint32_t r, uint32_t lim, uint64_t P,
                                  uint64_t d, uint64_t cap, lzl::Seq* sq) {
        if (r + kMargin > lim || cap < d) return false;
        const uint32_t tok = b[r];
        uint32_t q = r + 1, lit = tok >> 4;
        if (lit == 15 && !ext_rel(b, &q, &lit)) return false;
        const uint32_t ls = q;
        q += lit;  // the offset's position
        if (q + 2 + kExtCap + kSrcSlack > lim) return false;
        const uint32_t off = b[q] | (static_cast<uint32_t>(b[q + 1]) << 8);
        q += 2;
        uint32_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15 && !ext_rel(b, &q, &ml)) return false;
        const uint64_t room = cap - d;
        if (lit > room || room - lit < kMfLimit || off == 0 || off > d + lit ||
            ml + kLastLiterals > room - lit)
            return false;
        sq->lit_src = P + (ls - r);
        sq->lit = lit;
        sq->ml = ml;
        sq->off = off;
        sq->next = P + (q - r);
        sq->done = false;
        return true;
    }
};

// Raw Snappy: one element per step; an element that ends at S steps to S
// (the chunk's end: Snappy's finish decides there).
struct SnappyF : lzl::SnappyLadder {
    static constexpr uint32_t kMaxTok = kTile / 2 + 3;  // elements span >= 2 bytes
    static constexpr bool kSnappy = true;

    template <class R>
    CDB_HD static uint64_t step(const R& in, uint64_t S, uint64_t P, uint32_t,
                                uint64_t* olen) {
        if (P >= S) return kStepEnd;
        const uint32_t tag = in.at(P);
        const uint32_t kind = tag & 3;
        if (kind == 0) {
            const uint32_t l6 = tag >> 2;
            uint64_t hdr = 1, n = l6;
            if (l6 >= 60) {
                const uint32_t extra = l6 - 59;
                if (extra > S - P - 1) return kStepEnd;
                n = 0;
                for (uint32_t i = 0; i < extra; ++i)
                    n |= static_cast<uint64_t>(in.at(P + 1 + i)) << (8 * i);
                hdr += extra;
            }
            n += 1;
            const uint64_t q = P + hdr;
            *olen = n;
            if (n > S - q) return kStepEnd;
            return q + n;
        }
        const uint64_t hdr = kind == 1 ? 2 : (kind == 2 ? 3 : 5);
        *olen = kind == 1 ? 4 + ((tag >> 2) & 7) : (tag >> 2) + 1;
        if (hdr > S - P) return kStepEnd;
        return P + hdr;
    }
    template <class R>
    CDB_HD static uint64_t lit_src(const R& in, uint64_t P, uint64_t) {
        const uint32_t tag = in.at(P);
        const uint32_t l6 = tag >> 2;
        return P + 1 + (l6 >= 60 ? l6 - 59 : 0);
    }

    // Fast forms over the staged bytes (see Lz4F): elements whose length
    // is in the tag; copies with 1- or 2-byte offsets.
    CDB_HD static uint32_t step_rel(const uint8_t* b, uint32_t r, uint32_t lim,
                                    uint32_t* olen) {
        const uint32_t tag = b[r];
        const uint32_t kind = tag & 3, l6 = tag >> 2;
        uint32_t nx;
        if (kind == 0) {
            if (l6 >= 60) return kSlowRel;
            nx = r + 2 + l6;
            *olen = l6 + 1;
        } else if (kind == 3) {
            return kSlowRel;
        } else {
            nx = r + 1 + kind;
            *olen = kind == 1 ? 4 + (l6 & 7) : l6 + 1;
        }
        return nx <= lim ? nx : kSlowRel;
    }
    // The ladder's answer (src/snappy_block.h:249-435) for such an element
    // when it accepts it; false: the full ladder decides.
    CDB_HD static bool accept_rel(const uint8_t* b, uint32_t r, uint32_t lim, uint64_t P,
                                  uint64_t d, uint64_t declared, lzl::Seq* sq) {
        const uint32_t tag = b[r];
        const uint32_t kind = tag & 3, l6 = tag >> 2;
        if (kind == 3 || (kind == 0 && l6 >= 60) || declared < d) return false;
        const uint64_t room = declared - d;
        if (kind == 0) {
            const uint32_t n = l6 + 1;
            if (r + 1 + n > lim || n > room) return false;
            sq->lit_src = P + 1;
            sq->lit = n;
            sq->ml = 0;
            sq->off = 0;
            sq->next = P + 1 + n;
        } else {
            if (r + 1 + kind > lim) return false;
            uint32_t off, len;
            if (kind == 1) {
                off = ((tag >> 5) << 8) | b[r + 1];
                len = 4 + (l6 & 7);
            } else {
                off = b[r + 1] | (static_cast<uint32_t>(b[r + 2]) << 8);
                len = l6 + 1;
            }
            if (off == 0 || off > d || len > room) return false;
            sq->lit_src = P;
            sq->lit = 0;
            sq->ml = len;
            sq->off = off;
            sq->next = P + 1 + kind;
        }
        sq->done = false;
        return true;
    }
};

// ---------------------------------------------------------------------------
// The tile's token records. LZ4: 32-bit fields, a token's position reused
// during execution for the in-group part of its match source. Snappy (up to
// kTile / 2 tokens a tile): 16-bit positions and lengths (lengths saturate:
// a longer token is a whole-CTA token, re-read by the ladder) and the
// in-group sources in their own array, so that four CTAs share an SM.
template <class F, bool Narrow = F::kSnappy>
struct TokRecs;
template <class F>
struct TokRecs<F, false> {
    static constexpr uint64_t kSat = 0xFFFFFFFFull;
    uint32_t pos[F::kMaxTok];  // token position - e; executing: its match's in-group source
    uint32_t lit[F::kMaxTok];  // saturated at kSat
    uint32_t ml[F::kMaxTok];
    uint32_t off[F::kMaxTok];
    uint32_t out[F::kMaxTok];  // output offset - d0
    CDB_HD uint32_t& dep(uint32_t i, uint32_t) { return pos[i]; }
};
template <class F>
struct TokRecs<F, true> {
    static constexpr uint64_t kSat = 0xFFFFull;
    uint16_t pos[F::kMaxTok];  // token position - e (< kTile)
    uint16_t lit[F::kMaxTok];  // saturated at kSat
    uint16_t ml[F::kMaxTok];
    uint32_t off[F::kMaxTok];
    uint32_t out[F::kMaxTok];       // output offset - d0
    uint32_t deps[kGroupTok];       // executing: per group token, its match's in-group source
    CDB_HD uint32_t& dep(uint32_t i, uint32_t g0) { return deps[i - g0]; }
};

// ---------------------------------------------------------------------------
// Shared memory of one CTA.
template <class F>
struct Shm {
    static constexpr uint32_t kMaxTok = F::kMaxTok;
    alignas(16) uint8_t in[kInBytes];  // staged input: positions [ibase, ibase + kInBytes)
    union {
        struct {
            uint32_t ex[kExIdx];                  // segment exits by position
            uint8_t rec[kSupers][kSupSegs][kCand];  // [w][segment][lane] entry codes
            uint32_t cand_exit[kSupers][kCand];
            uint8_t ovr[kSupers][kSupSegs];       // exact-walk entries
        } p;
        TokRecs<F> t;
    } u;
    alignas(16) uint8_t ring[kRing];
    uint32_t pend_bits[kGroupOut / 32 + 8];
    uint32_t seg_entry[kThreads];  // relative entry, or kUnknown for none
    uint32_t seg_cnt[kThreads];    // tokens; after the scan, the first token's index
    uint64_t seg_olen[kThreads];   // output bytes; after the scan, the first token's offset
    uint8_t pend[kThreads];        // per-thread pending match masks
    uint8_t chosen[kSupers];
    uint32_t wsum_c[kWarps];  // block scan: per-warp totals
    uint64_t wsum_o[kWarps];
    uint32_t first_ev;  // index of the first event token
    uint8_t ev_kind;
    int32_t ev_status;
    uint32_t cut;       // group cut (first big or overflowing token)
    uint32_t ntok;      // tokens in the tile
    uint64_t ototal;    // output bytes of the tile's tokens
    uint64_t tile_exit; // absolute position of the next tile, or kStepEnd
    uint64_t e;         // tile entry (absolute input position)
    uint64_t ibase;     // staged input base (absolute position)
    uint64_t d0;        // output position of the tile's first token
    uint64_t vlo;       // positions >= vlo are valid in the ring
    uint64_t flushed;   // positions < flushed are in the destination
    uint64_t dend;      // output length so far (end of the last executed token)
    int32_t status;     // chunk status (CUDEC_OK while running)
    uint32_t finished;  // the chunk is decided
};

// Input reader over the staged tile with the chunk's global bytes behind it
// (the ladders read only positions below S).
struct Reader {
    const uint8_t* g;
    const uint8_t* buf;
    uint64_t ibase;
    CDB_HD uint32_t at(uint64_t q) const {
        const uint64_t r = q - ibase;
        return r < kInBytes ? buf[r] : LZC_LDG(g + q);
    }
};

CDB_HD uint32_t exi(uint32_t r) { return r + (r >> 4); }  // padded exit index

// ---------------------------------------------------------------------------
// Ring helpers (positions are output offsets of the chunk).
struct Ring {
    uint8_t* ring;
    uint8_t* dst;
    uintptr_t dbase;
    CDB_HD uint32_t idx(uint64_t pos) const {
        return static_cast<uint32_t>((dbase + pos) & (kRing - 1));
    }
    // 16 ring bytes at position a: the five aligned words they touch.
    CDB_HD V16 get16(uint64_t a) const {
        constexpr uint32_t kMask = kRing / 4 - 1;
        const uint32_t ia = idx(a);
        const uint32_t wi = ia >> 2, sh = (ia & 3) * 8;
        const uint32_t* r32 = reinterpret_cast<const uint32_t*>(ring);
        const uint32_t w0 = r32[wi], w1 = r32[(wi + 1) & kMask], w2 = r32[(wi + 2) & kMask];
        const uint32_t w3 = r32[(wi + 3) & kMask], w4 = r32[(wi + 4) & kMask];
        return V16{{fsr(w0, w1, sh), fsr(w1, w2, sh), fsr(w2, w3, sh), fsr(w3, w4, sh)}};
    }
    // OR the first m (1..16) bytes of v into the ring at position x (the
    // bytes start at zero and each has one writer).
    CDB_HD void put16(uint64_t x, const V16& v, uint32_t m) const {
        const uint32_t ix = idx(x);
        const uint32_t sh = 8 * (ix & 3);
        const uint32_t bits = 8 * m;
        const uint32_t w0 = keep_low(v.w[0], bits);
        const uint32_t w1 = keep_low(v.w[1], bits > 32 ? bits - 32 : 0);
        const uint32_t w2 = keep_low(v.w[2], bits > 64 ? bits - 64 : 0);
        const uint32_t w3 = keep_low(v.w[3], bits > 96 ? bits - 96 : 0);
        uint32_t* r32 = reinterpret_cast<uint32_t*>(ring);
        constexpr uint32_t kMask = kRing / 4 - 1;
        const uint32_t wi = ix >> 2;
        at_or(r32 + wi, w0 << sh);
        at_or(r32 + ((wi + 1) & kMask), fsl(w0, w1, sh));
        at_or(r32 + ((wi + 2) & kMask), fsl(w1, w2, sh));
        at_or(r32 + ((wi + 3) & kMask), fsl(w2, w3, sh));
        if (sh) at_or(r32 + ((wi + 4) & kMask), w3 >> (32 - sh));
    }
};

// m (1..16) bytes at global address p, read as the aligned words holding
// them (no word past the last wanted byte is touched).
CDB_HD V16 gload16(const uint8_t* p, uint32_t m, bool readonly) {
    const uintptr_t ad = reinterpret_cast<uintptr_t>(p);
    const uint32_t s4 = static_cast<uint32_t>(ad & 3), sh = 8 * s4;
    const uint32_t* q = reinterpret_cast<const uint32_t*>(ad - s4);
    const uint32_t lw = (s4 + m - 1) >> 2;  // last word holding a wanted byte, 0..4
    uint32_t w[5] = {0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < 5; ++j)
        if (j <= lw) w[j] = readonly ? LZC_LDG(q + j) : q[j];
    return V16{{fsr(w[0], w[1], sh), fsr(w[1], w[2], sh), fsr(w[2], w[3], sh),
                fsr(w[3], w[4], sh)}};
}

// m (1..16) staged-or-global input bytes at absolute position a.
CDB_HD V16 in16(const Reader& in, uint64_t a, uint32_t m) {
    const uint64_t r = a - in.ibase;
    if (r < kInBytes && r + m <= kInBytes) {
        const uint32_t s4 = static_cast<uint32_t>(r & 3), sh = 8 * s4;
        const uint32_t* q = reinterpret_cast<const uint32_t*>(in.buf + (r - s4));
        const uint32_t lw = (s4 + m - 1) >> 2;
        uint32_t w[5] = {0, 0, 0, 0, 0};
        for (uint32_t j = 0; j < 5; ++j)
            if (j <= lw && (r - s4) + 4 * j < kInBytes) w[j] = q[j];
        return V16{{fsr(w[0], w[1], sh), fsr(w[1], w[2], sh), fsr(w[2], w[3], sh),
                    fsr(w[3], w[4], sh)}};
    }
    return gload16(in.g + a, m, true);
}

// The period expansion of a match with offset off < 16 starting from its
// first 16 bytes' source (low off bytes of v are the period): the match's
// first 16 bytes. Every later byte repeats the one rest(off) bytes back.
CDB_HD V16 period16(const V16& v, uint32_t off) {
    // Without branches, computed in every lane and selected: periods up to 8
    // bytes doubled in 64 bits, the next 8 bytes starting r = 8 mod off into
    // the period; for 9..15 bytes the first 16 - off bytes repeat once.
    const uint64_t lo = (static_cast<uint64_t>(v.w[1]) << 32) | v.w[0];
    const uint64_t hi = (static_cast<uint64_t>(v.w[3]) << 32) | v.w[2];
    const uint32_t d = off < 16 ? off : 16u;
    const uint32_t sb = 8 * d;  // 8..128
    uint64_t plo = lo & (~0ull >> ((64 - sb) & 63));
    plo |= sb < 64 ? plo << (sb & 63) : 0ull;
    plo |= sb < 32 ? plo << ((2 * sb) & 63) : 0ull;
    plo |= sb < 16 ? plo << ((4 * sb) & 63) : 0ull;
    // 8 mod d for d = 1..8, one nibble each
    const uint32_t r = static_cast<uint32_t>((0x012302000ull >> ((4 * d) & 63)) & 15);
    const uint64_t phi = (plo >> ((8 * r) & 63)) | (plo << ((8 * (d - r)) & 63));
    const uint32_t s2 = (sb - 64) & 63;
    const uint64_t qhi = (hi & ((1ull << s2) - 1)) | (lo << s2);
    const bool small = d <= 8;
    const uint64_t olo = small ? plo : lo, ohi = small ? phi : qhi;
    const V16 e{{static_cast<uint32_t>(olo), static_cast<uint32_t>(olo >> 32),
                 static_cast<uint32_t>(ohi), static_cast<uint32_t>(ohi >> 32)}};
    return off < 16 ? e : v;
}
CDB_HD uint32_t rest_distance(uint32_t off) {  // off * ceil(16 / off) for off < 16
    // Q - 16 for off = 1..15, one nibble each
    return off < 16 ? 16 + static_cast<uint32_t>((0xECA8642052402000ull >> (4 * (off & 15))) & 15)
                    : off;
}

// ---------------------------------------------------------------------------
// The chunk decoder (every thread of the CTA runs it; control flow depends
// only on shared state read after a barrier).
template <class F>
struct Chunk {
    Shm<F>& s;
    const uint8_t* g;  // compressed chunk
    uint64_t S;
    uint8_t* dst;
    uint64_t cap;
    uint64_t limit;    // LZ4: capacity; Snappy: declared length
    long long tl = 0;  // profiling builds: thread 0's last phase mark

    CDB_HD Reader reader() const { return Reader{g, s.in, s.ibase}; }
    // The staged bytes from the tile entry on, and how many of them the fast
    // forms may read (also bounded by the chunk's end).
    CDB_HD const uint8_t* staged() const { return s.in + (s.e - s.ibase); }
    CDB_HD uint32_t staged_lim() const {
        const uint64_t avail = kInBytes - (s.e - s.ibase);
        const uint64_t rest = S > s.e ? S - s.e : 0;
        return static_cast<uint32_t>(rest < avail ? rest : avail);
    }
    // The exact next position of the chain token at P (or kStepEnd) and its
    // output length: the fast form when it applies.
    CDB_HD uint64_t next_of(const Reader& in, const uint8_t* b, uint32_t lim, uint64_t P,
                            uint64_t* ol) const {
        if (P >= S) return kStepEnd;
        const uint64_t r = P - s.e;
        if (r < lim) {
            uint32_t o32 = 0;
            const uint32_t nr = F::step_rel(b, static_cast<uint32_t>(r), lim, &o32);
            if (nr != kSlowRel) {
                *ol = o32;
                return s.e + nr;
            }
        }
        return F::step(in, S, P, 0, ol);
    }
    CDB_HD Ring ring() const { return Ring{s.ring, dst, reinterpret_cast<uintptr_t>(dst)}; }

    // ---- 1. stage the tile's input
    CDB_HD void stage() {
        each([&](uint32_t tid) {
            if (tid == 0) {
                const uint64_t a = (reinterpret_cast<uintptr_t>(g) + s.e) & 15;
                s.ibase = s.e - a;  // may wrap below zero for the chunk's first block
            }
        });
        const int64_t ib = static_cast<int64_t>(s.ibase);
        each([&](uint32_t tid) {
            // aligned blocks holding at least one byte of [0, S) only
            for (uint32_t b = 16 * tid; b < kInBytes; b += 16 * kThreads) {
                const int64_t q = ib + b;
                if (q + 16 <= 0 || q >= static_cast<int64_t>(S)) continue;
                copy16_async(s.in + b, g + q);
            }
            land_async();
        });
    }

    // ---- 2. segment exits
    CDB_HD void seg_exits() {
        const Reader in = reader();
        const uint64_t e = s.e;
        const uint8_t* b = staged();
        const uint32_t lim = staged_lim();
        each([&](uint32_t t) {
            const uint32_t lo = t * kSeg, hi = lo + kSeg;
            for (int j = kSeg - 1; j >= 0; --j) {
                const uint32_t r = lo + static_cast<uint32_t>(j);
                const uint64_t P = e + r;
                uint32_t v;
                uint32_t o32 = 0;
                const uint32_t fr = r < lim ? F::step_rel(b, r, lim, &o32) : kSlowRel;
                if (fr != kSlowRel) {
                    v = fr >= hi ? fr : s.u.p.ex[exi(fr)];
                } else if (P >= S) {
                    v = kEndMark;
                } else {
                    uint64_t ol = 0;
                    const uint64_t n = F::step(in, S, P, kExtCap, &ol);
                    if (n == kStepUnknown) {
                        v = kUnknown;
                    } else if (n == kStepEnd) {
                        v = kEndMark;
                    } else {
                        const uint64_t nr = n - e;
                        if (nr >= hi) v = nr >= kFarRel ? kUnknown : static_cast<uint32_t>(nr);
                        else v = s.u.p.ex[exi(static_cast<uint32_t>(nr))];
                    }
                }
                s.u.p.ex[exi(r)] = v;
            }
        });
    }

    // ---- 3. candidate chase, lane k of warp w from position w * kSupPos + k
    CDB_HD void cand_chase() {
        each([&](uint32_t tid) {
            const uint32_t w = tid / 32, k = tid % 32;
            const uint32_t base = w * kSupPos;
            uint32_t xr = base + k;
            for (uint32_t j = 0; j < kSupSegs; ++j) {
                const uint32_t lo = base + j * kSeg;
                uint8_t code = kNoEntry;
                if (xr == kUnknown) {
                    code = kCodeUnk;
                } else if (xr == kEndMark) {
                    code = kCodeEnd;
                } else if (xr >= lo && xr < lo + kSeg) {
                    code = static_cast<uint8_t>(xr - lo);
                    xr = s.u.p.ex[exi(xr)];
                }
                s.u.p.rec[w][j][k] = code;
            }
            s.u.p.cand_exit[w][k] = xr;
        });
    }

    // Exact walk of super-segment w from the relative position xr (inside
    // it): records the entry of every segment the chain enters; returns the
    // chain's exit (absolute) or kStepEnd.
    CDB_HD uint64_t exact_walk(uint32_t w, uint64_t P) {
        const Reader in = reader();
        const uint64_t e = s.e;
        const uint64_t base = e + w * kSupPos, end = base + kSupPos;
        for (uint32_t j = 0; j < kSupSegs; ++j) s.u.p.ovr[w][j] = kNoEntry;
        while (P < end) {
            const uint32_t j = static_cast<uint32_t>((P - base) / kSeg);
            if (s.u.p.ovr[w][j] == kNoEntry)
                s.u.p.ovr[w][j] = static_cast<uint8_t>(P - base - j * kSeg);
            uint64_t ol = 0;
            const uint64_t n = P >= S ? kStepEnd : F::step(in, S, P, 0, &ol);
            if (n == kStepEnd) return kStepEnd;
            P = n;
        }
        return P;
    }

    // ---- 4. tile chase (one thread)
    CDB_HD void tile_chase() {
        each([&](uint32_t tid) {
            if (tid != 0) return;
            const uint64_t e = s.e;
            uint64_t P = e;  // the true chain's current position (absolute)
            for (uint32_t w = 0; w < kSupers; ++w) {
                const uint64_t base = e + w * kSupPos;
                if (P == kStepEnd) {
                    s.chosen[w] = kCodeEnd;
                    continue;
                }
                if (P >= base + kSupPos) {  // no token starts in this super-segment
                    s.chosen[w] = kNoEntry;
                    continue;
                }
                const uint64_t k = P - base;
                const uint32_t cx = k < kCand ? s.u.p.cand_exit[w][k] : kUnknown;
                if (k < kCand && cx != kUnknown) {
                    s.chosen[w] = static_cast<uint8_t>(k);
                    P = cx == kEndMark ? kStepEnd : e + cx;
                } else {
                    s.chosen[w] = kChoseOvr;
                    LZC_EVENT(5, 1);
                    P = exact_walk(w, P);
                }
            }
            s.tile_exit = P;
        });
    }

    // The entry code of thread t's segment after the tile chase.
    CDB_HD uint8_t entry_code(uint32_t t) const {
        const uint32_t w = t / kSupSegs, j = t % kSupSegs;
        const uint8_t c = s.chosen[w];
        if (c == kChoseOvr) return s.u.p.ovr[w][j];
        if (c < kCand) return s.u.p.rec[w][j][c];
        return kNoEntry;
    }

    // Exclusive prefix of the per-segment token counts and output bytes (in
    // place) and the tile's totals.
    CDB_HD void scan_counts() {
#if defined(__CUDA_ARCH__)
        const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
        const uint32_t c = s.seg_cnt[t];
        const uint64_t o = s.seg_olen[t];
        uint32_t ci = c;
        uint64_t oi = o;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t c2 = __shfl_up_sync(0xffffffffu, ci, d);
            const uint64_t o2 = __shfl_up_sync(0xffffffffu, oi, d);
            if (lane >= d) {
                ci += c2;
                oi += o2;
            }
        }
        if (lane == 31) {
            s.wsum_c[w] = ci;
            s.wsum_o[w] = oi;
        }
        __syncthreads();
        uint32_t cb = 0;
        uint64_t ob = 0;
        for (uint32_t k = 0; k < w; ++k) {
            cb += s.wsum_c[k];
            ob += s.wsum_o[k];
        }
        s.seg_cnt[t] = cb + ci - c;
        s.seg_olen[t] = ob + oi - o;
        if (t == kThreads - 1) {
            s.ntok = cb + ci;
            s.ototal = ob + oi;
        }
        __syncthreads();
#else
        uint32_t cb = 0;
        uint64_t ob = 0;
        for (uint32_t t = 0; t < kThreads; ++t) {
            const uint32_t c = s.seg_cnt[t];
            const uint64_t o = s.seg_olen[t];
            s.seg_cnt[t] = cb;
            s.seg_olen[t] = ob;
            cb += c;
            ob += o;
        }
        s.ntok = cb;
        s.ototal = ob;
#endif
    }

    // ---- 5. count tokens and output bytes per segment (exact steps)
    CDB_HD void count() {
        const Reader in = reader();
        const uint64_t e = s.e;
        const uint8_t* b = staged();
        const uint32_t lim = staged_lim();
        each([&](uint32_t t) {
            const uint8_t c = entry_code(t);
            uint32_t n = 0;
            uint64_t ol_sum = 0;
            uint32_t entry = kUnknown;
            if (c < kSeg) {
                entry = t * kSeg + c;
                uint64_t P = e + entry;
                const uint64_t hi = e + (t + 1) * kSeg;
                while (P < hi) {
                    ++n;
                    uint64_t ol = 0;
                    const uint64_t nx = next_of(in, b, lim, P, &ol);
                    ol_sum += ol;
                    if (nx == kStepEnd) break;
                    P = nx;
                }
            }
            s.seg_entry[t] = entry;
            s.seg_cnt[t] = n;
            s.seg_olen[t] = ol_sum;
        });
        scan_counts();
    }

    // The ladder's answer for token i of the tile (its position and output
    // offset from the records): status, and whether it ends the chunk.
    CDB_HD int ladder_at(uint64_t P, uint64_t d, lzl::Seq* sq) const {
        *sq = lzl::Seq{};
        if (F::kSnappy && P == S) {
            sq->done = true;
            return F::finish(d, limit);
        }
        return F::parse(reader(), S, limit, P, d, sq);
    }

    // ---- 6. exact ladder per token; records; first event
    CDB_HD void check() {
        const Reader in = reader();
        const uint64_t e = s.e, d0 = s.d0;
        const uint8_t* b = staged();
        const uint32_t lim = staged_lim();
        each([&](uint32_t t) {
            if (t == 0) s.first_ev = 0xFFFFFFFFu;
        });
        each([&](uint32_t t) {
            const uint32_t entry = s.seg_entry[t];
            if (entry == kUnknown) return;
            uint32_t i = s.seg_cnt[t];
            uint64_t o = s.seg_olen[t];
            uint64_t P = e + entry;
            const uint64_t hi = e + (t + 1) * kSeg;
            while (P < hi) {
                if (i >= F::kMaxTok || o > 0xFFFFFFFFull) {  // unreachable (tile bounds)
                    at_min(&s.first_ev, i < F::kMaxTok ? i : F::kMaxTok - 1);
                    break;
                }
                lzl::Seq sq;
                int st = CUDEC_OK;
                uint64_t nx, ol;
                const uint64_t r = P - e;
                if (r < lim && F::accept_rel(b, static_cast<uint32_t>(r), lim, P, d0 + o, limit,
                                             &sq)) {
                    nx = sq.next;
                    ol = sq.lit + sq.ml;
                } else {
                    st = ladder_at(P, d0 + o, &sq);
                    ol = 0;
                    nx = next_of(in, b, lim, P, &ol);
                }
                constexpr uint64_t kSat = TokRecs<F>::kSat;
                s.u.t.pos[i] = static_cast<uint32_t>(P - e);
                s.u.t.lit[i] = static_cast<uint32_t>(sq.lit > kSat ? kSat : sq.lit);
                s.u.t.ml[i] = static_cast<uint32_t>(sq.ml > kSat ? kSat : sq.ml);
                s.u.t.off[i] = sq.off;
                s.u.t.out[i] = static_cast<uint32_t>(o);
                // the first failing or terminal token ends the chunk; a step
                // that disagrees with the ladder cannot happen, and would be
                // reported as an internal error below
                if (st != CUDEC_OK || sq.done || nx != sq.next) {
                    at_min(&s.first_ev, i);
                    break;
                }
                ++i;
                o += ol;
                P = nx;
            }
        });
        each([&](uint32_t t) {
            if (t != 0) return;
            const uint32_t fe = s.first_ev;
            s.ev_kind = kEvNone;
            s.ev_status = CUDEC_OK;
            if (fe == 0xFFFFFFFFu) return;
            if (fe >= s.ntok) {  // unreachable (tile bounds)
                s.ev_kind = kEvFail;
                s.ev_status = CUDEC_ERR_CUDA;
                return;
            }
            lzl::Seq sq;
            const int st = ladder_at(e + s.u.t.pos[fe], d0 + s.u.t.out[fe], &sq);
            if (st != CUDEC_OK) {
                s.ev_kind = kEvFail;
                s.ev_status = st;
            } else if (sq.done) {
                s.ev_kind = kEvDone;
            } else {
                s.ev_kind = kEvFail;
                s.ev_status = CUDEC_ERR_CUDA;
            }
        });
    }

    // ---- 7. execution
    CDB_HD bool is_big(uint32_t i) const {
        const uint64_t n = static_cast<uint64_t>(s.u.t.lit[i]) + s.u.t.ml[i];
        return n > kBig;
    }

    // Copy ring bytes [flushed, end) to the destination: the head up to the
    // first aligned boundary and, when `fin`, the tail by bytes; whole
    // aligned 16-byte blocks as vector stores.
    CDB_HD void flush(uint64_t end, bool fin) {
        const Ring rg = ring();
        const uint64_t f = s.flushed;
        if (end <= f) return;
        // in addresses: the first aligned boundary at or after f, the last at
        // or before end (the latter may lie below the former when [f, end)
        // sits inside one partial block)
        const uintptr_t db = reinterpret_cast<uintptr_t>(dst);
        const uintptr_t fa_abs = (db + f + 15) & ~static_cast<uintptr_t>(15);
        const uintptr_t ea_abs = (db + end) & ~static_cast<uintptr_t>(15);
        const uint64_t hend = (fa_abs < db + end ? fa_abs : db + end) - db;
        const bool blocks = ea_abs > fa_abs;
        const uint64_t fa = fa_abs - db, ea = blocks ? ea_abs - db : hend;
        each([&](uint32_t t) {
            if (f + t < hend) dst[f + t] = rg.ring[rg.idx(f + t)];
            if (blocks)
                for (uint64_t b = fa + 16ull * t; b < ea; b += 16ull * kThreads)
                    st16(dst + b, s.ring + rg.idx(b));
            if (fin && ea < end && ea + t < end) dst[ea + t] = rg.ring[rg.idx(ea + t)];
        });
        const uint64_t nf = fin ? end : ea;
        each([&](uint32_t t) {
            if (t == 0) s.flushed = nf;
        });
    }

    // m (1..16) already-written output bytes at position a.
    CDB_HD V16 fetch16(const Ring& rg, uint64_t a, uint32_t m) const {
        const uint64_t vlo = s.vlo;
        if (a >= vlo) return rg.get16(a);
        if (a + m <= vlo) return gload16(dst + a, m, false);
        V16 v{{0, 0, 0, 0}};
        for (uint32_t j = 0; j < m; ++j) {
            const uint64_t q = a + j;
            const uint32_t b = q >= vlo ? rg.ring[rg.idx(q)] : dst[q];
            v.w[j >> 2] |= b << (8 * (j & 3));
        }
        return v;
    }

    CDB_HD void copy_match_ring(const Ring& rg, uint64_t o, uint32_t n, uint32_t off) const {
        const uint32_t m0 = n < 16 ? n : 16u;
        rg.put16(o, period16(fetch16(rg, o - off, off < 16 ? off : m0), off), m0);
        const uint32_t d = rest_distance(off);
        for (uint32_t k = 16; k < n; k += 16) {
            const uint32_t m = n - k < 16 ? n - k : 16u;
            rg.put16(o + k, fetch16(rg, o + k - d, m), m);
        }
    }

    // bits [a, b) of the pending map (group-relative output offsets)
    CDB_HD bool bits_clear(uint32_t a, uint32_t b) const {
        for (uint32_t w = a >> 5; w <= (b - 1) >> 5; ++w) {
            uint32_t m = ~0u;
            if (w == a >> 5) m &= ~0u << (a & 31);
            if (w == (b - 1) >> 5) m &= ~0u >> (31 - ((b - 1) & 31));
            if (*static_cast<volatile uint32_t*>(&s.pend_bits[w]) & m) return false;
        }
        return true;
    }
    CDB_HD void bits_set(uint32_t a, uint32_t b, bool set) {
        for (uint32_t w = a >> 5; w <= (b - 1) >> 5; ++w) {
            uint32_t m = ~0u;
            if (w == a >> 5) m &= ~0u << (a & 31);
            if (w == (b - 1) >> 5) m &= ~0u >> (31 - ((b - 1) & 31));
            if (set) at_or(&s.pend_bits[w], m);
            else at_and(&s.pend_bits[w], ~m);
        }
    }

    // Token i's match if its source is ready: copied, then published.
    CDB_HD bool try_match(const Ring& rg, uint32_t i, uint32_t g0, uint64_t G0) {
        // the in-group part of its source, packed at the literal phase
        const uint32_t dep = s.u.t.dep(i, g0);
        const uint32_t lo = dep & 0xFFFFu, hi = dep >> 16;
        if (lo < hi && !bits_clear(lo, hi)) return false;
        const uint32_t lit = s.u.t.lit[i], ml = s.u.t.ml[i], off = s.u.t.off[i];
        const uint64_t ms = s.d0 + s.u.t.out[i] + lit;
#if defined(__CUDA_ARCH__)
        __threadfence_block();  // the source bytes' writers published before their bits cleared
#endif
        copy_match_ring(rg, ms, ml, off);
#if defined(__CUDA_ARCH__)
        __threadfence_block();  // the bytes land before the bits that publish them
#endif
        const uint32_t a = static_cast<uint32_t>(ms - G0);
        bits_set(a, a + ml, false);
        return true;
    }

    // Tokens [g0, g1), all of at most kBig bytes, output [G0, G1) within
    // kGroupOut: literals, then matches in rounds, through the ring.
    CDB_HD void exec_group(uint32_t g0, uint32_t g1) {
        const Reader in = reader();
        const Ring rg = ring();
        const uint64_t d0 = s.d0, e = s.e;
        const uint64_t G0 = d0 + s.u.t.out[g0];
        const uint64_t G1 = d0 + s.u.t.out[g1 - 1] + s.u.t.lit[g1 - 1] + s.u.t.ml[g1 - 1];
        // the clear below may zero up to 15 bytes past G1, whose slots held
        // positions up to G1 + 15 - kRing: those are read back from dst
        each([&](uint32_t t) {
            if (t == 0 && G1 + 16 > s.vlo + kRing) s.vlo = G1 + 16 - kRing;
        });
        // clear the group's ring bytes and its pending map
        const uint32_t ib = rg.idx(G0);
        const uint32_t span = static_cast<uint32_t>(G1 - G0);
        each([&](uint32_t t) {
            uint32_t* r32 = reinterpret_cast<uint32_t*>(s.ring);
            const uint32_t w0 = ib >> 2;
            if (t == 0) at_and(r32 + w0, (1u << (8 * (ib & 3))) - 1);
            if (t >= 1 && t < 4 - (w0 & 3)) r32[w0 + t] = 0;
            const uint32_t end = ib + span;
            for (uint32_t q = (ib & ~15u) + 16 + 16 * t; q < end; q += 16 * kThreads)
                zero16(s.ring + (q & (kRing - 1)));
            for (uint32_t w = t; w < kGroupOut / 32 + 8; w += kThreads) s.pend_bits[w] = 0;
        });
        // literals; pending bits of the matches
        each([&](uint32_t t) {
            uint8_t pm = 0;
            for (uint32_t k = 0; k < kPerThread; ++k) {
                const uint32_t i = g0 + t + k * kThreads;
                if (i >= g1) break;
                const uint32_t lit = s.u.t.lit[i], ml = s.u.t.ml[i];
                const uint64_t o = d0 + s.u.t.out[i];
                if (lit) {
                    const uint64_t ls = F::lit_src(in, e + s.u.t.pos[i], lit);
                    for (uint32_t q = 0; q < lit; q += 16) {
                        const uint32_t m = lit - q < 16 ? lit - q : 16u;
                        rg.put16(o + q, in16(in, ls + q, m), m);
                    }
                }
                if (ml) {
                    const uint32_t a = static_cast<uint32_t>(o + lit - G0);
                    bits_set(a, a + ml, true);
                    pm |= static_cast<uint8_t>(1u << k);
                    // the part of its source inside the group, [lo, hi)
                    // relative to G0 (empty: every source byte precedes the
                    // group); the token's position is not needed past here
                    const uint64_t ms = o + lit, src = ms - s.u.t.off[i];
                    const uint64_t lo = src > G0 ? src : G0;
                    const uint64_t hi = src + ml < ms ? src + ml : ms;
                    s.u.t.dep(i, g0) = lo < hi ? static_cast<uint32_t>(lo - G0) |
                                                     (static_cast<uint32_t>(hi - G0) << 16)
                                               : 0u;
                }
            }
            s.pend[t] = pm;
        });
        LZC_PHASE(6);
        LZC_EVENT(3, 1);
        // matches, as data flow: every thread copies each of its pending
        // matches once no byte its source reads is still pending, then
        // publishes it (block fence, then its pending bits cleared). The
        // lowest pending match of the group is always ready, so every pass
        // over the CTA makes progress; passes per thread are bounded.
#if defined(__CUDA_ARCH__)
        each([&](uint32_t t) {
            uint8_t pm = s.pend[t];
            uint32_t spin = 0;
            for (; pm; ++spin) {
                // a thread's matches in order (its lowest pending first): a
                // warp's lanes then hold consecutive tokens and copy together
                for (uint32_t k = 0; k < kPerThread; ++k)
                    if (pm & (1u << k)) {
                        if (try_match(rg, g0 + t + k * kThreads, g0, G0))
                            pm = static_cast<uint8_t>(pm & ~(1u << k));
                        break;
                    }
                if (pm && spin >= kSpinCap) {  // unreachable: see above
                    atomicExch(reinterpret_cast<int*>(&s.status), CUDEC_ERR_CUDA);
                    break;
                }
            }
#ifdef CDB_PHASE_TIMING
            // one global add per warp (the counts summed across its lanes)
            const unsigned ws = __reduce_add_sync(0xffffffffu, spin);
            if ((t & 31) == 0) atomicAdd(&lzc_events[6], static_cast<unsigned long long>(ws));
#endif
        });
#else
        for (uint32_t pass = 0;; ++pass) {
            bool any = false;
            for (uint32_t t = 0; t < kThreads; ++t) {
                uint8_t pm = s.pend[t];
                for (uint32_t k = 0; k < kPerThread; ++k)
                    if ((pm & (1u << k)) && try_match(rg, g0 + t + k * kThreads, g0, G0))
                        pm = static_cast<uint8_t>(pm & ~(1u << k));
                s.pend[t] = pm;
                any = any || pm != 0;
            }
            if (!any) break;
            if (pass > g1 - g0) {  // unreachable: every pass finishes a match
                s.status = CUDEC_ERR_CUDA;
                break;
            }
        }
#endif
        LZC_EVENT(2, 1);
        LZC_PHASE(7);
        flush(G1, false);
        each([&](uint32_t t) {
            if (t == 0) s.dend = G1;
        });
        LZC_PHASE(8);
    }

    // One token longer than kBig: the whole CTA copies it straight to the
    // destination (its exact 64-bit lengths from the ladder).
    CDB_HD void exec_big(uint32_t i) {
        const Reader in = reader();
        const uint64_t P = s.e + s.u.t.pos[i];
        const uint64_t o = s.d0 + s.u.t.out[i];
        lzl::Seq sq;
        (void)in;
        (void)ladder_at(P, o, &sq);  // accepted before: the same exact lengths
        flush(o, true);
        // literal run: input -> destination
        const uint64_t lit = sq.lit;
        const uint64_t ls = sq.lit_src;
        each([&](uint32_t t) {
            for (uint64_t q = 16ull * t; q < lit; q += 16ull * kThreads) {
                const uint32_t m = lit - q < 16 ? static_cast<uint32_t>(lit - q) : 16u;
                const V16 v = gload16(g + ls + q, m, true);
                put_global(dst + o + q, v, m);
            }
        });
        // match: waves that never read their own output
        const uint64_t ms = o + lit, ml = sq.ml;
        const uint32_t off = sq.off;
        if (ml) {
            if (off >= 16 * kThreads) {
                for (uint64_t wv = 0; wv < ml; wv += 16ull * kThreads) {
                    each([&](uint32_t t) {
                        const uint64_t q = wv + 16ull * t;
                        if (q >= ml) return;
                        const uint32_t m = ml - q < 16 ? static_cast<uint32_t>(ml - q) : 16u;
                        put_global(dst + ms + q, gload16(dst + ms + q - off, m, false), m);
                    });
                }
            } else {
                // the period (off < 4096 bytes) in the ring, then each byte is
                // period[(x - ms) mod off]
                each([&](uint32_t t) {
                    for (uint32_t j = t; j < off; j += kThreads) s.ring[j] = dst[ms - off + j];
                });
                each([&](uint32_t t) {
                    for (uint64_t q = 16ull * t; q < ml; q += 16ull * kThreads) {
                        const uint32_t m = ml - q < 16 ? static_cast<uint32_t>(ml - q) : 16u;
                        uint32_t ph = static_cast<uint32_t>(q % off);
                        V16 v{{0, 0, 0, 0}};
                        for (uint32_t j = 0; j < m; ++j) {
                            v.w[j >> 2] |= static_cast<uint32_t>(s.ring[ph]) << (8 * (j & 3));
                            ph = ph + 1 == off ? 0 : ph + 1;
                        }
                        put_global(dst + ms + q, v, m);
                    }
                });
            }
        }
        const uint64_t end = ms + ml;
        each([&](uint32_t t) {
            if (t == 0) {
                s.flushed = end;
                s.vlo = end;
                s.dend = end;
            }
        });
        LZC_PHASE(9);
        LZC_EVENT(4, 1);
    }

    CDB_HD void execute(uint32_t ne) {
        uint32_t g0 = 0;
        while (g0 < ne && s.status == CUDEC_OK) {
            // the group: up to kGroupTok tokens, cut at a big token or where
            // the output passes kGroupOut
            const uint32_t lim = ne - g0 < kGroupTok ? ne : g0 + kGroupTok;
            const uint32_t o0 = s.u.t.out[g0];
            each([&](uint32_t t) {
                if (t == 0) s.cut = lim;
            });
            each([&](uint32_t t) {
                for (uint32_t i = g0 + t; i < lim; i += kThreads) {
                    const uint64_t end = static_cast<uint64_t>(s.u.t.out[i]) - o0 +
                                         s.u.t.lit[i] + s.u.t.ml[i];
                    if (is_big(i) || end > kGroupOut) {
                        at_min(&s.cut, i);
                        break;
                    }
                }
            });
            const uint32_t c = s.cut;
            LZC_PHASE(10);
            if (c == g0) {
                exec_big(g0);
                g0 += 1;
            } else {
                exec_group(g0, c);
                g0 = c;
            }
        }
    }

    // ---- the chunk
    CDB_HD int run(uint64_t* written) {
        uint64_t first = 0, lim = 0;
        int st = F::begin(Reader{g, s.in, ~0ull >> 1}, S, cap, &first, &lim);
        if (st != CUDEC_OK) return st;
        limit = lim;
        each([&](uint32_t t) {
            if (t == 0) {
                s.e = first;
                s.d0 = 0;
                s.vlo = 0;
                s.flushed = 0;
                s.dend = 0;
                s.status = CUDEC_OK;
                s.finished = 0;
            }
        });
        // every tile holds at least one token and consumes at least one
        // position, so the chunk's tiles number at most S + 1
        uint64_t fuel = S == ~0ull ? ~0ull : S + 1;
        LZC_START();
        for (;;) {
            stage();
            LZC_PHASE(0);
            seg_exits();
            LZC_PHASE(1);
            cand_chase();
            LZC_PHASE(2);
            tile_chase();
            LZC_PHASE(3);
            count();
            LZC_PHASE(4);
            if (s.ntok > F::kMaxTok) return CUDEC_ERR_CUDA;  // unreachable (tile bounds)
            check();
            LZC_PHASE(5);
            LZC_EVENT(0, 1);
            LZC_EVENT(1, s.ntok);
            const uint32_t fe = s.first_ev;
#ifdef LZC_TRACE
            LZC_TRACE(s.e, s.d0, s.ntok, s.ototal, fe, s.ev_kind, s.ev_status, s.tile_exit);
            if (fe != 0xFFFFFFFFu && s.ev_kind == kEvFail) LZC_TRACE_SEGS(s);
#endif
            if (fe != 0xFFFFFFFFu && s.ev_kind == kEvFail) return s.ev_status;
            const uint32_t ne = fe != 0xFFFFFFFFu ? fe + 1 : s.ntok;
            execute(ne);
            if (s.status != CUDEC_OK) return s.status;
            if (fe != 0xFFFFFFFFu) break;  // terminal token executed
            if (s.tile_exit == kStepEnd || fuel-- == 0) return CUDEC_ERR_CORRUPT_INPUT;
            const uint64_t nd = s.d0 + s.ototal;
            const uint64_t ne_pos = s.tile_exit;
            each([&](uint32_t t) {
                if (t == 0) {
                    s.e = ne_pos;
                    s.d0 = nd;
                }
            });
        }
        const uint64_t d = s.dend;
        flush(d, true);
        *written = d;
        return CUDEC_OK;
    }
};


// ---------------------------------------------------------------------------
// The batch kernel: one CTA per chunk at a time, persistent grid-stride over
// the batch. Dynamic shared memory: sizeof(Shm<F>).
#if defined(__CUDACC__)
template <class F>
__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    lz_cta_kernel(const void* const* src_ptrs, const size_t* src_sizes, void* const* dst_ptrs,
                  const size_t* dst_caps, size_t n, cudec_chunk_result* results) {
    extern __shared__ __align__(16) uint8_t lzc_smem[];
    Shm<F>& s = *reinterpret_cast<Shm<F>*>(lzc_smem);
    for (size_t c = blockIdx.x; c < n; c += gridDim.x) {
        Chunk<F> ch{s, static_cast<const uint8_t*>(src_ptrs[c]), src_sizes[c],
                    static_cast<uint8_t*>(dst_ptrs[c]), dst_caps[c], 0};
        uint64_t written = 0;
        const int st = ch.run(&written);
        if (threadIdx.x == 0) {
            results[c].status = st;
            results[c].reserved = 0;
            results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
        __syncthreads();  // the next chunk reuses the shared state
    }
}
#endif

}  // namespace lzc
}  // namespace cdb
