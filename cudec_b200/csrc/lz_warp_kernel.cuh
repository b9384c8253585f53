// Warp-per-chunk decoder for the byte-oriented LZ formats (LZ4 block, raw
// Snappy).
//
// One warp owns one chunk at a time (persistent grid-stride over the batch).
// The chunk's compressed bytes stream through a per-warp shared-memory input
// window (kIn bytes, filled ahead of the parse by cp.async). Tokens are
// handled in groups of up to 32:
//
//   1. the group walk finds the next 32 tokens of the chain: every lane takes
//      the format's branch-free step at two of the next 64 positions, and
//      the chain through those positions is followed with shuffles, four
//      hops per branch (the uncommon token headers take a general step);
//      lane k ends up with the k-th token's position and output offset;
//   2. each lane runs the format's exact accept/reject ladder on its token
//      (output position from the walk's running sum of lengths); the first
//      failing or terminal token decides the chunk exactly as the serial
//      parser would;
//   3. tokens of at most kBig bytes execute lane-parallel through a per-warp
//      output ring (kRing bytes, indexed by destination address mod kRing,
//      so ring blocks and destination blocks share alignment): literal runs
//      first, then matches in rounds (a lane copies once no unfinished
//      match's output overlaps the bytes its source reads). Every byte has
//      one writer, so pieces are OR-ed into the cleared ring as five aligned
//      words; a match's first piece is one fetch and one write in every
//      lane, a period under 16 bytes expanded in registers (period16), the
//      rest copied at rest_distance. Completed 16-byte blocks leave the
//      ring as aligned, coalesced 16-byte stores. Match sources older than
//      the ring are read back from the destination. Longer tokens are
//      copied by the whole warp straight to the destination.
//
// On this in-order, latency-bound warp a data-dependent branch that splits
// the lanes costs more than the work it skips, so the copy paths compute
// and select (masks by clamped funnel shifts, all five OR-words, the period
// expansion in every lane) rather than branch per lane.
//
// Statuses follow the reference ladders exactly: LZ4 iderex/cudec
// src/lz4_block.h:95-258, Snappy src/snappy_block.h:172-435.
#pragma once

#include <cstdint>

#include "cudec.h"
#include "lz_ladder.cuh"

namespace cdb {
namespace lzw {

constexpr uint32_t kWarps = 4;               // warps per CTA
constexpr uint32_t kThreads = 32 * kWarps;
constexpr uint32_t kRing = 8192;             // output ring per warp (bytes)
constexpr uint32_t kIn = 4096;               // input window per warp (bytes)
constexpr uint32_t kInAhead = kIn - 64;      // largest fill distance past the parse
constexpr uint32_t kBatchMax = 4096;         // largest output staged per ring batch
constexpr uint64_t kBig = 256;               // longer tokens are copied by the whole warp
constexpr uint32_t kPW = 1024;               // largest parse reach (input bytes landed ahead)
constexpr uint32_t kHops = 4;                // chain hops per branch in the group walk
constexpr uint32_t kStop = ~0u;              // the group walk stops at this token
constexpr uint32_t kWordStop = ~0u;          // packed-step marker: take the general step
constexpr uint32_t kRefill = 1024;           // input progress between window refills
constexpr uint32_t kWarpSmem = kRing + kIn;
constexpr unsigned kFull = 0xffffffffu;
static_assert(kBatchMax + 32 <= kRing, "a batch never overwrites unflushed bytes");

// Per-launch (or per size bucket) shape of the decode: parse reach (input
// bytes past a group's first token that must have landed in the window
// before the group is walked, <= kPW, a multiple of 32), input fill
// distance past the parse (pw + 64 .. kInAhead) and output bytes per ring
// batch (<= kBatchMax). Any values in range decode identically; they only
// move time.
struct Tune {
    uint32_t pw, ahead, batch;
};
constexpr Tune kDefaultTune{kPW, kInAhead, kBatchMax};

__host__ __device__ constexpr bool tune_valid(const Tune& t) {
    return t.pw >= 32 && t.pw <= kPW && t.pw % 32 == 0 && t.ahead >= t.pw + 64 &&
           t.ahead <= kInAhead && t.batch >= 256 && t.batch <= kBatchMax;
}

// Profiling builds (-DCDB_PHASE_TIMING) accumulate per-phase SM cycles and
// event counts over all chunks of a launch. Cycles: 0 window refill, 1 walk,
// 2 checks, 3 execute (of which 4 clear, 6 literals, 7 match rounds), 5 the
// whole chunk. Events: 0 groups, 1 tokens, 2 match rounds, 3 tokens copied
// straight to the destination.
#ifdef CDB_PHASE_TIMING
__device__ unsigned long long lzw_cycles[8];
__device__ unsigned long long lzw_events[8];
#define LZW_T(v) const long long v = clock64()
#define LZW_ADD(i, t0) \
    if (lane == 0) atomicAdd(&lzw_cycles[i], static_cast<unsigned long long>(clock64() - (t0)))
#define LZW_EV(i, n) \
    if (lane == 0) atomicAdd(&lzw_events[i], static_cast<unsigned long long>(n))
#else
#define LZW_T(v)
#define LZW_ADD(i, t0)
#define LZW_EV(i, n)
#endif

using Seq = lzl::Seq;

__device__ __forceinline__ uint32_t ldb(const uint8_t* g, uint64_t p) {
    return __ldg(g + p);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// The chunk's bytes straight from global memory (the ladders' reader for a
// chunk's preamble).
struct GBytes {
    const uint8_t* g;
    __device__ __forceinline__ uint32_t at(uint64_t q) const { return ldb(g, q); }
};

// The chunk's compressed bytes: positions in [lo, lo + span) come from the
// shared-memory window (indexed by global address mod kIn, so its 16-byte
// blocks are the input's aligned blocks), others straight from global. A
// refill in flight only writes slots of positions below lo.
struct In {
    const uint8_t* g;
    const uint8_t* win;
    uintptr_t gbase;
    uint64_t lo, span;  // the window holds positions [lo, lo + span)
    __device__ __forceinline__ bool held(uint64_t q, uint64_t m) const {
        return q >= lo && q - lo + m <= span;
    }
    __device__ __forceinline__ uint32_t at(uint64_t q) const {
        if (q - lo < span)
            return win[(static_cast<uint32_t>(gbase) + static_cast<uint32_t>(q)) & (kIn - 1)];
        return ldb(g, q);
    }
};

// ---------------------------------------------------------------------------
// LZ4 block: the exact ladder (lz_ladder.cuh) plus the group walk's steps.
struct Lz4 : lzl::Lz4Ladder {
    // The group walk reads token headers from the landed window only: r is a
    // position relative to the group's first token, its window slot is
    // (gb + r) & (kIn - 1), and e bounds what may be read (the input end or
    // the window end, whichever comes first).
    //
    // Branch-free step for the common token: each length carries at most one
    // extension byte (below 255) and the token lies well inside [0, e).
    // Returns whether it applied; *nr (the next token) and *len (literal +
    // match bytes) are meaningful only then. Every load is a masked window
    // slot, so none leaves the window whatever r is. The next position does
    // not depend on the match's extension byte, so one load latency (token
    // and literal extension in parallel) separates consecutive tokens.
    __device__ __forceinline__ static bool step_simple(const uint8_t* win, uint32_t gb, uint32_t e,
                                                       uint32_t r, uint32_t* nr, uint32_t* len) {
        const uint32_t tok = win[(gb + r) & (kIn - 1)];
        const uint32_t b1 = win[(gb + r + 1) & (kIn - 1)];
        const uint32_t lit0 = tok >> 4, mlc = tok & 15;
        const bool le = lit0 == 15, me = mlc == 15;
        const uint32_t lit = le ? 15 + b1 : lit0;
        const uint32_t q = r + (le ? 2u : 1u) + lit;  // the offset's position
        const uint32_t b2 = win[(gb + q + 2) & (kIn - 1)];
        *nr = q + (me ? 3u : 2u);
        *len = lit + (me ? 19 + b2 : mlc + 4);
        return !(le & (b1 == 255)) & !(me & (b2 == 255)) & (q + kSrcSlack <= e);
    }

    // General step inside [0, e): the next token's relative position and the
    // token's output length, or kStop when the token is not a non-terminal
    // one whose header lies wholly inside [0, e) (the exact ladder then
    // decides it). Equals the exact ladder's next position and lengths for
    // every token the ladder accepts as non-terminal.
    __device__ __forceinline__ static uint32_t walk(const uint8_t* win, uint32_t gb, uint32_t e,
                                                    uint32_t r, uint32_t* len) {
        if (r >= e) return kStop;
        const uint32_t tok = win[(gb + r) & (kIn - 1)];
        uint32_t q = r + 1;
        uint32_t lit = tok >> 4;
        if (lit == 15) {
            uint32_t b;
            do {
                if (q >= e) return kStop;
                b = win[(gb + q) & (kIn - 1)];
                ++q;
                lit += b;
            } while (b == 255);
        }
        if (lit > e - q) return kStop;
        q += lit;
        if (e - q < kSrcSlack) return kStop;
        q += 2;
        uint32_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15) {
            uint32_t b;
            do {
                if (q >= e) return kStop;
                b = win[(gb + q) & (kIn - 1)];
                ++q;
                ml += b;
            } while (b == 255);
        }
        *len = lit + ml;
        return q;
    }

};

// ---------------------------------------------------------------------------
// Raw Snappy: the exact ladder (lz_ladder.cuh) plus the group walk's steps.
struct Snappy : lzl::SnappyLadder {
    // Branch-free step for tags whose length is in the tag (see
    // Lz4::step_simple). Strict bound: an element ending at e may end the
    // input, which only the general step (with its end check) decides.
    __device__ __forceinline__ static bool step_simple(const uint8_t* win, uint32_t gb, uint32_t e,
                                                       uint32_t r, uint32_t* nr, uint32_t* len) {
        const uint32_t tag = win[(gb + r) & (kIn - 1)];
        const uint32_t kind = tag & 3, l6 = tag >> 2;
        const uint32_t hdr = kind == 0 ? 1 : (kind == 1 ? 2 : (kind == 2 ? 3 : 5));
        const uint32_t n = kind == 1 ? 4 + (l6 & 7) : l6 + 1;
        *nr = r + hdr + (kind == 0 ? n : 0);
        *len = n;
        return !(kind == 0 && l6 >= 60) & (*nr < e);
    }

    // General step inside [0, e) (see Lz4::walk): one element per step.
    __device__ __forceinline__ static uint32_t walk(const uint8_t* win, uint32_t gb, uint32_t e,
                                                    uint32_t r, uint32_t* len) {
        if (r >= e) return kStop;
        const uint32_t tag = win[(gb + r) & (kIn - 1)];
        const uint32_t kind = tag & 3;
        if (kind == 0) {
            const uint32_t l6 = tag >> 2;
            uint32_t hdr = 1, n = l6;
            if (l6 >= 60) {
                const uint32_t extra = l6 - 59;
                hdr += extra;
                if (hdr > e - r) return kStop;
                n = 0;
                for (uint32_t i = 0; i < extra; ++i)
                    n |= static_cast<uint32_t>(win[(gb + r + 1 + i) & (kIn - 1)]) << (8 * i);
                if (n >= e) return kStop;  // also keeps n + 1 from wrapping
            }
            n += 1;
            const uint32_t q = r + hdr;
            if (n > e - q) return kStop;
            *len = n;
            return q + n;
        }
        const uint32_t hdr = kind == 1 ? 2 : (kind == 2 ? 3 : 5);
        if (hdr > e - r) return kStop;
        *len = kind == 1 ? 4 + ((tag >> 2) & 7) : (tag >> 2) + 1;
        return r + hdr;
    }

};

// ---------------------------------------------------------------------------
// 16-byte windows. A window is 4 little-endian words holding bytes
// [a, a + 16); only the first m are meaningful.

// Bytes [mis, mis + 16) of the 32-byte pair (lo, hi).
__device__ __forceinline__ uint4 shift32(uint4 lo, uint4 hi, uint32_t mis) {
    const uint32_t k = mis >> 2, r = (mis & 3) * 8;
    uint32_t w0, w1, w2, w3, w4;
    if (k == 0) {
        w0 = lo.x; w1 = lo.y; w2 = lo.z; w3 = lo.w; w4 = hi.x;
    } else if (k == 1) {
        w0 = lo.y; w1 = lo.z; w2 = lo.w; w3 = hi.x; w4 = hi.y;
    } else if (k == 2) {
        w0 = lo.z; w1 = lo.w; w2 = hi.x; w3 = hi.y; w4 = hi.z;
    } else {
        w0 = lo.w; w1 = hi.x; w2 = hi.y; w3 = hi.z; w4 = hi.w;
    }
    return make_uint4(__funnelshift_r(w0, w1, r), __funnelshift_r(w1, w2, r),
                      __funnelshift_r(w2, w3, r), __funnelshift_r(w3, w4, r));
}

// m (1..16) input bytes at p (read-only for the kernel). The second aligned
// block is read only when the m bytes reach into it, so no load touches an
// aligned block without a requested byte in it.
__device__ __forceinline__ uint4 ld16_input(const uint8_t* p, uint32_t m) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t mis = a & 15;
    const uint4* b = reinterpret_cast<const uint4*>(a - mis);
    const uint4 lo = __ldg(b);
    const uint4 hi = mis + m > 16 ? __ldg(b + 1) : make_uint4(0, 0, 0, 0);
    return shift32(lo, hi, mis);
}

// m output bytes at p, written earlier by this warp (coherent loads).
__device__ __forceinline__ uint4 ld16_output(const uint8_t* p, uint32_t m) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t mis = a & 15;
    const uint4* b = reinterpret_cast<const uint4*>(a - mis);
    const uint4 lo = b[0];
    const uint4 hi = mis + m > 16 ? b[1] : make_uint4(0, 0, 0, 0);
    return shift32(lo, hi, mis);
}

// m (1..16) output bytes at p, read as the aligned words that hold them
// (no word past the last wanted byte is touched) joined by funnel shifts.
__device__ __forceinline__ uint4 ld16_words(const uint8_t* p, uint32_t m) {
    const uintptr_t ad = reinterpret_cast<uintptr_t>(p);
    const uint32_t s4 = static_cast<uint32_t>(ad & 3), sh = 8 * s4;
    const uint32_t* q = reinterpret_cast<const uint32_t*>(ad - s4);
    const uint32_t lw = (s4 + m - 1) >> 2;  // last word holding a wanted byte, 0..4
    const uint32_t w0 = q[0];
    const uint32_t w1 = lw >= 1 ? q[1] : 0u, w2 = lw >= 2 ? q[2] : 0u;
    const uint32_t w3 = lw >= 3 ? q[3] : 0u, w4 = lw >= 4 ? q[4] : 0u;
    return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                      __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
}

// Per-warp output state. Positions are byte offsets into the chunk's output.
struct Out {
    uint8_t* ring;     // kRing bytes of shared memory
    uint8_t* dst;      // destination
    uintptr_t dbase;   // destination address (ring index = (dbase + pos) mod kRing)
    uint64_t vlo;      // positions >= vlo are held by the ring
    uint64_t flushed;  // positions < flushed are in the destination

    __device__ __forceinline__ uint32_t idx(uint64_t pos) const {
        return static_cast<uint32_t>((dbase + pos) & (kRing - 1));
    }

    // 16 ring bytes at position a: the five aligned words they touch, joined
    // by funnel shifts.
    __device__ __forceinline__ uint4 ring16(uint64_t a) const {
        constexpr uint32_t kMask = kRing / 4 - 1;
        const uint32_t ia = idx(a);
        const uint32_t wi = ia >> 2, sh = (ia & 3) * 8;
        const uint32_t* r32 = reinterpret_cast<const uint32_t*>(ring);
        const uint32_t w0 = r32[wi], w1 = r32[(wi + 1) & kMask], w2 = r32[(wi + 2) & kMask];
        const uint32_t w3 = r32[(wi + 3) & kMask], w4 = r32[(wi + 4) & kMask];
        return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                          __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
    }

    // m (1..16) already-written output bytes at position a. Outside the
    // ring, the destination holds them: vlo <= flushed always, and they are
    // equal only right after a token copied straight to the destination,
    // when a source may straddle vlo with its upper bytes in the ring alone.
    __device__ __forceinline__ uint4 fetch16(uint64_t a, uint32_t m) const {
        if (a >= vlo) return ring16(a);
        if (a + m <= flushed) return ld16_words(dst + a, m);
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (uint32_t j = 0; j < 16; ++j) {
            if (j < m) {
                const uint64_t x = a + j;
                const uint32_t b = x >= vlo ? ring[idx(x)] : dst[x];
                w[j >> 2] |= b << ((j & 3) * 8);
            }
        }
        return make_uint4(w[0], w[1], w[2], w[3]);
    }

    // Write the first m (1..16) bytes of v at output position x (ring). The
    // ring bytes of the current batch start at zero (clear()) and every byte
    // has one writer, so the bytes are OR-ed in as five aligned words;
    // neighbouring lanes may share the edge words.
    __device__ __forceinline__ void put16(uint64_t x, const uint4& v, uint32_t m) const {
        const uint32_t ix = idx(x);
        const uint32_t sb = ix & 3, sh = 8 * sb;
        // keep bytes [0, m): word j keeps its low 8 m - 32 j bits (0..32),
        // a right funnel shift of ones by the rest (clamped at 32)
        const uint32_t bits = 8 * m;
        const uint32_t w0 = v.x & __funnelshift_rc(~0u, 0u, bits >= 32 ? 0u : 32u - bits);
        const uint32_t w1 = v.y & __funnelshift_rc(~0u, 0u, bits >= 64 ? 0u : 64u - bits);
        const uint32_t w2 = v.z & __funnelshift_rc(~0u, 0u, bits >= 96 ? 0u : 96u - bits);
        const uint32_t w3 = v.w & __funnelshift_rc(~0u, 0u, 128u - bits);
        // all five words: past the last byte they are zero, and OR-ing zero
        // leaves a word as it is
        uint32_t* r32 = reinterpret_cast<uint32_t*>(ring);
        constexpr uint32_t kMask = kRing / 4 - 1;
        const uint32_t wi = ix >> 2;
        atomicOr(r32 + wi, w0 << sh);
        atomicOr(r32 + ((wi + 1) & kMask), __funnelshift_l(w0, w1, sh));
        atomicOr(r32 + ((wi + 2) & kMask), __funnelshift_l(w1, w2, sh));
        atomicOr(r32 + ((wi + 3) & kMask), __funnelshift_l(w2, w3, sh));
        atomicOr(r32 + ((wi + 4) & kMask), __funnelshift_l(w3, 0u, sh));
    }

    // Zero the ring bytes of output positions [b, e) (e - b <= kRing - 32)
    // before a batch ORs its bytes in. Bytes below b in the first word keep
    // their contents; the rest of that word's 16-byte block is cleared word
    // by word, then whole 16-byte blocks through the one holding e - 1, so
    // up to 15 bytes past e may be cleared too (they belong to later output,
    // whose batch clears them again). The caller keeps vlo above every
    // position whose slot this clears.
    __device__ __forceinline__ void clear(uint64_t b, uint64_t e, uint32_t lane) const {
        if (e <= b) return;
        uint32_t* r32 = reinterpret_cast<uint32_t*>(ring);
        const uint32_t ib = idx(b);
        const uint32_t sb = ib & 3;
        const uint32_t w0 = ib >> 2;
        if (lane == 0) atomicAnd(r32 + w0, (1u << (8 * sb)) - 1);
        if (lane >= 1 && lane < 4 - (w0 & 3)) r32[w0 + lane] = 0;  // same block: no wrap
        const uint32_t end = ib + static_cast<uint32_t>(e - b);     // unwrapped ring index
        for (uint32_t x = (ib & ~15u) + 16 + 16 * lane; x < end; x += 512)
            *reinterpret_cast<uint4*>(ring + (x & (kRing - 1))) = make_uint4(0, 0, 0, 0);
        __syncwarp();
    }

    // Copy positions [flushed, end) that are ready to the destination: the
    // head up to the first aligned boundary and, when `final`, the tail by
    // byte stores; whole aligned 16-byte blocks by coalesced vector stores.
    __device__ __forceinline__ void flush(uint64_t end, bool final, uint32_t lane) {
        const uint64_t f = flushed;
        if (end <= f) return;
        // in addresses: the first aligned boundary at or after f, the last at
        // or before end (the latter may lie below the former when [f, end)
        // sits inside one partial block)
        const uintptr_t fa_abs = (dbase + f + 15) & ~static_cast<uintptr_t>(15);
        const uintptr_t ea_abs = (dbase + end) & ~static_cast<uintptr_t>(15);
        const uint64_t hend = (fa_abs < dbase + end ? fa_abs : dbase + end) - dbase;
        if (f + lane < hend) dst[f + lane] = ring[idx(f + lane)];
        uint64_t nf = hend;
        if (ea_abs > fa_abs) {
            const uint64_t fa = fa_abs - dbase, ea = ea_abs - dbase;
            for (uint64_t b = fa + 16ull * lane; b < ea; b += 16ull * 32)
                *reinterpret_cast<uint4*>(dst + b) = *reinterpret_cast<const uint4*>(ring + idx(b));
            nf = ea;
        }
        if (final && nf < end) {
            if (nf + lane < end) dst[nf + lane] = ring[idx(nf + lane)];
            nf = end;
        }
        flushed = nf;
        __syncwarp();
    }
};

// m (1..16) input bytes at position a, from the window when all of them
// are there.
__device__ __forceinline__ uint4 in16(const In& in, uint64_t a, uint32_t m) {
    if (in.held(a, m)) {
        // the five aligned window words the 16 bytes touch, joined by
        // funnel shifts
        constexpr uint32_t kMask = kIn / 4 - 1;
        const uint32_t ia = static_cast<uint32_t>((in.gbase + a) & (kIn - 1));
        const uint32_t wi = ia >> 2, sh = (ia & 3) * 8;
        const uint32_t* w32 = reinterpret_cast<const uint32_t*>(in.win);
        const uint32_t w0 = w32[wi], w1 = w32[(wi + 1) & kMask], w2 = w32[(wi + 2) & kMask];
        const uint32_t w3 = w32[(wi + 3) & kMask], w4 = w32[(wi + 4) & kMask];
        return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                          __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
    }
    return ld16_input(in.g + a, m);
}

// Copy n input bytes from position src to output position o.
__device__ __forceinline__ void copy_literal(const Out& out, const In& in, uint64_t src,
                                             uint64_t o, uint32_t n) {
    for (uint32_t k = 0; k < n; k += 16) {
        const uint32_t m = n - k < 16 ? n - k : 16u;
        out.put16(o + k, in16(in, src + k, m), m);
    }
}

// Output [o, o + n) = the match with offset off (out[x] = out[x - off]);
// every source byte below o is already written.
// A match at distance off < 16 starts from its period alone: the low off
// bytes of v. period16 returns the match's first 16 bytes, expanded in
// registers without branches and computed in every lane. A lane with
// off >= 16 gets v back. Periods up to 8 bytes are doubled in 64 bits, and
// the next 8 bytes start r = 8 mod off bytes into the period, so byte j of
// them is byte j + r of the first 8 (j < 8 - r) or byte j + r - off. For
// 9..15 bytes, the first 16 - off bytes repeat once. Every later byte of the
// match repeats the one rest_distance(off) = off * ceil(16 / off) (16..30)
// bytes back, which is written by then, so the rest of the match is a plain
// copy at that distance.
__device__ __forceinline__ uint4 period16(const uint4& v, uint32_t off) {
    const uint64_t lo = (static_cast<uint64_t>(v.y) << 32) | v.x;
    const uint64_t hi = (static_cast<uint64_t>(v.w) << 32) | v.z;
    const uint32_t d = off < 16 ? off : 16u;
    const uint32_t s = 8 * d;  // 8..128
    uint64_t plo = lo & (~0ull >> ((64 - s) & 63));
    plo |= s < 64 ? plo << (s & 63) : 0ull;
    plo |= s < 32 ? plo << ((2 * s) & 63) : 0ull;
    plo |= s < 16 ? plo << ((4 * s) & 63) : 0ull;
    // 8 mod d for d = 1..8, one nibble each
    const uint32_t r = static_cast<uint32_t>((0x012302000ull >> ((4 * d) & 63)) & 15);
    const uint64_t phi = (plo >> ((8 * r) & 63)) | (plo << ((8 * (d - r)) & 63));
    const uint32_t s2 = (s - 64) & 63;
    const uint64_t qhi = (hi & ((1ull << s2) - 1)) | (lo << s2);
    const bool small = d <= 8;
    const uint64_t olo = small ? plo : lo, ohi = small ? phi : qhi;
    const uint4 e = make_uint4(static_cast<uint32_t>(olo), static_cast<uint32_t>(olo >> 32),
                               static_cast<uint32_t>(ohi), static_cast<uint32_t>(ohi >> 32));
    return off < 16 ? e : v;
}

__device__ __forceinline__ uint32_t rest_distance(uint32_t off) {
    // Q - 16 for off = 1..15, one nibble each
    return off < 16 ? 16 + static_cast<uint32_t>((0xECA8642052402000ull >> (4 * (off & 15))) & 15)
                    : off;
}

// Lane-parallel match copy through the ring: the first piece is one fetch
// and one write in every lane (period16), the rest a plain copy at
// rest_distance(off).
__device__ __forceinline__ void copy_match(const Out& out, uint64_t o, uint32_t n, uint32_t off) {
    const uint32_t m0 = n < 16 ? n : 16u;
    out.put16(o, period16(out.fetch16(o - off, off < 16 ? off : m0), off), m0);
    const uint32_t d = rest_distance(off);
    for (uint32_t k = 16; k < n; k += 16) {
        const uint32_t m = n - k < 16 ? n - k : 16u;
        out.put16(o + k, out.fetch16(o + k - d, m), m);
    }
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        const uint64_t o = __shfl_xor_sync(kFull, v, s);
        v = o < v ? o : v;
    }
    return v;
}

// Input window filler: aligned 16-byte blocks of the chunk, by cp.async.
// Only blocks holding at least one byte of [0, S) are read, so no load leaves
// the 16-byte blocks the chunk itself occupies.
struct Filler {
    const uint8_t* g;
    uint8_t* win;
    uintptr_t gbase;
    uint64_t S;
    int64_t next;   // chunk-relative start of the next block to fetch
    int64_t first;  // blocks [first, next) are fetched or in flight

    // Issue fetches for the blocks from position `from` up to `until`
    // (exclusive); blocks before `from` that were never fetched are skipped.
    __device__ __forceinline__ void issue(uint64_t from, uint64_t until, uint32_t lane) {
        if (S == 0) return;
        const int64_t lim = static_cast<int64_t>(until < S ? until : S);
        if (next < static_cast<int64_t>(from)) {
            next = static_cast<int64_t>(from) - static_cast<int64_t>((gbase + from) & 15);
            first = next;
        }
        if (next >= lim) return;
        for (int64_t b = next + 16 * static_cast<int64_t>(lane); b < lim; b += 16 * 32) {
            const uint8_t* src = g + b;  // 16-byte aligned by construction
            uint8_t* dst = win + ((gbase + b) & (kIn - 1));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)),
                         "l"(src)
                         : "memory");
        }
        next += ((lim - next + 15) / 16) * 16;
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    // Lowest position that is fetched and whose slot no fetch issued so far
    // overwrites.
    __device__ __forceinline__ uint64_t low() const {
        int64_t r = next - static_cast<int64_t>(kIn);
        if (r < first) r = first;
        return r > 0 ? static_cast<uint64_t>(r) : 0;
    }
    // Wait for everything issued; afterwards positions below the returned
    // bound (and at or above low()) are in the window.
    __device__ __forceinline__ uint64_t land() const {
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        const int64_t r = next < static_cast<int64_t>(S) ? next : static_cast<int64_t>(S);
        return r > 0 ? static_cast<uint64_t>(r) : 0;
    }
};

// ---------------------------------------------------------------------------
// The group walk: the next (up to) 32 tokens of the chain from a known
// token, every lane taking the same steps. Each lane takes the format's
// branch-free step at two of the next 64 positions (r + lane, r + 32 +
// lane); the chain through them is followed by shuffles, kHops hops per
// branch. A token whose step is not the simple one goes through the general
// step; a chain that leaves the 64 positions starts the next 64 at its
// token. Lane k gets the k-th token's position and output offset, both
// relative to the group's first token; cnt is the number of tokens found
// (at least one). It reads only the landed window: gb is the window slot of
// the first token, e the readable bound relative to it (0 when the first
// token is not in the window: lane 0 then holds it alone and the exact
// ladder decides it). Out of line, so that the copy code of the group is
// compiled as if the walk were not there.
struct Walk {
    uint32_t myr, myo, cnt;
};

template <class F>
__device__ __noinline__ Walk walk_group(const uint8_t* win, uint32_t gb, uint32_t e, uint64_t p,
                                        uint64_t S, uint32_t lane) {
    uint32_t od = 0, myo = 0, r = 0, myr = 0, cnt = 0;
    if (e == 0) return Walk{0, 0, 1};
    for (;;) {
        uint32_t n0, l0, n1, l1;
        const bool k0 = F::step_simple(win, gb, e, r + lane, &n0, &l0);
        const bool k1 = F::step_simple(win, gb, e, r + 32 + lane, &n1, &l1);
        // packed per position: next token relative to r (below 512) |
        // output length << 16 (below 2^10), or kWordStop for the general step
        const uint32_t pk0 = k0 ? (n0 - r) | (l0 << 16) : kWordStop;
        const uint32_t pk1 = k1 ? (n1 - r) | (l1 << 16) : kWordStop;
        uint32_t cur = 0, prev = 0;
        bool alive = true;
        while (alive) {
#pragma unroll
            for (uint32_t u = 0; u < kHops; ++u) {
                // The previous token's word is the next shuffle's index (the
                // source lane is taken modulo 32, and the word's low bits are
                // the next position); both halves are read and bit 5 picks
                // one, so a hop's dependent path is one shuffle and a select.
                // After the chain stops, the reads are masked by alive.
                const uint32_t a = __shfl_sync(kFull, pk0, prev);
                const uint32_t b = __shfl_sync(kFull, pk1, prev);
                const uint32_t pk = (prev & 32) ? b : a;
                const bool take = alive & (pk != kWordStop);
                if (take & (lane == cnt)) {
                    myr = r + cur;
                    myo = od;
                }
                const uint32_t nx = pk & 0xffffu;
                cnt += take ? 1u : 0u;
                od += take ? pk >> 16 : 0u;
                alive = take & (cnt < 32) & (nx < 64);
                cur = take ? nx : cur;
                prev = pk;
            }
        }
        r += cur;
        if (cnt >= 32) break;
        if (cur >= 64) continue;  // the chain left the 64 positions at a token
        // the token at r needs the general step
        if (lane == cnt) {
            myr = r;
            myo = od;
        }
        ++cnt;
        if (cnt >= 32 || r >= e) break;
        uint32_t len = 0;
        const uint32_t nr = F::walk(win, gb, e, r, &len);
        if (nr == kStop || F::at_end(p + nr, S)) break;
        r = nr;
        od += len;
    }
    return Walk{myr, myo, cnt};
}

// Store m (1..16) bytes of v at global p (16-byte store when aligned and whole).
__device__ __forceinline__ void st16_global(uint8_t* p, const uint4& v, uint32_t m) {
    if (m == 16 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        *reinterpret_cast<uint4*>(p) = v;
        return;
    }
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (uint32_t j = 0; j < 16; ++j)
        if (j < m) p[j] = static_cast<uint8_t>(w[j >> 2] >> ((j & 3) * 8));
}

// The whole warp copies n input bytes at g + src to dst + o (no overlap):
// destination-aligned 16-byte stores, four in flight per lane.
__device__ __forceinline__ void coop_literal(uint8_t* dst, uint64_t o, const uint8_t* src, uint64_t n,
                             uint32_t lane) {
    uint8_t* D = dst + o;
    uint64_t head = (16 - (reinterpret_cast<uintptr_t>(D) & 15)) & 15;
    if (head > n) head = n;
    if (lane < head) D[lane] = __ldg(src + lane);
    const uint64_t body_end = head + ((n - head) & ~15ull);
    uint64_t k = head + 16ull * lane;
    for (; k + 3 * 512 < body_end; k += 4 * 512) {
        const uint4 v0 = ld16_input(src + k, 16), v1 = ld16_input(src + k + 512, 16);
        const uint4 v2 = ld16_input(src + k + 1024, 16), v3 = ld16_input(src + k + 1536, 16);
        *reinterpret_cast<uint4*>(D + k) = v0;
        *reinterpret_cast<uint4*>(D + k + 512) = v1;
        *reinterpret_cast<uint4*>(D + k + 1024) = v2;
        *reinterpret_cast<uint4*>(D + k + 1536) = v3;
    }
    for (; k < body_end; k += 512) *reinterpret_cast<uint4*>(D + k) = ld16_input(src + k, 16);
    if (body_end + lane < n) D[body_end + lane] = __ldg(src + body_end + lane);
}

// The whole warp writes the match dst[ms, ms + n) with offset off; every byte
// before ms is in dst. `scratch` (>= 512 bytes of shared memory, free) holds
// a short period.
__device__ __forceinline__ void coop_match(uint8_t* dst, uint64_t ms, uint64_t n, uint32_t off,
                           uint8_t* scratch, uint32_t lane) {
    uint8_t* D = dst + ms;
    uint64_t head = (16 - (reinterpret_cast<uintptr_t>(D) & 15)) & 15;
    if (head > n) head = n;
    const uint64_t body_end = head + ((n - head) & ~15ull);
    if (off >= 512) {
        // A wave of 32 x 16 bytes never reads its own output.
        if (lane < head) D[lane] = D[static_cast<int64_t>(lane) - off];
        __syncwarp();
        for (uint64_t w = head; w < body_end; w += 512) {
            const uint64_t k = w + 16ull * lane;
            if (k < body_end) {
                const uint4 v = ld16_output(D + k - off, 16);
                *reinterpret_cast<uint4*>(D + k) = v;
            }
            __syncwarp();
        }
        for (uint64_t k = body_end; k < n; ++k) {  // < 16 bytes, serial order
            if (lane == 0) D[k] = D[k - off];
            __syncwarp();
        }
        return;
    }
    // Period off < 512: stage it, then every byte is period[(x - ms) mod off].
    for (uint32_t j = lane; j < off; j += 32) scratch[j] = D[static_cast<int64_t>(j) - off];
    __syncwarp();
    if (lane < head) D[lane] = scratch[lane % off];
    for (uint64_t k = head + 16ull * lane; k < body_end; k += 512) {
        uint32_t ph = static_cast<uint32_t>(k % off);
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (uint32_t j = 0; j < 16; ++j) {
            w[j >> 2] |= static_cast<uint32_t>(scratch[ph]) << ((j & 3) * 8);
            ph = ph + 1 == off ? 0 : ph + 1;
        }
        *reinterpret_cast<uint4*>(D + k) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    if (body_end + lane < n) D[body_end + lane] = scratch[(body_end + lane) % off];
    __syncwarp();
}

// Lane-parallel execution of tokens whose output fits one ring batch: each
// active lane (lanes first.. of the group) holds one token (literal li bytes
// from input lsrc to o, then a match of mi bytes at offset off); the batch's
// output is [bstart, bend).
__device__ __forceinline__ void exec_small(Out& out, const In& in, bool act, uint64_t o,
                                           uint64_t li, uint64_t lsrc, uint64_t mi,
                                           uint32_t off, uint64_t bstart, uint64_t bend,
                                           uint32_t first, uint32_t lane) {
    // clear() may zero up to 15 bytes past bend, whose slots held positions
    // up to bend + 15 - kRing: those are read back from the destination.
    if (bend + 16 > out.vlo + kRing) out.vlo = bend + 16 - kRing;
    LZW_T(t_clear);
    out.clear(bstart, bend, lane);
    LZW_ADD(4, t_clear);
    LZW_T(t_lit);
    const uint64_t ms = o + li;
    if (act && li) copy_literal(out, in, lsrc, o, static_cast<uint32_t>(li));
    __syncwarp();
    LZW_ADD(6, t_lit);
    LZW_T(t_rounds);
    // Matches in rounds: a match copies once no unfinished match's output
    // overlaps the bytes its source reads in this batch ([rs, re), relative
    // to bstart; everything before bstart and every literal is written).
    // Match starts grow with the lane, so the unfinished matches starting
    // below re are the pending lanes among a prefix of lanes; the last of
    // them ending by rs clears the source (the earlier ones end before it).
    // The lowest unfinished match always clears, so every round finishes at
    // least one.
    // sorted by lane: tokens of earlier batches first, unused lanes last
    const uint32_t rms = act ? static_cast<uint32_t>(ms - bstart) : (lane < first ? 0u : ~0u);
    bool pend = act && mi != 0;
    uint32_t rs = 0, re = 0;
    if (pend) {
        const uint64_t s0 = ms - off;
        const uint64_t e0 = s0 + mi < ms ? s0 + mi : ms;
        rs = s0 > bstart ? static_cast<uint32_t>(s0 - bstart) : 0u;
        re = e0 > bstart ? static_cast<uint32_t>(e0 - bstart) : 0u;
    }
    while (__any_sync(kFull, pend)) {
        const unsigned pm = __ballot_sync(kFull, pend);
        const uint32_t rme = rms + static_cast<uint32_t>(mi);  // read only for pending lanes
        uint32_t l = 0;  // the last lane whose match starts below re
#pragma unroll
        for (uint32_t st = 16; st; st >>= 1) {
            const uint32_t c = l + st;
            if (__shfl_sync(kFull, rms, c) < re) l = c;
        }
        const bool below = __shfl_sync(kFull, rms, 0) < re;
        const unsigned cand = below ? pm & (l == 31 ? kFull : ((2u << l) - 1)) : 0u;
        const uint32_t last = cand ? 31 - __clz(cand) : 0u;
        const uint32_t last_end = __shfl_sync(kFull, rme, last);
        const bool ready = pend && (re <= rs || cand == 0 || last_end <= rs);
        if (ready) copy_match(out, ms, static_cast<uint32_t>(mi), off);
        __syncwarp();
        pend = pend && !ready;
        LZW_EV(2, 1);
    }
    LZW_ADD(7, t_rounds);
    out.flush(bend, false, lane);
}

// One token of a group as a lane holds it: literal run li bytes from input
// position lsrc to output position o, then a match of mi bytes at offset off.
struct Tok {
    uint64_t o, li, lsrc, mi;
    uint32_t off;
};

// Executes checked groups of tokens: tokens of at most kBig bytes lane-
// parallel through the output ring (batches of up to tn.batch bytes), longer
// ones by the whole warp straight to the destination. Literal bytes come
// from the input window when `in` holds them, else from global memory.
struct ExecSink {
    Out out;
    const uint8_t* g;
    uint8_t* dst;
    const In* in;
    Tune tn;
    uint32_t lane;

    __device__ __forceinline__ void group(const Tok& t, uint32_t m) {
        const bool act = lane < m;
        const uint64_t tend = t.o + t.li + t.mi;
        const bool big = act && t.li + t.mi > kBig;
        uint32_t s0 = 0;
        while (s0 < m) {
            const uint64_t os = __shfl_sync(kFull, t.o, s0);
            const unsigned cut =
                __ballot_sync(kFull, act && lane >= s0 && (big || tend - os > tn.batch));
            const uint32_t e = cut ? __ffs(cut) - 1 : m;
            if (e == s0) {
                const uint64_t bo = os;
                const uint64_t bli = __shfl_sync(kFull, t.li, s0);
                const uint64_t bls = __shfl_sync(kFull, t.lsrc, s0);
                const uint64_t bmi = __shfl_sync(kFull, t.mi, s0);
                const uint32_t boff = __shfl_sync(kFull, t.off, s0);
                out.flush(bo, true, lane);
                if (bli) coop_literal(dst, bo, g + bls, bli, lane);
                __syncwarp();
                if (bmi) coop_match(dst, bo + bli, bmi, boff, out.ring, lane);
                __syncwarp();
                out.flushed = out.vlo = bo + bli + bmi;
                LZW_EV(3, 1);
                ++s0;
                continue;
            }
            const uint64_t bend = __shfl_sync(kFull, tend, e - 1);
            exec_small(out, *in, act && lane >= s0 && lane < e, t.o, t.li, t.lsrc, t.mi, t.off,
                       os, bend, s0, lane);
            s0 = e;
        }
    }
    __device__ __forceinline__ void finish(uint64_t d) { out.flush(d, true, lane); }
};

// Parses one chunk (window tables, hop composition, the exact ladder per
// token) and hands every checked group of up to 32 tokens to the sink in
// chain order: sink.group(tok, m, last, dend) returns false to abandon the
// chunk. Returns the chunk's status; *dend is the output length on success.
template <class F, class Sink>
__device__ __forceinline__ int parse_chunk(const uint8_t* g, uint64_t S, uint64_t cap,
                                           uint8_t* win, const Tune& tn, uint32_t lane,
                                           Sink& sink, In& in, uint64_t* dend_out) {
    *dend_out = 0;
    uint64_t p, limit;
    int status = F::begin(GBytes{g}, S, cap, &p, &limit);
    if (status != CUDEC_OK) return status;

    const uintptr_t gbase = reinterpret_cast<uintptr_t>(g);
    Filler fill{g, win, gbase, S, -static_cast<int64_t>(gbase & 15),
                -static_cast<int64_t>(gbase & 15)};
    in = In{g, win, gbase, 0, 0};
    fill.issue(p, p + tn.ahead, lane);
    uint64_t d = 0;  // output position of the next token
    LZW_T(t_chunk);
    uint64_t refill_at = 0;
    // Fuel: every token consumes at least one source byte, so a chunk of S
    // bytes holds at most S + 1 tokens (saturating at the top of the range).
    // No input reaches the cap; it turns a parser fault into a rejected
    // chunk instead of a warp that never leaves this loop (the reference's
    // cap, src/lz4_decode.cuh:99,152). m is warp-uniform, so the test is too.
    uint64_t fuel = S == ~0ull ? ~0ull : S + 1;
    for (;;) {
        LZW_T(t_land);
        if (p >= refill_at) {
            uint64_t ready = fill.land();
            // Refill ahead of the parse; it overwrites only positions before
            // p - 64, and those leave the window's valid range.
            fill.issue(p, p + tn.ahead, lane);
            in.lo = fill.low();
            const uint64_t want = S - p < tn.pw ? S : p + tn.pw;
            if (ready < want) ready = fill.land();  // the parse jumped past the window
            in.span = ready > in.lo ? ready - in.lo : 0;
            refill_at = p + kRefill;
        }
        LZW_ADD(0, t_land);
        if (F::at_end(p, S)) {
            status = F::finish(d, limit);
            if (status == CUDEC_OK && !sink.group(Tok{}, 0, true, d)) status = CUDEC_ERR_CUDA;
            break;
        }
        // ---- the next (up to) 32 tokens of the chain
        LZW_T(t_walk);
        const uint64_t wend = in.lo + in.span < S ? in.lo + in.span : S;
        const uint32_t e = (p >= in.lo && p < wend) ? static_cast<uint32_t>(wend - p) : 0;
        const Walk wk = walk_group<F>(win, static_cast<uint32_t>(gbase + p), e, p, S, lane);
        LZW_ADD(1, t_walk);
        LZW_T(t_grp);
        // ---- each lane checks its token exactly; the first failing or
        // terminal token decides the chunk as the serial parser would
        const bool valid = lane < wk.cnt;
        const uint64_t x = p + wk.myr;
        const uint64_t dl = d + wk.myo;
        Seq sq{};
        int st = CUDEC_OK;
        if (valid) st = F::parse(in, S, limit, x, dl, &sq);
        uint32_t m = wk.cnt;
        bool last = false;
        const unsigned ev = __ballot_sync(kFull, valid && (st != CUDEC_OK || sq.done));
        if (ev) {
            const int k = __ffs(ev) - 1;
            const int se = __shfl_sync(kFull, st, k);
            if (se != CUDEC_OK) {
                status = se;
                break;
            }
            m = k + 1;
            last = true;
        }
        if (m > fuel) {
            status = CUDEC_ERR_CORRUPT_INPUT;
            break;
        }
        fuel -= m;
        const uint64_t tend = dl + sq.lit + sq.ml;
        const uint64_t nxt = __shfl_sync(kFull, sq.next, m - 1);
        const uint64_t dend = __shfl_sync(kFull, tend, m - 1);
        LZW_ADD(2, t_grp);
        LZW_EV(0, 1);
        LZW_EV(1, m);
        LZW_T(t_exec);
        if (!sink.group(Tok{dl, sq.lit, sq.lit_src, sq.ml, sq.off}, m, last, dend)) {
            status = CUDEC_ERR_CUDA;
            break;
        }
        d = dend;
        LZW_ADD(3, t_exec);
        if (last) break;
        p = nxt;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    LZW_ADD(5, t_chunk);
    if (status != CUDEC_OK) return status;
    *dend_out = d;
    return CUDEC_OK;
}

// The single-warp sink: execute each group as soon as it is checked.
struct DirectSink {
    ExecSink* ex;
    __device__ __forceinline__ bool group(const Tok& t, uint32_t m, bool, uint64_t) {
        ex->group(t, m);
        return true;
    }
};

// Decode one chunk with the calling warp. Returns the status; *written is
// the output length on success.
template <class F>
__device__ __forceinline__ int decode_chunk(const uint8_t* g, uint64_t S, uint8_t* dst, uint64_t cap,
                            uint8_t* ring, uint8_t* win, const Tune& tn,
                            uint32_t lane, uint64_t* written) {
    *written = 0;
    In in{g, win, reinterpret_cast<uintptr_t>(g), 0, 0};
    ExecSink ex{Out{ring, dst, reinterpret_cast<uintptr_t>(dst), 0, 0}, g, dst, &in, tn, lane};
    DirectSink sink{&ex};
    uint64_t d = 0;
    const int st = parse_chunk<F>(g, S, cap, win, tn, lane, sink, in, &d);
    if (st != CUDEC_OK) return st;
    ex.finish(d);
    *written = d;
    return CUDEC_OK;
}

template <class F>
__global__ void __launch_bounds__(kThreads, 2)
    lz_warp_kernel(const void* const* src_ptrs, const size_t* src_sizes, void* const* dst_ptrs,
                   const size_t* dst_caps, size_t n, cudec_chunk_result* results, Tune tn) {
    extern __shared__ __align__(16) uint8_t lzw_smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t* base = lzw_smem + warp * kWarpSmem;
    uint8_t* ring = base;
    uint8_t* win = base + kRing;
    const size_t total = static_cast<size_t>(gridDim.x) * kWarps;
    for (size_t c = static_cast<size_t>(blockIdx.x) * kWarps + warp; c < n; c += total) {
        uint64_t written = 0;
        const int st = decode_chunk<F>(static_cast<const uint8_t*>(src_ptrs[c]), src_sizes[c],
                                       static_cast<uint8_t*>(dst_ptrs[c]), dst_caps[c], ring,
                                       win, tn, lane, &written);
        if (lane == 0) {
            results[c].status = st;
            results[c].reserved = 0;
            results[c].bytes_written = st == CUDEC_OK ? written : 0;
        }
        __syncwarp();
    }
}

}  // namespace lzw
}  // namespace cdb
