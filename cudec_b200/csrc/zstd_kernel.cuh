// Zstd frame decode on sm_100a: one warp per frame, warps independent.
//
// Semantics follow the reference's v1 subset and reject ladder
// (iderex/cudec src/zstd_frame.h:196-409, src/zstd_bitstream.h:481-638,
// src/zstd_fse.h:259-676, src/zstd_huf.h:198-460, src/zstd_literals.h:211-547,
// src/zstd_seq.h:320-676, src/zstd_repcode.h:98-184) and the status mapping
// of its frame driver (tests/zstd_twin_driver.h:178-390): a literal, table,
// sequence, repeat-offset or window fault is CUDEC_ERR_CORRUPT_INPUT; the
// declared content size above the capacity, or output past it, is
// CUDEC_ERR_OUTPUT_TOO_SMALL; skippable frames, dictionary ids, frames
// without a content size and windows above 8 MB are CUDEC_ERR_UNSUPPORTED.
//
// Data path per frame (all lanes run the serial parts redundantly, so every
// branch is warp-uniform and no broadcast is needed):
//  * tables live in the warp's shared memory: Huffman (2^11 cells), the three
//    sequence FSE tables (512/256/512 cells), kept across blocks for the
//    treeless and repeat modes;
//  * Huffman literals decode with one lane per stream (4 streams -> 4 lanes)
//    into the warp's slot of the caller's workspace; raw literals are read in
//    place, RLE literals are a byte;
//  * sequences decode 32 at a time (the FSE state chain is serial), each lane
//    keeping one, every sequence's fields taken from one 64-bit window of the
//    bitstream at its absolute position (BitWin); positions and the
//    reference's execution checks then run lane-parallel per batch, and the
//    32 sequences execute lane-parallel: literal copies first, then match
//    copies in rounds, a match running once no unfinished match's output
//    overlaps its source;
//  * the table descriptions and the first states are read with a checked
//    64-bit backward bit container (BitIn) with the reference's strictness: a
//    read of more bits than remain is a reject, a peek past the end reads
//    zeros; the windowed reads keep that strictness by testing the position
//    once per batch (it goes negative on an over-read).
#pragma once

#include <cstdint>

#include "cudec.h"

namespace cdb {
namespace zstd {

constexpr int kWarpsPerCta = 4;
constexpr int kCtaThreads = kWarpsPerCta * 32;
constexpr uint32_t kLitSlot = 128 * 1024;   // per-warp literal buffer (block maximum)
constexpr uint64_t kMaxWindow = 8ull << 20;
// Frame sequences (decode_frames): the largest window log libzstd's
// one-shot decoder takes (ZSTD_WINDOWLOG_MAX on 64-bit hosts). The window
// costs nothing here (matches read the destination), and offsets stay below
// 2^32 (an offset code is at most 31).
constexpr uint32_t kMaxWindowLogSeq = 31;

constexpr uint32_t kFseCells = 512;  // FSE decode cells per field (table log <= 9)

struct __align__(16) WarpSmem {
    uint16_t huf[1 << 11];   // symbol | bits << 8
    uint32_t fse[3][kFseCells];  // next << 16 | symbol << 8 | bits
    uint32_t wcells[64];     // Huffman-weight FSE table
    int16_t counts[64];
    uint16_t next[64];
    uint8_t weights[260];
    uint8_t period[512];     // a short match period staged for a warp copy
};

__device__ __forceinline__ unsigned hibit32(uint32_t v) { return 31u - __clz(v); }

__device__ __forceinline__ uint64_t rd_le(const uint8_t* p, unsigned n) {
    uint64_t v = 0;
    for (unsigned i = 0; i < n; ++i) v |= static_cast<uint64_t>(p[i]) << (8 * i);
    return v;
}

// Backward bit reader: bits are read from the last byte (below its marker
// bit) toward the first, most significant first.
struct BitIn {
    const uint8_t* src;
    int64_t pos;       // next byte to load (descending)
    uint64_t c;        // container, next bit at bit 63
    int32_t n;         // valid bits in c (negative once reads ran past the end)
    int64_t left;      // bits remaining in the stream (negative: over-read)

    // Tops the container up to at least 57 bits (or the stream's end). With
    // eight bytes behind the cursor it takes every whole byte that fits in
    // one step: the 8 bytes ending at pos, read as a little-endian word (byte
    // pos on top) from the two aligned 8-byte blocks that hold them - each
    // block holds a requested byte, so no load leaves the stream's blocks.
    __device__ __forceinline__ void refill() {
        if (n > 56 || pos < 0) return;
        if (pos >= 7) {
            const uint32_t b = static_cast<uint32_t>(64 - n) >> 3;  // 1..8 whole bytes fit
            const uintptr_t a = reinterpret_cast<uintptr_t>(src + pos - 7);
            const uint32_t mis = static_cast<uint32_t>(a & 7);
            const uint64_t* blk = reinterpret_cast<const uint64_t*>(a - mis);
            uint64_t x = blk[0];
            if (mis) x = (x >> (8 * mis)) | (blk[1] << (64 - 8 * mis));
            const uint64_t top = b == 8 ? x : (x >> (64 - 8 * b)) << (64 - 8 * b);
            c |= top >> n;
            n += 8 * b;
            pos -= b;
            return;
        }
        while (n <= 56 && pos >= 0) {
            c |= static_cast<uint64_t>(src[pos]) << (56 - n);
            n += 8;
            --pos;
        }
    }
    __device__ bool start(const uint8_t* s, uint64_t size) {
        src = s;
        if (size == 0) return false;
        const uint32_t last = s[size - 1];
        if (last == 0) return false;
        const uint32_t m = hibit32(last);
        left = static_cast<int64_t>((size - 1) * 8 + m);
        c = m ? (static_cast<uint64_t>(last & ((1u << m) - 1u)) << (64 - m)) : 0;
        n = static_cast<int32_t>(m);
        pos = static_cast<int64_t>(size) - 2;
        refill();
        return true;
    }
    // At least k (<= 57) bits buffered, or all that remain (bits past the
    // stream's end read as zeros).
    __device__ __forceinline__ void ensure(uint32_t k) {
        if (n < static_cast<int32_t>(k)) refill();
    }
    // The next k bits; needs ensure(k) first.
    __device__ __forceinline__ uint32_t peek(uint32_t k) const {
        return k ? static_cast<uint32_t>(c >> (64 - k)) : 0u;
    }
    // Strict: more bits than remain is a reject.
    __device__ __forceinline__ bool read(uint32_t k, uint64_t* v) {
        if (k == 0) {
            *v = 0;
            return true;
        }
        if (static_cast<int64_t>(k) > left) return false;
        ensure(k);
        *v = c >> (64 - k);
        c <<= k;
        n -= k;
        left -= k;
        return true;
    }
};

// Backward bitstream read by absolute position: bits [0, bp) of the stream
// (little-endian bit order, bit i = byte i/8 >> i%8) remain and the next
// bits are the highest, as BitIn reads them. window() returns the 64 bits
// below bp (bit 63 = stream bit bp - 1) as hi:lo, bits outside the stream
// reading as zeros; field() takes k (<= 31) of them counted from the top.
// No state but bp: a sequence's fields come from one window and bp drops by
// their total, with no refill and no per-read checks (bp < 0 is an
// over-read, tested by the caller).
struct BitWin {
    const uint8_t* s;
    int64_t size;
    const uint32_t* abase;  // s rounded down to a 4-byte boundary
    uint32_t boff;          // bit offset of s within that word

    __device__ __forceinline__ void init(const uint8_t* src, uint64_t n) {
        s = src;
        size = static_cast<int64_t>(n);
        abase = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(src) & ~uintptr_t{3});
        boff = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(src) & 3) * 8;
    }
    __device__ __forceinline__ void window(int32_t bp, uint32_t* hi, uint32_t* lo) const {
        if (bp >= 96) {
            // three aligned words hold the 64 bits; each holds a stream byte
            // (the third is read only when the bits reach into it)
            const uint32_t t = boff + static_cast<uint32_t>(bp) - 64;
            const uint32_t* p = abase + (t >> 5);
            const uint32_t sh = t & 31;
            const uint32_t w0 = __ldg(p), w1 = __ldg(p + 1);
            const uint32_t w2 = sh ? __ldg(p + 2) : 0u;
            *lo = __funnelshift_r(w0, w1, sh);
            *hi = __funnelshift_r(w1, w2, sh);
            return;
        }
        // near (or past) the stream's start: byte by byte
        const int64_t low = static_cast<int64_t>(bp) - 64;
        uint64_t x = 0;
        for (int64_t q = low >> 3; q <= (static_cast<int64_t>(bp) - 1) >> 3; ++q) {
            if (q < 0 || q >= size) continue;
            const int64_t at = 8 * q - low;  // byte q's bit 0 within the window, in (-8, 64)
            const uint64_t b = s[q];
            x |= at >= 0 ? b << at : b >> (-at);
        }
        *lo = static_cast<uint32_t>(x);
        *hi = static_cast<uint32_t>(x >> 32);
    }
    __device__ __forceinline__ static uint32_t field(uint32_t hi, uint32_t lo, uint32_t at,
                                                     uint32_t k) {
        const uint32_t t = at < 32 ? __funnelshift_lc(lo, hi, at) : __funnelshift_lc(0u, lo, at - 32);
        return __funnelshift_rc(t, 0u, 32 - k);
    }
};

// Forward little-endian bit reader for FSE descriptions.
struct DescIn {
    const uint8_t* src;
    uint64_t size, byte;
    uint32_t bit;
    __device__ bool avail(uint32_t k) const {
        return static_cast<uint64_t>((bit + k + 7) / 8) <= size - byte;
    }
    __device__ uint32_t peek(uint32_t k) const {
        uint32_t v = 0;
        uint64_t by = byte;
        uint32_t bi = bit;
        for (uint32_t i = 0; i < k; ++i) {
            const uint32_t t = by < size ? (src[by] >> bi) & 1u : 0u;
            v |= t << i;
            if (++bi == 8) {
                bi = 0;
                ++by;
            }
        }
        return v;
    }
    __device__ void adv(uint32_t k) {
        const uint32_t t = bit + k;
        byte += t / 8;
        bit = t % 8;
    }
};

// FSE description (src/zstd_fse.h ZstdFseReadNCount). Returns false on reject.
__device__ inline bool fse_ncount(const uint8_t* src, uint64_t size, unsigned max_sym,
                           unsigned max_log, int16_t* counts, unsigned* out_max,
                           unsigned* out_log, uint64_t* used) {
    if (size == 0) return false;
    const unsigned nsym = max_sym + 1;
    for (unsigned s = 0; s < nsym; ++s) counts[s] = 0;
    DescIn r{src, size, 0, 0};
    if (!r.avail(4)) return false;
    const unsigned log = r.peek(4) + 5;
    r.adv(4);
    if (log > max_log) return false;
    int32_t remaining = static_cast<int32_t>(1u << log) + 1;
    int32_t threshold = static_cast<int32_t>(1u << log);
    unsigned nbits = log + 1, sc = 0;
    bool prev0 = false;
    for (unsigned it = 0; it < nsym; ++it) {
        if (prev0) {
            bool open = true;
            for (unsigned step = 0; step < nsym && open; ++step) {
                if (!r.avail(2)) return false;
                const unsigned rep = r.peek(2);
                r.adv(2);
                sc += rep;
                if (rep != 3) open = false;
                if (sc >= nsym) return false;
            }
            if (open) return false;
            prev0 = false;
        }
        const int32_t small = (2 * threshold - 1) - remaining;
        const uint32_t pk = r.peek(nbits);
        const int32_t narrow = static_cast<int32_t>(pk & static_cast<uint32_t>(threshold - 1));
        int32_t prob;
        unsigned w;
        if (narrow < small) {
            prob = narrow;
            w = nbits - 1;
        } else {
            prob = static_cast<int32_t>(pk & static_cast<uint32_t>(2 * threshold - 1));
            if (prob >= threshold) prob -= small;
            w = nbits;
        }
        if (!r.avail(w)) return false;
        r.adv(w);
        --prob;
        remaining -= prob < 0 ? -prob : prob;
        counts[sc] = static_cast<int16_t>(prob);
        ++sc;
        prev0 = prob == 0;
        if (remaining < threshold) {
            if (remaining <= 1) break;
            nbits = hibit32(static_cast<uint32_t>(remaining)) + 1;
            threshold = static_cast<int32_t>(1u << (nbits - 1));
        }
        if (sc >= nsym) break;
    }
    if (remaining != 1) return false;
    *out_max = sc - 1;
    *out_log = log;
    *used = r.byte + (r.bit ? 1 : 0);
    return true;
}

// Table spread and cells (src/zstd_fse.h ZstdFseBuildDTable); all lanes run
// it redundantly, lane 0 writes.
__device__ inline bool fse_build(const int16_t* counts, unsigned max_sym, unsigned log,
                          uint32_t* cells, uint16_t* next, uint32_t lane) {
    const uint32_t size = 1u << log;
    uint32_t claimed = 0;
    for (unsigned s = 0; s <= max_sym; ++s) {
        const int16_t p = counts[s];
        if (p < -1) return false;
        const uint32_t m = p < 0 ? 1u : static_cast<uint32_t>(p);
        if (m > size - claimed) return false;
        claimed += m;
    }
    if (claimed != size) return false;
    __syncwarp();
    uint32_t high = size - 1;
    for (unsigned s = 0; s <= max_sym; ++s) {
        if (counts[s] < 0) {
            if (lane == 0) cells[high] = s << 8;
            --high;
            if (lane == 0) next[s] = 1;
        } else if (lane == 0) {
            next[s] = static_cast<uint16_t>(counts[s]);
        }
    }
    const uint32_t mask = size - 1, step = (size >> 1) + (size >> 3) + 3;
    uint32_t pos = 0;
    bool ok = true;
    for (unsigned s = 0; s <= max_sym && ok; ++s) {
        for (int16_t k = 0; k < counts[s]; ++k) {
            if (lane == 0) cells[pos] = s << 8;
            pos = (pos + step) & mask;
            uint32_t fuel = size;
            while (pos > high) {
                if (fuel == 0) {
                    ok = false;
                    break;
                }
                --fuel;
                pos = (pos + step) & mask;
            }
            if (!ok) break;
        }
    }
    __syncwarp();
    if (!ok) return false;
    if (lane == 0) {
        for (uint32_t cidx = 0; cidx < size; ++cidx) {
            const uint32_t s = (cells[cidx] >> 8) & 0xff;
            const uint32_t ns = next[s]++;
            const uint32_t b = log - hibit32(ns);
            cells[cidx] = (((ns << b) - size) << 16) | (s << 8) | b;
        }
    }
    __syncwarp();
    return true;
}

// Huffman weights (src/zstd_huf.h ZstdHufReadWeights, literals cap 11).
__device__ inline bool huf_weights(const uint8_t* src, uint64_t size, WarpSmem& w, uint32_t lane,
                            unsigned* count, unsigned* table_log, uint64_t* used) {
    if (size == 0) return false;
    const unsigned hdr = src[0];
    unsigned written = 0;
    uint8_t* wt = w.weights;
    if (hdr >= 128) {
        written = hdr - 127;
        const uint64_t pay = (written + 1u) / 2u;
        if (pay + 1 > size) return false;
        if (written + 1 > 256) return false;
        for (unsigned i = lane; i < written; i += 32) {
            const unsigned b = src[1 + i / 2];
            wt[i] = static_cast<uint8_t>((i % 2) == 0 ? (b >> 4) : (b & 15));
        }
        __syncwarp();
        *used = pay + 1;
    } else {
        const uint64_t pay = hdr;
        if (pay + 1 > size) return false;
        unsigned fmax, flog;
        uint64_t desc;
        if (!fse_ncount(src + 1, pay, 12, 6, w.counts, &fmax, &flog, &desc)) return false;
        if (!fse_build(w.counts, fmax, flog, w.wcells, w.next, lane)) return false;
        BitIn r;
        if (!r.start(src + 1 + desc, pay - desc)) return false;
        const uint32_t tsize = 1u << flog, cap = 255;
        uint64_t b;
        uint32_t st[2];
        if (!r.read(flog, &b)) return false;
        st[0] = static_cast<uint32_t>(b);
        if (!r.read(flog, &b)) return false;
        st[1] = static_cast<uint32_t>(b);
        uint32_t produced = 0;
        bool done = false;
        for (uint32_t stp = 0; stp < cap; ++stp) {
            uint32_t& act = st[stp & 1];
            const uint32_t oth = st[(stp + 1) & 1];
            if (act >= tsize) return false;
            const uint32_t cell = w.wcells[act];
            if (lane == 0) wt[produced] = static_cast<uint8_t>(cell >> 8);
            ++produced;
            const uint32_t nb = cell & 0xff;
            if (static_cast<int64_t>(nb) > r.left) {
                if (produced == cap) return false;
                if (oth >= tsize) return false;
                if (lane == 0) wt[produced] = static_cast<uint8_t>(w.wcells[oth] >> 8);
                ++produced;
                done = true;
                break;
            }
            if (!r.read(nb, &b)) return false;
            act = (cell >> 16) + static_cast<uint32_t>(b);
        }
        __syncwarp();
        if (!done) return false;
        written = produced;
        *used = pay + 1;
    }
    uint32_t total = 0;
    for (unsigned i = 0; i < written; ++i) {
        if (wt[i] > 11) return false;
        total += (1u << wt[i]) >> 1;
    }
    if (total == 0) return false;
    const unsigned tl = hibit32(total) + 1;
    if (tl > 11) return false;
    const uint32_t rest = (1u << tl) - total;
    const unsigned last = hibit32(rest) + 1;
    if ((1u << (last - 1)) != rest) return false;
    __syncwarp();
    if (lane == 0) wt[written] = static_cast<uint8_t>(last);
    __syncwarp();
    unsigned deep = 0;
    for (unsigned i = 0; i <= written; ++i) deep += wt[i] == 1;
    if (deep < 2) return false;
    *count = written + 1;
    *table_log = tl;
    return true;
}

// Decoding table from weights (src/zstd_huf.h ZstdHufBuildDTable): symbols in
// weight order, each weight-w symbol spans 2^(w-1) cells of tl+1-w bits.
__device__ inline bool huf_build(WarpSmem& w, unsigned count, unsigned tl, uint32_t lane) {
    const uint8_t* wt = w.weights;
    const uint32_t size = 1u << tl;
    uint32_t rc[13];
    for (int k = 0; k < 13; ++k) rc[k] = 0;
    uint32_t claimed = 0;
    for (unsigned i = 0; i < count; ++i) {
        if (wt[i] > tl) return false;
        ++rc[wt[i]];
        claimed += (1u << wt[i]) >> 1;
    }
    if (claimed != size) return false;
    uint32_t start[13];
    uint32_t nx = 0;
    start[0] = 0;
    for (unsigned k = 1; k <= tl; ++k) {
        start[k] = nx;
        nx += rc[k] * ((1u << k) >> 1);
    }
    for (unsigned k = tl + 1; k < 13; ++k) start[k] = nx;
    // Each symbol's first cell: start of its weight + spans of earlier
    // symbols of the same weight. Lanes take symbols round-robin; the
    // per-weight running offsets come from a serial prefix over symbols.
    for (unsigned s0 = 0; s0 < count; s0 += 32) {
        const unsigned s = s0 + lane;
        const unsigned k = s < count ? wt[s] : 0;
        // offset of s among same-weight symbols of this group
        uint32_t my_off = 0;
        for (unsigned j = 0; j < 32 && s0 + j < count; ++j) {
            const unsigned kj = wt[s0 + j];
            if (j < lane && kj == k) my_off += (1u << kj) >> 1;
        }
        if (s < count && k) {
            const uint32_t span = (1u << k) >> 1;
            const uint32_t at = start[k] + my_off;
            const uint16_t cell = static_cast<uint16_t>(s | ((tl + 1 - k) << 8));
            for (uint32_t j = 0; j < span; ++j) w.huf[at + j] = cell;
        }
        // advance every weight's start past this group's symbols
        for (unsigned j = 0; j < 32 && s0 + j < count; ++j) {
            const unsigned kj = wt[s0 + j];
            if (kj) start[kj] += (1u << kj) >> 1;
        }
    }
    __syncwarp();
    return true;
}

// One Huffman stream of `count` symbols; writes to dst when non-null.
__device__ inline bool huf_stream(const uint8_t* src, uint64_t size, const uint16_t* huf, unsigned tl,
                           uint8_t* dst, uint64_t count) {
    // Five symbols per 64-bit window read at the absolute bit position
    // (5 x 11 <= 55 bits, 11 the largest table log) and no per-symbol
    // checks: reads past the stream's start see zeros and drive bp
    // negative, and the stream is accepted only when exactly all its bits
    // were used, which is what per-symbol checks plus a final "all bits
    // used" check amount to.
    if (size == 0) return false;
    const uint32_t last = src[size - 1];
    if (last == 0) return false;  // no padding marker
    int32_t bp = static_cast<int32_t>((size - 1) * 8 + hibit32(last));  // size <= 128 KiB
    BitWin bw;
    bw.init(src, size);
    for (uint64_t i = 0; i < count; i += 5) {
        uint32_t hi, lo;
        bw.window(bp, &hi, &lo);
        uint32_t at = 0;
#pragma unroll
        for (uint32_t j = 0; j < 5; ++j) {
            if (i + j < count) {
                const uint16_t cell = huf[BitWin::field(hi, lo, at, tl)];
                at += cell >> 8;
                dst[i + j] = static_cast<uint8_t>(cell & 0xff);
            }
        }
        bp -= static_cast<int32_t>(at);
    }
    return bp == 0;
}

// Baseline | extra-bit count << 24 per code, one constant read per field.
static __constant__ uint32_t kLLCode[36] = {
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15,
    16 | 1u << 24, 18 | 1u << 24, 20 | 1u << 24, 22 | 1u << 24, 24 | 2u << 24, 28 | 2u << 24,
    32 | 3u << 24, 40 | 3u << 24, 48 | 4u << 24, 64 | 6u << 24, 128 | 7u << 24,
    256 | 8u << 24, 512 | 9u << 24, 1024 | 10u << 24, 2048 | 11u << 24, 4096 | 12u << 24,
    8192 | 13u << 24, 16384 | 14u << 24, 32768 | 15u << 24, 65536 | 16u << 24};
static __constant__ uint32_t kMLCode[53] = {
    3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18,
    19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34,
    35 | 1u << 24, 37 | 1u << 24, 39 | 1u << 24, 41 | 1u << 24, 43 | 2u << 24, 47 | 2u << 24,
    51 | 3u << 24, 59 | 3u << 24, 67 | 4u << 24, 83 | 4u << 24, 99 | 5u << 24,
    131 | 7u << 24, 259 | 8u << 24, 515 | 9u << 24, 1027 | 10u << 24, 2051 | 11u << 24,
    4099 | 12u << 24, 8195 | 13u << 24, 16387 | 14u << 24, 32771 | 15u << 24,
    65539 | 16u << 24};
static __constant__ int16_t kPreLL[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                   2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
static __constant__ int16_t kPreOF[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};
static __constant__ int16_t kPreML[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                   1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};

struct Tables {
    uint32_t size[3];
    unsigned log[3];
    bool present[3];
    unsigned huf_log;
    bool huf_present;
};

// Sequence table load (src/zstd_seq.h ZstdSeqLoadTable).
__device__ inline bool seq_table(WarpSmem& w, Tables& t, unsigned field, unsigned mode,
                          const uint8_t* src, uint64_t size, uint64_t* used, uint32_t lane) {
    const unsigned symmax = field == 0 ? 35 : field == 1 ? 31 : 52;
    const unsigned logmax = field == 1 ? 8 : 9;
    *used = 0;
    if (mode == 3) return t.present[field];
    if (mode == 1) {
        if (size == 0) return false;
        const unsigned s = src[0];
        if (s > symmax) return false;
        __syncwarp();
        if (lane == 0) w.fse[field][0] = s << 8;
        __syncwarp();
        t.size[field] = 1;
        t.log[field] = 0;
        t.present[field] = true;
        *used = 1;
        return true;
    }
    unsigned dmax, log;
    if (mode == 0) {
        const int16_t* pre = field == 0 ? kPreLL : field == 1 ? kPreOF : kPreML;
        dmax = field == 0 ? 35 : field == 1 ? 28 : 52;
        log = field == 1 ? 5 : 6;
        __syncwarp();
        for (unsigned s = lane; s <= dmax; s += 32) w.counts[s] = pre[s];
        __syncwarp();
    } else {
        if (!fse_ncount(src, size, symmax, logmax, w.counts, &dmax, &log, used)) return false;
    }
    if (!fse_build(w.counts, dmax, log, w.fse[field], w.next, lane)) {
        *used = 0;
        return false;
    }
    t.size[field] = 1u << log;
    t.log[field] = log;
    t.present[field] = true;
    return true;
}



}  // namespace zstd
}  // namespace cdb
