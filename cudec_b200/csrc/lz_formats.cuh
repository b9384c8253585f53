// Byte-oriented LZ formats decoded by the block kernel: LZ4 block and raw
// Snappy. Each format is a policy with four device functions:
//
//   begin(...)   per-chunk preamble: first token position (+ declared length)
//   step(p)      speculative: where the next token would start if a token
//                started at p (no validation beyond staying inside the input);
//                used to run the parallel speculative token chains
//   fields(p)    the sequence at a true token: literal source/length, match
//                length and offset (unchecked)
//   check(p, d)  the full accept/reject ladder for the token at p with d
//                bytes already produced, in the reference's check order, so a
//                chunk's status is exactly the serial decoder's status
//
// A token position that `step` walks is a "sequence" for LZ4 (literal run +
// match) and an "element" for Snappy (literal OR copy). Both are described by
// the same Seq record: out bytes = lit_len literal bytes from the input, then
// match_len bytes copied from `off` bytes back in the output.
#pragma once

#include <cstdint>

#include "cudec.h"

namespace cdb {

constexpr uint64_t kBad = ~0ull;  // a step that cannot be a valid token

// Read-only view of one chunk's compressed bytes: the window staged in shared
// memory, else the global copy.
struct InView {
    const uint8_t* g;   // global chunk base
    const uint8_t* sm;  // shared buffer; sm[i] is byte lo + i
    uint64_t lo, len;
    __device__ __forceinline__ uint32_t at(uint64_t p) const {
        const uint64_t r = p - lo;
        return r < len ? static_cast<uint32_t>(sm[r])
                       : static_cast<uint32_t>(__ldg(g + p));
    }
};

struct Seq {
    uint64_t lit_src, lit_len, match_len;
    uint32_t off;
    // Every check that does not depend on the output position passed (and,
    // for LZ4, the run is not a terminal one): `fast_ok` can then decide the
    // sequence from its output position alone.
    bool clean;
};

// --------------------------------------------------------------------------
// LZ4 block: follows iderex/cudec src/lz4_block.h:139-258 (Lz4Parser::Next)
// and :95-128 (AccumulateLength); format constants at :46-66.
// --------------------------------------------------------------------------
struct Lz4Format {
    static constexpr uint64_t kEndSlackDst = 12;  // MFLIMIT
    static constexpr uint64_t kEndSlackSrc = 8;   // 2 + 1 + LASTLITERALS
    static constexpr uint64_t kLastLiterals = 5;

    // No preamble: the first token is at 0. `limit` is the capacity.
    __device__ static int begin(const uint8_t*, uint64_t, uint64_t cap,
                                uint64_t* first, uint64_t* limit) {
        *first = 0;
        *limit = cap;
        return CUDEC_OK;
    }

    __device__ __forceinline__ static uint64_t step(const InView& in,
                                                    uint64_t S, uint64_t p) {
        const uint32_t tok = in.at(p);
        uint64_t q = p + 1;
        uint64_t lit = tok >> 4;
        if (lit == 15) {
            uint32_t b;
            do {
                if (q >= S) return kBad;
                b = in.at(q++);
                lit += b;
            } while (b == 255);
        }
        if (lit > S - q) return kBad;
        q += lit;
        if (S - q < kEndSlackSrc) return q == S ? S : kBad;
        q += 2;
        if ((tok & 15) == 15) {
            uint32_t b;
            do {
                if (q >= S) return kBad;
                b = in.at(q++);
            } while (b == 255);
        }
        return q;
    }

    __device__ __forceinline__ static void fields(const InView& in, uint64_t S,
                                                  uint64_t p, Seq* s) {
        const uint32_t tok = in.at(p);
        uint64_t q = p + 1;
        uint64_t lit = tok >> 4;
        s->match_len = 0;
        s->off = 1;
        s->clean = false;
        if (lit == 15) {
            if (q + 15 >= S) { s->lit_src = q; s->lit_len = 0; return; }
            uint32_t b;
            do {
                if (q >= S) { s->lit_src = q; s->lit_len = 0; return; }
                b = in.at(q++);
                lit += b;
                if (q + 15 > S) { s->lit_src = q; s->lit_len = 0; return; }
            } while (b == 255);
        }
        s->lit_src = q;
        s->lit_len = lit;
        if (lit > S - q) return;
        q += lit;
        if (S - q < kEndSlackSrc) return;
        s->off = in.at(q) | (in.at(q + 1) << 8);
        q += 2;
        uint64_t ml = (tok & 15) + 4;
        bool ok = s->off != 0;
        if ((tok & 15) == 15) {
            uint32_t b;
            do {
                if (q >= S) { ok = false; break; }
                b = in.at(q++);
                ml += b;
                if (q + 4 > S) { ok = false; break; }
            } while (b == 255);
        }
        s->match_len = ml;
        s->clean = ok;
    }

    // A clean, non-terminal sequence that fits with the end-of-block slack to
    // spare passes every rung of `check` and is not the terminal run.
    __device__ __forceinline__ static bool fast_ok(const Seq& s, uint64_t cap,
                                                   uint64_t d) {
        return s.clean && d <= cap && s.off <= d + s.lit_len &&
               cap - d >= s.lit_len + s.match_len + kEndSlackDst;
    }

    // AccumulateLength (lz4_block.h:95-128): `room` = capacity - dst_pos.
    __device__ __forceinline__ static int extend(const InView& in, uint64_t S,
                                                 uint64_t* q, uint64_t* len,
                                                 uint64_t room, uint64_t margin,
                                                 bool pre) {
        if (pre && *q + margin >= S) return CUDEC_ERR_CORRUPT_INPUT;
        uint32_t b;
        do {
            if (*q >= S) return CUDEC_ERR_CORRUPT_INPUT;
            if (*len > room) return CUDEC_ERR_OUTPUT_TOO_SMALL;
            b = in.at((*q)++);
            *len += b;
            if (*q + margin > S) return CUDEC_ERR_CORRUPT_INPUT;
        } while (b == 255);
        return CUDEC_OK;
    }

    __device__ static int check(const InView& in, uint64_t S, uint64_t cap,
                                uint64_t p, uint64_t d, bool* done) {
        *done = false;
        if (p >= S) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t tok = in.at(p);
        uint64_t q = p + 1;
        uint64_t lit = tok >> 4;
        if (lit == 15) {
            int st = extend(in, S, &q, &lit, cap - d, 15, true);
            if (st != CUDEC_OK) return st;
        }
        if (lit > S - q) return CUDEC_ERR_CORRUPT_INPUT;
        if (lit > cap - d) return CUDEC_ERR_OUTPUT_TOO_SMALL;
        if (cap - d - lit < kEndSlackDst || S - q - lit < kEndSlackSrc) {
            if (q + lit != S) return CUDEC_ERR_CORRUPT_INPUT;
            // Capacity zero accepts only the single byte 0x00 (lz4_block.h:178-187).
            if (cap == 0 && tok != 0) return CUDEC_ERR_CORRUPT_INPUT;
            *done = true;
            return CUDEC_OK;
        }
        q += lit;
        d += lit;
        const uint64_t off = in.at(q) | (in.at(q + 1) << 8);
        q += 2;
        if (off == 0) return CUDEC_ERR_CORRUPT_INPUT;  // stricter than liblz4
        if (off > d) return CUDEC_ERR_CORRUPT_INPUT;
        uint64_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15) {
            int st = extend(in, S, &q, &ml, cap - d, 4, false);
            if (st != CUDEC_OK) return st;
        }
        if (ml > cap - d) return CUDEC_ERR_OUTPUT_TOO_SMALL;
        if (ml > cap - d - kLastLiterals) return CUDEC_ERR_CORRUPT_INPUT;
        return CUDEC_OK;
    }

    // The chain ran out of tokens without a terminal run: the serial decoder
    // asks for one more token and finds none.
    __device__ static int finish(bool, uint64_t, uint64_t) {
        return CUDEC_ERR_CORRUPT_INPUT;
    }
};

// --------------------------------------------------------------------------
// Raw Snappy: follows iderex/cudec src/snappy_block.h:172-223
// (SnappyDeclaredLength) and :249-435 (SnappyParser::Begin/Next).
// --------------------------------------------------------------------------
struct SnappyFormat {
    // Varint32 preamble; `limit` becomes the declared length.
    __device__ static int begin(const uint8_t* g, uint64_t S, uint64_t cap,
                                uint64_t* first, uint64_t* limit) {
        uint64_t v = 0;
        for (uint64_t k = 0; k < 5; ++k) {
            if (k >= S) return CUDEC_ERR_CORRUPT_INPUT;
            const uint32_t b = g[k];
            if (k == 4 && b >= 16) return CUDEC_ERR_CORRUPT_INPUT;
            v |= static_cast<uint64_t>(b & 0x7f) << (7 * k);
            if (!(b & 0x80)) {
                if (v > cap) return CUDEC_ERR_OUTPUT_TOO_SMALL;
                *first = k + 1;
                *limit = v;
                return CUDEC_OK;
            }
        }
        return CUDEC_ERR_CORRUPT_INPUT;
    }

    __device__ __forceinline__ static uint64_t step(const InView& in,
                                                    uint64_t S, uint64_t p) {
        const uint32_t tag = in.at(p);
        const uint32_t kind = tag & 3;
        if (kind == 0) {
            const uint32_t l6 = tag >> 2;
            uint64_t hdr = 1, len = l6;
            if (l6 >= 60) {
                const uint32_t extra = l6 - 59;
                hdr += extra;
                if (hdr > S - p) return kBad;
                len = 0;
                for (uint32_t i = 0; i < extra; ++i)
                    len |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
            }
            len += 1;
            const uint64_t q = p + hdr;
            if (len > S - q) return kBad;
            return q + len;
        }
        const uint64_t hdr = kind == 1 ? 2 : (kind == 2 ? 3 : 5);
        if (hdr > S - p) return kBad;
        return p + hdr;
    }

    __device__ __forceinline__ static void fields(const InView& in, uint64_t S,
                                                  uint64_t p, Seq* s) {
        const uint32_t tag = in.at(p);
        const uint32_t kind = tag & 3;
        s->lit_len = 0;
        s->match_len = 0;
        s->off = 1;
        s->lit_src = p;
        s->clean = false;
        if (kind == 0) {
            const uint32_t l6 = tag >> 2;
            uint64_t hdr = 1, len = l6;
            if (l6 >= 60) {
                const uint32_t extra = l6 - 59;
                hdr += extra;
                if (hdr > S - p) return;
                len = 0;
                for (uint32_t i = 0; i < extra; ++i)
                    len |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
            }
            s->lit_src = p + hdr;
            s->lit_len = len + 1;
            s->clean = s->lit_len <= S - s->lit_src;
            return;
        }
        const uint32_t ob = kind == 1 ? 1 : (kind == 2 ? 2 : 4);
        if (1 + ob > S - p) return;
        uint64_t off = 0;
        for (uint32_t i = 0; i < ob; ++i)
            off |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
        if (kind == 1) {
            off |= static_cast<uint64_t>(tag >> 5) << 8;
            s->match_len = 4 + ((tag >> 2) & 7);
        } else {
            s->match_len = (tag >> 2) + 1;
        }
        s->off = static_cast<uint32_t>(off);
        s->clean = off != 0;
    }

    // A clean element whose source and length fit the produced/declared
    // bounds passes every rung of `check`.
    __device__ __forceinline__ static bool fast_ok(const Seq& s, uint64_t declared,
                                                   uint64_t d) {
        const uint64_t len = s.lit_len + s.match_len;
        return s.clean && d <= declared && len <= declared - d &&
               (s.match_len == 0 || s.off <= d);
    }

    // `declared` is the preamble's length (already bounded by capacity).
    __device__ static int check(const InView& in, uint64_t S, uint64_t declared,
                                uint64_t p, uint64_t d, bool* done) {
        *done = false;
        const uint32_t tag = in.at(p);
        const uint32_t kind = tag & 3;
        if (kind == 0) {
            const uint32_t l6 = tag >> 2;
            uint64_t hdr = 1, len = l6;
            if (l6 >= 60) {
                const uint32_t extra = l6 - 59;
                hdr += extra;
                if (hdr > S - p) return CUDEC_ERR_CORRUPT_INPUT;
                len = 0;
                for (uint32_t i = 0; i < extra; ++i)
                    len |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
            }
            len += 1;  // 64-bit: the 0xFFFFFFFF spelling is refused, not wrapped
            const uint64_t q = p + hdr;
            if (len > S - q) return CUDEC_ERR_CORRUPT_INPUT;
            if (len > declared - d) return CUDEC_ERR_CORRUPT_INPUT;
            return CUDEC_OK;
        }
        const uint32_t ob = kind == 1 ? 1 : (kind == 2 ? 2 : 4);
        if (1 + ob > S - p) return CUDEC_ERR_CORRUPT_INPUT;
        uint64_t off = 0, len;
        for (uint32_t i = 0; i < ob; ++i)
            off |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
        if (kind == 1) {
            off |= static_cast<uint64_t>(tag >> 5) << 8;
            len = 4 + ((tag >> 2) & 7);
        } else {
            len = (tag >> 2) + 1;
        }
        if (off == 0) return CUDEC_ERR_CORRUPT_INPUT;
        if (off > d) return CUDEC_ERR_CORRUPT_INPUT;
        if (len > declared - d) return CUDEC_ERR_CORRUPT_INPUT;
        return CUDEC_OK;
    }

    // Elements exhausted: success only at exact consumption and exact
    // production of the declared length.
    __device__ static int finish(bool at_end, uint64_t produced,
                                 uint64_t declared) {
        return (at_end && produced == declared) ? CUDEC_OK
                                                : CUDEC_ERR_CORRUPT_INPUT;
    }
};

}  // namespace cdb
