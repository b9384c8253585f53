// Exact accept/reject ladders of the byte-oriented LZ formats (LZ4 block,
// raw Snappy), shared by every decoder of those formats in this library and
// by host code. Each decoder proposes token positions its own way; the
// ladder at a position, with the output length produced before it, decides
// the token exactly as the serial parser would.
//
// The input is read through a reader R with `uint32_t at(uint64_t q)` for
// q < S (the chunk's bytes); the ladders never read at or past S.
//
// LZ4 follows iderex/cudec src/lz4_block.h:95-258 (Lz4Parser::Next,
// AccumulateLength; constants :46-66); Snappy src/snappy_block.h:172-435
// (SnappyDeclaredLength, SnappyParser::Begin/Next).
#pragma once

#include <cstdint>

#include "cudec.h"

#ifndef CDB_HD
#if defined(__CUDACC__)
#define CDB_HD __host__ __device__ __forceinline__
#else
#define CDB_HD inline
#endif
#endif

namespace cdb {
namespace lzl {

// One parsed sequence: lit literal bytes from input offset lit_src, then ml
// bytes copied from off bytes back; next = the following token's position;
// done = the chunk ends after this sequence (LZ4's terminal literal run).
struct Seq {
    uint64_t lit_src, lit, ml, next;
    uint32_t off;
    bool done;
};

// ---------------------------------------------------------------------------
// LZ4 block.
struct Lz4Ladder {
    static constexpr uint64_t kMfLimit = 12;
    static constexpr uint64_t kSrcSlack = 8;
    static constexpr uint64_t kLastLiterals = 5;

    template <class R>
    CDB_HD static int begin(const R&, uint64_t, uint64_t cap, uint64_t* first,
                             uint64_t* limit) {
        *first = 0;
        *limit = cap;
        return CUDEC_OK;
    }
    CDB_HD static bool at_end(uint64_t, uint64_t) { return false; }
    CDB_HD static int finish(uint64_t, uint64_t) { return CUDEC_OK; }

    template <class R>
    CDB_HD static int extend(const R& in, uint64_t S, uint64_t* q,
                             uint64_t* len, uint64_t room, uint64_t margin,
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

    // The token at p with d bytes already produced; cap is the capacity.
    template <class R>
    CDB_HD static int parse(const R& in, uint64_t S, uint64_t cap,
                             uint64_t p, uint64_t d, Seq* s) {
        if (p >= S) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t tok = in.at(p);
        uint64_t q = p + 1;
        uint64_t lit = tok >> 4;
        if (lit == 15) {
            const int st = extend(in, S, &q, &lit, cap - d, 15, true);
            if (st != CUDEC_OK) return st;
        }
        if (lit > S - q) return CUDEC_ERR_CORRUPT_INPUT;
        if (lit > cap - d) return CUDEC_ERR_OUTPUT_TOO_SMALL;
        s->lit_src = q;
        s->lit = lit;
        if (cap - d - lit < kMfLimit || S - q - lit < kSrcSlack) {
            if (q + lit != S) return CUDEC_ERR_CORRUPT_INPUT;
            // Capacity zero accepts only the single byte 0x00 (lz4_block.h:178-187).
            if (cap == 0 && tok != 0) return CUDEC_ERR_CORRUPT_INPUT;
            s->ml = 0;
            s->off = 0;
            s->next = S;
            s->done = true;
            return CUDEC_OK;
        }
        q += lit;
        d += lit;
        const uint32_t off = in.at(q) | (in.at(q + 1) << 8);
        q += 2;
        if (off == 0) return CUDEC_ERR_CORRUPT_INPUT;  // stricter than liblz4
        if (off > d) return CUDEC_ERR_CORRUPT_INPUT;
        uint64_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15) {
            const int st = extend(in, S, &q, &ml, cap - d, 4, false);
            if (st != CUDEC_OK) return st;
        }
        if (ml > cap - d) return CUDEC_ERR_OUTPUT_TOO_SMALL;
        if (ml > cap - d - kLastLiterals) return CUDEC_ERR_CORRUPT_INPUT;
        s->ml = ml;
        s->off = off;
        s->next = q;
        s->done = false;
        return CUDEC_OK;
    }
};

// ---------------------------------------------------------------------------
// Raw Snappy. One element (literal OR copy) per Seq.
struct SnappyLadder {
    template <class R>
    CDB_HD static int begin(const R& in, uint64_t S, uint64_t cap, uint64_t* first,
                             uint64_t* limit) {
        uint64_t v = 0;
        for (uint64_t k = 0; k < 5; ++k) {
            if (k >= S) return CUDEC_ERR_CORRUPT_INPUT;
            const uint32_t b = in.at(k);
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
    CDB_HD static bool at_end(uint64_t p, uint64_t S) { return p == S; }
    // Elements exhausted: success only at exact production of the declared length.
    CDB_HD static int finish(uint64_t d, uint64_t declared) {
        return d == declared ? CUDEC_OK : CUDEC_ERR_CORRUPT_INPUT;
    }

    template <class R>
    CDB_HD static int parse(const R& in, uint64_t S,
                             uint64_t declared, uint64_t p, uint64_t d,
                                                Seq* s) {
        const uint32_t tag = in.at(p);
        const uint32_t kind = tag & 3;
        s->done = false;
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
            s->lit_src = q;
            s->lit = len;
            s->ml = 0;
            s->off = 0;
            s->next = q + len;
            return CUDEC_OK;
        }
        const uint32_t ob = kind == 1 ? 1 : (kind == 2 ? 2 : 4);
        if (1 + ob > S - p) return CUDEC_ERR_CORRUPT_INPUT;
        uint64_t off = 0, len;
        for (uint32_t i = 0; i < ob; ++i) off |= static_cast<uint64_t>(in.at(p + 1 + i)) << (8 * i);
        if (kind == 1) {
            off |= static_cast<uint64_t>(tag >> 5) << 8;
            len = 4 + ((tag >> 2) & 7);
        } else {
            len = (tag >> 2) + 1;
        }
        if (off == 0) return CUDEC_ERR_CORRUPT_INPUT;
        if (off > d) return CUDEC_ERR_CORRUPT_INPUT;
        if (len > declared - d) return CUDEC_ERR_CORRUPT_INPUT;
        s->lit_src = p;
        s->lit = 0;
        s->ml = len;
        s->off = static_cast<uint32_t>(off);
        s->next = p + 1 + ob;
        return CUDEC_OK;
    }
};

}  // namespace lzl
}  // namespace cdb
