// One GDeflate page decoded by one warp: the 32 substreams are the 32 lanes.
//
// Each lane keeps its substream's bit buffer (64 bits) and occupancy in
// registers; the word cursor is warp-uniform. A round is one operation per
// lane on its own bits, then the refill: every lane below 32 buffered bits
// takes the next word, in lane order (word = cursor + the number of lower
// lanes that also refill) - the schedule of iderex/cudec
// src/gdeflate_schedule.h:129-165 executed for all 32 lanes at once. Block
// headers, table descriptions, stored bytes and symbols follow the round
// structure documented in oracle_gdeflate_decode (the CPU restatement this
// kernel is checked against): the draft's sections 5-11 and divergences
// D1-D6 from RFC 1951, with the open points decided there.
//
// Symbols: a 10-bit lookup table per code (litlen, distance) in shared
// memory, canonical decoding for longer codes; the precode has a complete
// 7-bit table. End-of-block quiesce is a ballot: lanes after the first lane
// that read end-of-block (and have no distance pending) do not consume.
// Output positions come from a warp scan of the round's item lengths; bytes
// go straight to the destination (a page is at most 64 KiB) and copies read
// them back from there. Shared memory holds only the tables (about 6 KB per
// warp), so many pages decode per SM: staging the page in shared memory
// measured 5x slower for lack of resident warps.
//
// Errors are reported in serial order: an operation's error at lane l
// precedes lane l's refill, which precedes lane l+1's operation.
#pragma once

#include <cstdint>

#include "cudec.h"
#include "lz_warp_kernel.cuh"

namespace cdb {
namespace gdf {

constexpr uint32_t kPageMax = 65536;
constexpr uint32_t kTabBits = 10;
constexpr uint32_t kNoEvent = 64;  // event index when none (2 * lane + phase otherwise)

// Per-warp decode tables (shared memory).
struct __align__(16) Tables {
    uint16_t ltab[1 << kTabBits];  // sym | len << 9, 0 = use the canonical path
    uint16_t dtab[1 << kTabBits];
    uint16_t ptab[128];
    uint16_t lcount[16], dcount[16];
    uint16_t lsym[288], dsym[32];
    uint16_t code[320];  // canonical codes during a table build
    uint8_t lens[320];
    uint8_t plen[20];
    // canonical-decode state after the lengths the lookup table covers
    // (first code and symbol index at length kTabBits + 1), per table
    int32_t lfirst, lindex, dfirst, dindex;
};


static __constant__ uint16_t kLBase[29] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  13,
                                    15, 17, 19, 23, 27, 31, 35, 43,  51,  59,
                                    67, 83, 99, 115, 131, 163, 195, 227, 3};
static __constant__ uint8_t kLExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                    2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 16};
static __constant__ uint32_t kDBase[32] = {1,     2,     3,     4,     5,     7,    9,    13,
                                    17,    25,    33,    49,    65,    97,   129,  193,
                                    257,   385,   513,   769,   1025,  1537, 2049, 3073,
                                    4097,  6145,  8193,  12289, 16385, 24577, 32769, 49153};
static __constant__ uint8_t kDExtra[32] = {0, 0, 0, 0, 1, 1, 2, 2, 3,  3,  4,  4,  5,  5,  6,  6,
                                    7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14};
static __constant__ uint8_t kPerm[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 11, 12, 13, 14, 15, 5, 4, 3, 2, 1};

struct Lane {
    const uint8_t* pg;
    bool aligned;
    uint64_t words, cursor;
    uint64_t bb;
    uint32_t left;

    __device__ __forceinline__ uint32_t word(uint64_t i) const {
        const uint8_t* p = pg + 4 * i;
        if (aligned) return __ldg(reinterpret_cast<const uint32_t*>(p));
        return static_cast<uint32_t>(__ldg(p)) | (static_cast<uint32_t>(__ldg(p + 1)) << 8) |
               (static_cast<uint32_t>(__ldg(p + 2)) << 16) |
               (static_cast<uint32_t>(__ldg(p + 3)) << 24);
    }
    __device__ __forceinline__ void consume(uint32_t n) {
        bb >>= n;
        left -= n;
    }
    // The refill turn of every lane; returns the event index of the first
    // lane with no word left (2 * lane + 1), else kNoEvent.
    __device__ __forceinline__ uint32_t refill(uint32_t lane) {
        const bool need = left < 32;
        const unsigned m = __ballot_sync(0xffffffffu, need);
        const uint32_t rank = __popc(m & ((1u << lane) - 1));
        const uint64_t avail = words - cursor;
        const uint32_t want = __popc(m);
        if (need && rank < avail) {
            bb |= static_cast<uint64_t>(word(cursor + rank)) << left;
            left += 32;
        }
        uint32_t ev = kNoEvent;
        if (want > avail) {
            // the lane whose rank equals avail is the first that finds no word
            const unsigned short_lanes = __ballot_sync(0xffffffffu, need && rank >= avail);
            ev = 2 * (__ffs(short_lanes) - 1) + 1;
        }
        cursor += want < avail ? want : avail;
        return ev;
    }
};

// Table from code lengths (count/sorted symbols for the canonical path and a
// kTabBits lookup table). Lane 0 computes the canonical codes; all lanes fill
// the table. Returns false (all lanes) when the code is over-subscribed.
__device__ __forceinline__ bool build_code(Tables& sm, const uint8_t* lens, uint32_t n,
                                           uint16_t* tab, uint16_t* count, uint16_t* sym,
                                           uint32_t tbits, int32_t* first_out,
                                           int32_t* index_out, uint32_t lane) {
    __syncwarp();
    bool ok = true;
    if (lane == 0) {
        uint16_t cnt[16];
        for (int b = 0; b < 16; ++b) cnt[b] = 0;
        for (uint32_t s = 0; s < n; ++s) cnt[lens[s]]++;
        int leftk = 1;
        for (int b = 1; b < 16; ++b) {
            leftk <<= 1;
            leftk -= cnt[b];
            if (leftk < 0) ok = false;
        }
        uint16_t offs[16], next[16];
        offs[1] = 0;
        for (int b = 1; b < 15; ++b) offs[b + 1] = offs[b] + cnt[b];
        uint32_t c = 0;
        cnt[0] = 0;
        for (int b = 1; b < 16; ++b) {
            c = (c + cnt[b - 1]) << 1;
            next[b] = static_cast<uint16_t>(c);
        }
        for (int b = 0; b < 16; ++b) count[b] = cnt[b];
        // the canonical walk's first code and symbol index once it has passed
        // the lengths the lookup table holds (they depend on the counts only)
        int32_t f = 0, ix = 0;
        for (uint32_t b = 1; b <= tbits; ++b) {
            ix += cnt[b];
            f = (f + cnt[b]) << 1;
        }
        *first_out = f;
        *index_out = ix;
        for (uint32_t s = 0; s < n; ++s) {
            const uint32_t l = lens[s];
            if (l && ok) {
                sym[offs[l]++] = static_cast<uint16_t>(s);
                sm.code[s] = next[l]++;
            }
        }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (!ok) return false;
    const uint32_t size = 1u << tbits;
    for (uint32_t i = lane; i < size; i += 32) tab[i] = 0;
    __syncwarp();
    for (uint32_t s = lane; s < n; s += 32) {
        const uint32_t l = lens[s];
        if (l == 0 || l > tbits) continue;
        const uint32_t rc = __brev(static_cast<uint32_t>(sm.code[s])) >> (32 - l);
        const uint16_t e = static_cast<uint16_t>(s | (l << 9));
        for (uint32_t i = rc; i < size; i += 1u << l) tab[i] = e;
    }
    __syncwarp();
    return true;
}

// Decode a code from the low bits of bb: symbol and length, or false. Codes
// of up to kTabBits bits come from the lookup table; longer ones continue the
// canonical walk at length kTabBits + 1 from the state build_code stored (a
// zero table entry means no shorter code matched, so the walk would not have
// stopped earlier), with the code so far the first kTabBits bits in reading
// order.
__device__ __forceinline__ bool decode_sym(uint64_t bb, const uint16_t* tab, const uint16_t* count,
                                           const uint16_t* sym, int32_t first0, int32_t index0,
                                           uint32_t* s, uint32_t* len) {
    const uint16_t e = tab[bb & ((1u << kTabBits) - 1)];
    if (e) {
        *s = e & 511;
        *len = e >> 9;
        return true;
    }
    int code = static_cast<int>(
                   __brev(static_cast<uint32_t>(bb) & ((1u << kTabBits) - 1)) >> (32 - kTabBits))
               << 1;
    int first = first0, index = index0;
    for (int l = kTabBits + 1; l <= 15; ++l) {
        code |= static_cast<int>((bb >> (l - 1)) & 1);
        const int c = count[l];
        if (code - c < first) {
            *s = sym[index + (code - first)];
            *len = static_cast<uint32_t>(l);
            return true;
        }
        index += c;
        first += c;
        first <<= 1;
        code <<= 1;
    }
    return false;
}

// The first event of a round: op errors (phase 0, status in st) against the
// refill's first failure (phase 1, CORRUPT). Returns CUDEC_OK when none.
__device__ __forceinline__ int first_event(bool err, int st, uint32_t refill_ev, uint32_t lane) {
    const unsigned em = __ballot_sync(0xffffffffu, err);
    const uint32_t op_ev = em ? 2 * (__ffs(em) - 1) : kNoEvent;
    if (op_ev == kNoEvent && refill_ev == kNoEvent) return CUDEC_OK;
    if (op_ev < refill_ev) return __shfl_sync(0xffffffffu, st, op_ev / 2);
    return CUDEC_ERR_CORRUPT_INPUT;
}

// Copy [o, o + n) from o - d inside the page's output (d <= o), one lane,
// in 16-byte windows: the aligned words holding the bytes, joined by funnel
// shifts, then the widest stores the destination's alignment allows. The
// first window is one read and one write in every lane (a distance under 16
// is expanded to 16 bytes by lzw::period16), the rest a plain copy at
// lzw::rest_distance(d). Every byte a window reads was written before it, by
// this lane or earlier.
__device__ __forceinline__ void page_copy(uint8_t* out, uint32_t o, uint32_t n, uint32_t d) {
    uint8_t* D = out + o;
    const uint32_t m0 = n < 16 ? n : 16u;
    lzw::st16_global(D, lzw::period16(lzw::ld16_words(D - d, d < 16 ? d : m0), d), m0);
    const uint32_t q = lzw::rest_distance(d);
    for (uint32_t k = 16; k < n; k += 16) {
        const uint32_t m = n - k < 16 ? n - k : 16u;
        lzw::st16_global(D + k, lzw::ld16_words(D + k - q, m), m);
    }
}

// Decode one page; every lane returns the same status and *written. Output
// goes straight to dst (its bytes are only ever read back by this warp's own
// copies, ordered by __syncwarp), so a warp needs only its tables in shared
// memory and many warps share an SM.
__device__ __forceinline__ int decode_page(const uint8_t* pg, uint64_t N, uint8_t* dst,
                                           uint64_t cap, Tables& sm, uint32_t lane,
                                           uint64_t* written) {
    *written = 0;
    uint8_t* const out = dst;
    if (N % 4 != 0 || N / 4 < 32) return CUDEC_ERR_CORRUPT_INPUT;
    Lane ln{pg, (reinterpret_cast<uintptr_t>(pg) & 3) == 0, N / 4, 32, 0, 32};
    ln.bb = ln.word(lane);
    uint32_t pos = 0;
    const uint64_t room = cap;
    bool final = false;
    while (!final) {
        // ---- block header round (lane 0) ----
        const uint32_t hb = __shfl_sync(0xffffffffu, static_cast<uint32_t>(ln.bb & 7), 0);
        final = hb & 1;
        const uint32_t btype = hb >> 1;
        if (lane == 0) ln.consume(3);
        if (ln.refill(lane) != kNoEvent) return CUDEC_ERR_CORRUPT_INPUT;
        if (btype == 3) return CUDEC_ERR_CORRUPT_INPUT;
        if (btype == 0) {
            const uint32_t len = __shfl_sync(0xffffffffu, static_cast<uint32_t>(ln.bb & 0xFFFF), 0);
            if (lane == 0) ln.consume(16);
            if (ln.refill(lane) != kNoEvent) return CUDEC_ERR_CORRUPT_INPUT;
            for (uint32_t r = 0; r * 32 < len; ++r) {
                const bool act = r * 32 + lane < len;
                const uint32_t p = pos + r * 32 + lane;
                const uint8_t b = static_cast<uint8_t>(ln.bb);
                int st = CUDEC_OK;
                if (act) {
                    ln.consume(8);
                    if (p >= kPageMax) st = CUDEC_ERR_CORRUPT_INPUT;
                    else if (p >= room) st = CUDEC_ERR_OUTPUT_TOO_SMALL;
                    else out[p] = b;
                }
                const uint32_t rev = ln.refill(lane);
                const int s = first_event(st != CUDEC_OK, st, rev, lane);
                if (s != CUDEC_OK) return s;
            }
            pos += len;
            continue;
        }
        // ---- tables ----
        uint32_t hlit = 288, hdist = 32;
        if (btype == 1) {
            for (uint32_t s = lane; s < 320; s += 32)
                sm.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : s < 288 ? 8 : 5;
            __syncwarp();
        } else {
            const uint32_t h = __shfl_sync(0xffffffffu, static_cast<uint32_t>(ln.bb & 0x3FFF), 0);
            hlit = (h & 31) + 257;
            hdist = ((h >> 5) & 31) + 1;
            const uint32_t hclen = (h >> 10) + 4;
            if (lane == 0) ln.consume(14);
            if (ln.refill(lane) != kNoEvent) return CUDEC_ERR_CORRUPT_INPUT;
            if (hlit > 288 || hdist > 32) return CUDEC_ERR_CORRUPT_INPUT;
            if (lane < 19) sm.plen[kPerm[lane]] = 0;
            __syncwarp();
            if (lane < hclen) {
                sm.plen[kPerm[lane]] = static_cast<uint8_t>(ln.bb & 7);
                ln.consume(3);
            }
            if (ln.refill(lane) != kNoEvent) return CUDEC_ERR_CORRUPT_INPUT;
            // precode: complete 7-bit table (its codes are at most 7 bits)
            // (the precode's walk state is not used: its codes fit its table)
            if (!build_code(sm, sm.plen, 19, sm.ptab, sm.lcount, sm.lsym, 7, &sm.lfirst,
                            &sm.lindex, lane))
                return CUDEC_ERR_CORRUPT_INPUT;
            const uint32_t total = hlit + hdist;
            uint32_t have = 0;
            uint32_t prev_last = 0;  // the last length written so far
            while (have < total) {
                const uint16_t e = sm.ptab[ln.bb & 127];
                const bool valid = e != 0;
                const uint32_t sym = e & 511, clen = e >> 9;
                uint32_t rep = 1, xb = 0, val = sym;
                if (valid && sym >= 16) {
                    xb = sym == 16 ? 2 : sym == 17 ? 3 : 7;
                    const uint32_t x = static_cast<uint32_t>(ln.bb >> clen) & ((1u << xb) - 1);
                    rep = (sym == 16 ? 3 : sym == 17 ? 3 : 11) + x;
                    val = sym == 16 ? 0xFFFFu : 0;
                }
                // lane l is active while fewer than `total` lengths are known
                uint32_t incl = rep;
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) {
                    const uint32_t o = __shfl_up_sync(0xffffffffu, incl, k);
                    if (lane >= k) incl += o;
                }
                const uint32_t excl = incl - rep;
                // activity needs the decoded count of earlier lanes; an
                // invalid code stops the count (its lane errors if active)
                const unsigned badm = __ballot_sync(0xffffffffu, !valid);
                const uint32_t first_bad = badm ? __ffs(badm) - 1 : 32;
                const bool act = have + excl < total && lane <= first_bad;
                int st = CUDEC_OK;
                if (act) {
                    if (!valid) st = CUDEC_ERR_CORRUPT_INPUT;
                    else if (sym == 16 && have + excl == 0) st = CUDEC_ERR_CORRUPT_INPUT;
                    else if (have + incl > total) st = CUDEC_ERR_CORRUPT_INPUT;
                }
                // value of code 16 runs: the nearest earlier length
                uint32_t v = act ? val : 0xFFFFu;
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) {
                    const uint32_t o = __shfl_up_sync(0xffffffffu, v, k);
                    if (v == 0xFFFFu && lane >= k) v = o;
                }
                if (v == 0xFFFFu) v = prev_last;
                if (act && st == CUDEC_OK) {
                    ln.consume(clen + xb);
                    for (uint32_t k = 0; k < rep; ++k) sm.lens[have + excl + k] = static_cast<uint8_t>(v);
                }
                const uint32_t rev = ln.refill(lane);
                const int s = first_event(st != CUDEC_OK, st, rev, lane);
                if (s != CUDEC_OK) return s;
                const unsigned am = __ballot_sync(0xffffffffu, act);
                const uint32_t last = 31 - __clz(am);
                prev_last = __shfl_sync(0xffffffffu, v, last);
                have += __shfl_sync(0xffffffffu, incl, last);
                __syncwarp();
            }
            if (sm.lens[256] == 0) return CUDEC_ERR_CORRUPT_INPUT;
        }
        if (!build_code(sm, sm.lens, hlit, sm.ltab, sm.lcount, sm.lsym, kTabBits, &sm.lfirst,
                        &sm.lindex, lane))
            return CUDEC_ERR_CORRUPT_INPUT;
        if (!build_code(sm, sm.lens + hlit, hdist, sm.dtab, sm.dcount, sm.dsym, kTabBits,
                        &sm.dfirst, &sm.dindex, lane))
            return CUDEC_ERR_CORRUPT_INPUT;
        // ---- data rounds ----
        bool pend = false, eob = false;
        uint32_t ppos = 0, plen = 0;
        for (;;) {
            const bool want_dist = pend;
            const bool want_lit = !pend && !eob;
            uint32_t sym = 0, clen = 0;
            bool valid = true;
            // one decode for both kinds of lane (the code chosen per lane),
            // so the warp does not run the two in turn
            if (want_dist || want_lit) {
                const bool dd = want_dist;
                valid = decode_sym(ln.bb, dd ? sm.dtab : sm.ltab, dd ? sm.dcount : sm.lcount,
                                   dd ? sm.dsym : sm.lsym, dd ? sm.dfirst : sm.lfirst,
                                   dd ? sm.dindex : sm.lindex, &sym, &clen);
            }
            const unsigned eobm = __ballot_sync(0xffffffffu, want_lit && valid && sym == 256);
            const uint32_t e = eobm ? __ffs(eobm) - 1 : 32;
            // a bad code stops the round at its lane if that lane would act:
            // distance lanes always, literal lanes before end-of-block
            const unsigned badm =
                __ballot_sync(0xffffffffu, !valid && (want_dist || (want_lit && lane < e)));
            const uint32_t first_bad = badm ? __ffs(badm) - 1 : 32;
            const bool act = (want_dist || (want_lit && lane <= e)) && lane <= first_bad;
            uint32_t L = 0, xb = 0, d = 0;
            int st = CUDEC_OK;
            if (act) {
                if (!valid) {
                    st = CUDEC_ERR_CORRUPT_INPUT;
                } else if (want_dist) {
                    xb = kDExtra[sym];
                    d = kDBase[sym] + (static_cast<uint32_t>(ln.bb >> clen) & ((1u << xb) - 1));
                } else if (sym < 256) {
                    L = 1;
                } else if (sym > 256) {
                    if (sym > 285) {
                        st = CUDEC_ERR_CORRUPT_INPUT;
                    } else {
                        xb = kLExtra[sym - 257];
                        L = kLBase[sym - 257] +
                            (static_cast<uint32_t>(ln.bb >> clen) & ((1u << xb) - 1));
                    }
                }
            }
            uint32_t incl = L;
#pragma unroll
            for (uint32_t k = 1; k < 32; k <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, incl, k);
                if (lane >= k) incl += o;
            }
            const uint32_t p = pos + incl - L;
            if (act && st == CUDEC_OK) {
                if (L) {
                    if (p + L > kPageMax) st = CUDEC_ERR_CORRUPT_INPUT;
                    else if (p + L > room) st = CUDEC_ERR_OUTPUT_TOO_SMALL;
                }
                if (want_dist && d > ppos) st = CUDEC_ERR_CORRUPT_INPUT;
            }
            if (act && st == CUDEC_OK) ln.consume(clen + xb);
            const uint32_t rev = ln.refill(lane);
            const int s = first_event(st != CUDEC_OK, st, rev, lane);
            if (s != CUDEC_OK) return s;
            // literals of this round
            if (act && want_lit && sym < 256) out[p] = static_cast<uint8_t>(sym);
            __syncwarp();
            // copies whose distance arrived: frontier order by position
            bool go = act && want_dist;
            while (__any_sync(0xffffffffu, go)) {
                uint32_t front = go ? ppos : 0xFFFFFFFFu;
#pragma unroll
                for (uint32_t k = 16; k; k >>= 1) {
                    const uint32_t o = __shfl_xor_sync(0xffffffffu, front, k);
                    front = o < front ? o : front;
                }
                if (go) {
                    const uint32_t src_end = ppos - d + plen;
                    const uint32_t need = src_end < ppos ? src_end : ppos;
                    if (need <= front) {
                        page_copy(out, ppos, plen, d);
                        go = false;
                    }
                }
                __syncwarp();
            }
            if (act && want_dist) pend = false;
            if (act && want_lit && sym > 256) {
                pend = true;
                ppos = p;
                plen = L;
            }
            pos += __shfl_sync(0xffffffffu, incl, 31);
            if (e < 32) eob = true;
            if (eob && !__any_sync(0xffffffffu, pend)) break;
        }
    }
    if (ln.cursor != ln.words) return CUDEC_ERR_CORRUPT_INPUT;
    __syncwarp();
    *written = pos;
    return CUDEC_OK;
}

}  // namespace gdf
}  // namespace cdb
