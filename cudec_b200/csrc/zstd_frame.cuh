// One Zstd frame decoded by one warp: the frame loop, literals, sequence
// batches and their execution (RFC 8878 subset of the reference, statuses as
// iderex/cudec tests/zstd_twin_driver.h:178-390 maps them). Shared by the
// Zstd batch entry and the mixed-format persistent kernel.
#pragma once

#include <cstdint>

#include "cudec.h"
#include "lz_warp_kernel.cuh"
#include "zstd_kernel.cuh"

namespace cdb {
namespace zstd {

// Profiling builds (-DCDB_PHASE_TIMING) accumulate per-phase SM cycles and
// event counts over all frames of a launch.
#ifdef CDB_PHASE_TIMING
__device__ unsigned long long zs_cycles[8];
__device__ unsigned long long zs_events[8];
#define ZS_T(v) const long long v = clock64()
#define ZS_ADD(i, t0) \
    if (lane == 0) atomicAdd(&zs_cycles[i], static_cast<unsigned long long>(clock64() - (t0)))
#define ZS_EV(i, n) \
    if (lane == 0) atomicAdd(&zs_events[i], static_cast<unsigned long long>(n))
#else
#define ZS_T(v)
#define ZS_ADD(i, t0)
#define ZS_EV(i, n)
#endif

// XXH64 of p[0, n) with seed 0 (public xxHash specification), one lane.
__device__ inline uint64_t xxh64_dev(const uint8_t* p, uint64_t n) {
    const uint64_t P1 = 11400714785074694791ull, P2 = 14029467366897019727ull,
                   P3 = 1609587929392839161ull, P4 = 9650029242287828579ull,
                   P5 = 2870177450012600261ull;
    auto rotl = [](uint64_t x, int r) { return (x << r) | (x >> (64 - r)); };
    auto round = [&](uint64_t acc, uint64_t lane) { return rotl(acc + lane * P2, 31) * P1; };
    uint64_t i = 0, h;
    if (n >= 32) {
        uint64_t v1 = P1 + P2, v2 = P2, v3 = 0, v4 = 0 - P1;
        for (; i + 32 <= n; i += 32) {
            v1 = round(v1, rd_le(p + i, 8));
            v2 = round(v2, rd_le(p + i + 8, 8));
            v3 = round(v3, rd_le(p + i + 16, 8));
            v4 = round(v4, rd_le(p + i + 24, 8));
        }
        h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
        h = (h ^ round(0, v1)) * P1 + P4;
        h = (h ^ round(0, v2)) * P1 + P4;
        h = (h ^ round(0, v3)) * P1 + P4;
        h = (h ^ round(0, v4)) * P1 + P4;
    } else {
        h = P5;
    }
    h += n;
    for (; i + 8 <= n; i += 8) {
        h ^= round(0, rd_le(p + i, 8));
        h = rotl(h, 27) * P1 + P4;
    }
    if (i + 4 <= n) {
        h ^= rd_le(p + i, 4) * P1;
        h = rotl(h, 23) * P2 + P3;
        i += 4;
    }
    for (; i < n; ++i) {
        h ^= p[i] * P5;
        h = rotl(h, 11) * P1;
    }
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
}

// Copies and fills. Sources are read with ordinary (coherent) loads: literal
// bytes in the workspace and match sources in the destination were written
// by this warp earlier in the same launch. A 16-byte window of a source is
// two aligned block loads and a funnel shift (lzw::ld16_output), never a load
// of a block that holds no requested byte.

constexpr uint64_t kLaneCopyMax = 128;  // longer runs are copied by the whole warp

// The whole warp copies n bytes src -> dst (non-overlapping): destination-
// aligned 16-byte stores, four in flight per lane.
__device__ __forceinline__ void warp_copy(uint8_t* dst, const uint8_t* src, uint64_t n,
                                          uint32_t lane) {
    uint64_t head = (16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15;
    if (head > n) head = n;
    if (lane < head) dst[lane] = src[lane];
    const uint64_t body_end = head + ((n - head) & ~15ull);
    uint64_t k = head + 16ull * lane;
    for (; k + 3 * 512 < body_end; k += 4 * 512) {
        const uint4 v0 = lzw::ld16_output(src + k, 16), v1 = lzw::ld16_output(src + k + 512, 16);
        const uint4 v2 = lzw::ld16_output(src + k + 1024, 16);
        const uint4 v3 = lzw::ld16_output(src + k + 1536, 16);
        *reinterpret_cast<uint4*>(dst + k) = v0;
        *reinterpret_cast<uint4*>(dst + k + 512) = v1;
        *reinterpret_cast<uint4*>(dst + k + 1024) = v2;
        *reinterpret_cast<uint4*>(dst + k + 1536) = v3;
    }
    for (; k < body_end; k += 512) *reinterpret_cast<uint4*>(dst + k) = lzw::ld16_output(src + k, 16);
    if (body_end + lane < n) dst[body_end + lane] = src[body_end + lane];
}

// The whole warp writes n copies of byte b.
__device__ __forceinline__ void warp_fill(uint8_t* dst, uint8_t b, uint64_t n, uint32_t lane) {
    uint64_t head = (16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15;
    if (head > n) head = n;
    if (lane < head) dst[lane] = b;
    const uint64_t body_end = head + ((n - head) & ~15ull);
    const uint32_t w = 0x01010101u * b;
    const uint4 v = make_uint4(w, w, w, w);
    for (uint64_t k = head + 16ull * lane; k < body_end; k += 512)
        *reinterpret_cast<uint4*>(dst + k) = v;
    if (body_end + lane < n) dst[body_end + lane] = b;
}

// One lane copies n (<= kLaneCopyMax) bytes src -> dst, 16 at a time.
__device__ __forceinline__ void lane_copy(uint8_t* dst, const uint8_t* src, uint64_t n) {
    for (uint64_t k = 0; k < n; k += 16) {
        const uint32_t m = n - k < 16 ? static_cast<uint32_t>(n - k) : 16u;
        lzw::st16_global(dst + k, lzw::ld16_words(src + k, m), m);
    }
}

__device__ __forceinline__ void lane_fill(uint8_t* dst, uint8_t b, uint64_t n) {
    const uint32_t w = 0x01010101u * b;
    const uint4 v = make_uint4(w, w, w, w);
    for (uint64_t k = 0; k < n; k += 16)
        lzw::st16_global(dst + k, v, n - k < 16 ? static_cast<uint32_t>(n - k) : 16u);
}

// One lane writes the match dst[ms, ms + n) at offset off (every byte before
// ms is written; off is below the window, under 2^32), 16 bytes at a time: the
// first piece is one read and one write in every lane (lzw::period16 for
// periods under 16 bytes), the rest a plain copy at lzw::rest_distance(off).
__device__ __forceinline__ void lane_match(uint8_t* dst, uint64_t ms, uint64_t n, uint64_t off) {
    uint8_t* o = dst + ms;
    const uint32_t f = static_cast<uint32_t>(off);
    const uint32_t m0 = n < 16 ? static_cast<uint32_t>(n) : 16u;
    lzw::st16_global(o, lzw::period16(lzw::ld16_words(o - off, f < 16 ? f : m0), f), m0);
    const uint64_t d = lzw::rest_distance(f);
    for (uint64_t k = 16; k < n; k += 16) {
        const uint32_t m = n - k < 16 ? static_cast<uint32_t>(n - k) : 16u;
        lzw::st16_global(o + k, lzw::ld16_words(o + k - d, m), m);
    }
}

// Decode the frame at the start of f[0, N); every lane returns the same
// status, *written and *consumed (the frame's bytes). Bytes after the frame
// are not looked at. Wide: the frame-sequence reading, which also takes a
// frame without a content size (its output bounded by cap alone) and any
// window whose log is at most kMaxWindowLogSeq; otherwise the reference's
// subset.
template <bool Wide>
__device__ inline int decode_frame_part(const uint8_t* f, uint64_t N, uint8_t* dst, uint64_t cap,
                                        WarpSmem& w, uint8_t* litbuf, uint32_t lane,
                                        uint64_t* written, uint64_t* consumed) {
    *written = 0;
    *consumed = 0;
    if (N < 4) return CUDEC_ERR_CORRUPT_INPUT;
    const uint32_t magic = static_cast<uint32_t>(rd_le(f, 4));
    if (magic != 0xFD2FB528u) {
        if (magic >= 0x184D2A50u && magic <= 0x184D2A5Fu) return CUDEC_ERR_UNSUPPORTED;
        return CUDEC_ERR_CORRUPT_INPUT;
    }
    if (N < 5) return CUDEC_ERR_CORRUPT_INPUT;
    const unsigned d = f[4], fcs_flag = d >> 6, single = (d >> 5) & 1, csum = (d >> 2) & 1;
    if (d & 8) return CUDEC_ERR_CORRUPT_INPUT;
    if (d & 3) return CUDEC_ERR_UNSUPPORTED;
    const unsigned fcs_size = fcs_flag == 0 ? (single ? 1 : 0)
                            : fcs_flag == 1 ? 2 : fcs_flag == 2 ? 4 : 8;
    const bool has_fcs = fcs_size != 0;  // single segment implies a content size
    if (!has_fcs && !Wide) return CUDEC_ERR_UNSUPPORTED;
    const unsigned wbytes = single ? 0 : 1;
    const uint64_t hsz = 5 + wbytes + fcs_size;
    if (N < hsz) return CUDEC_ERR_CORRUPT_INPUT;
    uint64_t fcs = has_fcs ? rd_le(f + 5 + wbytes, fcs_size) : 0;
    if (fcs_size == 2) fcs += 256;
    uint64_t window;
    if (single) {
        window = fcs;
    } else {
        const uint64_t e = f[5] >> 3, m = f[5] & 7, base = 1ull << (10 + e);
        window = base + (base / 8) * m;
        if (!Wide && window > kMaxWindow) return CUDEC_ERR_UNSUPPORTED;
        if (Wide && 10 + e > kMaxWindowLogSeq) return CUDEC_ERR_UNSUPPORTED;
    }
    if (has_fcs && fcs > cap) return CUDEC_ERR_OUTPUT_TOO_SMALL;
    const uint64_t bmax = window < kLitSlot ? window : kLitSlot;

    Tables t;
    for (int k = 0; k < 3; ++k) {
        t.size[k] = 0;
        t.log[k] = 0;
        t.present[k] = false;
    }
    t.huf_log = 0;
    t.huf_present = false;
    // repeat offsets stay below 2^32 (offset codes are at most 31), so 32 bits
    uint32_t rep0 = 1, rep1 = 4, rep2 = 8;
    uint64_t pos = hsz, out = 0;
    for (;;) {
        if (N - pos < 3) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t raw = static_cast<uint32_t>(rd_le(f + pos, 3));
        ZS_EV(0, 1);
        const bool last = raw & 1;
        const unsigned btype = (raw >> 1) & 3;
        const uint32_t bsize = raw >> 3;
        if (btype == 3) return CUDEC_ERR_CORRUPT_INPUT;
        if (bsize > bmax) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t body = btype == 1 ? 1 : bsize;
        if (N - pos < 3ull + body) return CUDEC_ERR_CORRUPT_INPUT;
        const uint8_t* b = f + pos + 3;
        if (btype == 0) {
            if (bsize > cap - out) return CUDEC_ERR_OUTPUT_TOO_SMALL;
            warp_copy(dst + out, b, bsize, lane);
            out += bsize;
        } else if (btype == 1) {
            if (bsize > cap - out) return CUDEC_ERR_OUTPUT_TOO_SMALL;
            warp_fill(dst + out, b[0], bsize, lane);
            out += bsize;
        } else {
            // ---- literals section (src/zstd_literals.h:357-547) ----------
            if (body == 0) return CUDEC_ERR_CORRUPT_INPUT;
            const unsigned ltype = b[0] & 3, lfmt = (b[0] >> 2) & 3;
            uint64_t regen, csize = 0, lhs;
            unsigned streams = 0;
            if (ltype < 2) {
                unsigned hs = 1, sh = 3;
                if (lfmt == 1) { hs = 2; sh = 4; }
                else if (lfmt == 3) { hs = 3; sh = 4; }
                if (body < hs) return CUDEC_ERR_CORRUPT_INPUT;
                regen = rd_le(b, hs) >> sh;
                lhs = hs;
            } else {
                unsigned hs = 3, fb = 10;
                if (lfmt == 2) { hs = 4; fb = 14; }
                else if (lfmt == 3) { hs = 5; fb = 18; }
                if (body < hs) return CUDEC_ERR_CORRUPT_INPUT;
                const uint64_t rw = rd_le(b, hs), msk = (1ull << fb) - 1;
                regen = (rw >> 4) & msk;
                csize = (rw >> (4 + fb)) & msk;
                lhs = hs;
                streams = lfmt == 0 ? 1 : 4;
            }
            if (regen > bmax) return CUDEC_ERR_CORRUPT_INPUT;
            ZS_T(t_lit);
            const uint64_t after = body - lhs;
            const uint8_t* lit_src = nullptr;  // literal bytes (input or workspace)
            uint8_t lit_byte = 0;              // RLE literals
            uint64_t lused;
            if (ltype == 0) {
                if (regen > after) return CUDEC_ERR_CORRUPT_INPUT;
                lit_src = b + lhs;
                lused = lhs + regen;
            } else if (ltype == 1) {
                if (after < 1) return CUDEC_ERR_CORRUPT_INPUT;
                lit_byte = b[lhs];
                lused = lhs + 1;
            } else {
                if (csize > after) return CUDEC_ERR_CORRUPT_INPUT;
                const uint8_t* pay = b + lhs;
                uint64_t psize = csize;
                if (ltype == 2) {
                    unsigned cnt, tl;
                    uint64_t used;
                    if (!huf_weights(pay, psize, w, lane, &cnt, &tl, &used))
                        return CUDEC_ERR_CORRUPT_INPUT;
                    if (!huf_build(w, cnt, tl, lane)) return CUDEC_ERR_CORRUPT_INPUT;
                    t.huf_log = tl;
                    t.huf_present = true;
                    pay += used;
                    psize -= used;
                } else if (!t.huf_present) {
                    return CUDEC_ERR_CORRUPT_INPUT;
                }
                if (psize == 0) return CUDEC_ERR_CORRUPT_INPUT;
                ZS_T(t_huf);
                bool ok;
                if (streams == 1) {
                    bool mine = true;
                    if (lane == 0) mine = huf_stream(pay, psize, w.huf, t.huf_log, litbuf, regen);
                    ok = __shfl_sync(0xffffffffu, mine ? 1 : 0, 0) != 0;
                } else {
                    if (psize < 10) return CUDEC_ERR_CORRUPT_INPUT;
                    if (regen < 6) return CUDEC_ERR_CORRUPT_INPUT;
                    const uint64_t c0 = rd_le(pay, 2), c1 = rd_le(pay + 2, 2), c2 = rd_le(pay + 4, 2);
                    const uint64_t sb = psize - 6;
                    if (c0 + c1 + c2 >= sb) return CUDEC_ERR_CORRUPT_INPUT;
                    const uint64_t seg = (regen + 3) / 4;
                    bool mine = true;
                    if (lane < 4) {
                        const uint64_t cs = lane == 0 ? c0 : lane == 1 ? c1 : lane == 2 ? c2
                                          : sb - c0 - c1 - c2;
                        const uint64_t so = lane == 0 ? 0 : lane == 1 ? c0 : lane == 2 ? c0 + c1
                                          : c0 + c1 + c2;
                        const uint64_t rg = lane < 3 ? seg : regen - 3 * seg;
                        mine = huf_stream(pay + 6 + so, cs, w.huf, t.huf_log, litbuf + lane * seg, rg);
                    }
                    ok = __all_sync(0xffffffffu, mine);
                }
                if (!ok) return CUDEC_ERR_CORRUPT_INPUT;
                __syncwarp();
                ZS_ADD(1, t_huf);
                ZS_EV(2, regen);
                ZS_EV(3, streams);
                lit_src = litbuf;
                lused = lhs + csize;
            }
            ZS_ADD(0, t_lit);
            // ---- sequences section (src/zstd_seq.h:320-676) ---------------
            const uint8_t* sec = b + lused;
            uint64_t rem = body - lused;
            if (rem == 0) return CUDEC_ERR_CORRUPT_INPUT;
            uint32_t nseq;
            uint64_t cnum = 1;
            if (sec[0] < 128) {
                nseq = sec[0];
            } else if (sec[0] < 255) {
                if (rem < 2) return CUDEC_ERR_CORRUPT_INPUT;
                nseq = ((static_cast<uint32_t>(sec[0]) - 128) << 8) + sec[1];
                cnum = 2;
            } else {
                if (rem < 3) return CUDEC_ERR_CORRUPT_INPUT;
                nseq = static_cast<uint32_t>(sec[1]) + (static_cast<uint32_t>(sec[2]) << 8) + 0x7F00u;
                cnum = 3;
            }
            uint32_t lp = 0;          // literals consumed (at most a block)
            int exec = CUDEC_OK;      // first execution verdict
            if (nseq) {
                if (nseq > bmax / 3) return CUDEC_ERR_CORRUPT_INPUT;
                if (rem <= cnum) return CUDEC_ERR_CORRUPT_INPUT;
                const unsigned modes = sec[cnum++];
                if (modes & 3) return CUDEC_ERR_CORRUPT_INPUT;
                const unsigned mode[3] = {(modes >> 6) & 3, (modes >> 4) & 3, (modes >> 2) & 3};
                sec += cnum;
                rem -= cnum;
                ZS_T(t_tab);
                for (unsigned fld = 0; fld < 3; ++fld) {
                    uint64_t u;
                    if (!seq_table(w, t, fld, mode[fld], sec, rem, &u, lane))
                        return CUDEC_ERR_CORRUPT_INPUT;
                    sec += u;
                    rem -= u;
                }
                ZS_ADD(2, t_tab);
                ZS_EV(1, nseq);
                if (rem == 0) return CUDEC_ERR_CORRUPT_INPUT;
                BitIn r;
                if (!r.start(sec, rem)) return CUDEC_ERR_CORRUPT_INPUT;
                uint64_t v;
                uint32_t sll, sof, sml;
                if (!r.read(t.log[0], &v)) return CUDEC_ERR_CORRUPT_INPUT;
                sll = static_cast<uint32_t>(v);
                if (!r.read(t.log[1], &v)) return CUDEC_ERR_CORRUPT_INPUT;
                sof = static_cast<uint32_t>(v);
                if (!r.read(t.log[2], &v)) return CUDEC_ERR_CORRUPT_INPUT;
                sml = static_cast<uint32_t>(v);
                // from here the stream is read by absolute position
                BitWin bw;
                bw.init(sec, rem);
                int32_t bp = static_cast<int32_t>(r.left);  // at most 8 x 128 KiB bits
                uint64_t cur = out;   // output position including this batch
                for (uint32_t i0 = 0; i0 < nseq; i0 += 32) {
                    ZS_T(t_dec);
                    const uint32_t cnt = nseq - i0 < 32 ? nseq - i0 : 32;
                    // my sequence of this batch
                    uint64_t m_o = 0;
                    uint32_t m_ll = 0, m_lsrc = 0, m_off = 0, m_ml = 0;
                    bool m_has = false, m_zero = false;
                    // Branch-light: each sequence's bits come from one window
                    // at the absolute position bp with no per-read checks; bp
                    // going negative marks an over-read, tested once per
                    // batch (a stream fault is a reject whatever the
                    // execution verdicts were). Only the bitstream and the
                    // repeat offsets are serial; positions and the execution
                    // checks follow per batch, lane-parallel.
                    for (uint32_t k = 0; k < cnt; ++k) {
                        const uint32_t i = i0 + k;
                        // States stay below their table's size and codes
                        // within their field's range by construction: every
                        // table comes from seq_table (symbols checked against
                        // the field's maximum) and fse_build (a cell's next
                        // state base + its bits is below the table size), so
                        // the reference's per-sequence range checks cannot
                        // fire here; the masks only keep indexes in place.
                        const uint32_t cl_ = w.fse[0][sll & (kFseCells - 1)],
                                       co_ = w.fse[1][sof & (kFseCells - 1)],
                                       cm_ = w.fse[2][sml & (kFseCells - 1)];
                        const unsigned cl = (cl_ >> 8) & 0x3f, co = (co_ >> 8) & 0x1f,
                                       cm = (cm_ >> 8) & 0x3f;
                        const uint32_t lcode = kLLCode[cl], mcode = kMLCode[cm];
                        const unsigned mlb = mcode >> 24, llb = lcode >> 24;
                        const unsigned xb = co + mlb + llb;  // extra bits, at most 63
                        const bool upd = i + 1 < nseq;
                        const unsigned lb = cl_ & 0xff, mb = cm_ & 0xff, ob = co_ & 0xff;
                        const unsigned sb = upd ? lb + mb + ob : 0u;  // state bits
                        // offset, match and literal extras, then the ll, ml
                        // and of state bits, in stream order, from the top
                        uint32_t hi, lo;
                        bw.window(bp, &hi, &lo);
                        // offsets below 32 need no general field(): the offset
                        // and match extras start there, and the state fields
                        // come from the window moved past the extras
                        const uint32_t eo = __funnelshift_rc(hi, 0u, 32 - co);
                        const uint32_t em =
                            __funnelshift_rc(__funnelshift_lc(lo, hi, co), 0u, 32 - mlb);
                        const uint32_t el = BitWin::field(hi, lo, co + mlb, llb);
                        uint32_t h2, l2;
                        if (xb + sb <= 64) {
                            h2 = xb < 32 ? __funnelshift_lc(lo, hi, xb)
                                         : __funnelshift_lc(0u, lo, xb - 32);
                            l2 = xb < 32 ? lo << xb : 0u;
                        } else {  // long extras: the state bits from the next window
                            bw.window(bp - static_cast<int32_t>(xb), &h2, &l2);
                        }
                        const uint32_t ul = __funnelshift_rc(h2, 0u, 32 - lb);
                        const uint32_t um =
                            __funnelshift_rc(__funnelshift_lc(l2, h2, lb), 0u, 32 - mb);
                        const uint32_t uo =
                            __funnelshift_rc(__funnelshift_lc(l2, h2, lb + mb), 0u, 32 - ob);
                        bp -= static_cast<int32_t>(xb + sb);
                        if (upd) {
                            sll = (cl_ >> 16) + ul;
                            sml = (cm_ >> 16) + um;
                            sof = (co_ >> 16) + uo;
                        }
                        // values fit 32 bits: a code below 32 plus its extra
                        // bits, lengths below 2^17 + 2^16
                        const uint32_t ov = (1u << co) + eo;
                        const uint32_t ml = (mcode & 0xffffffu) + em;
                        const uint32_t ll = (lcode & 0xffffffu) + el;
                        // repeat offsets, the one serial part of the
                        // bookkeeping (state after a faulty sequence is
                        // never used, so it is updated unconditionally)
                        const bool nrep = ov > 3;
                        const unsigned tk = ll != 0 ? ov - 1 : (ov < 3 ? ov : 3u);
                        const uint32_t rsel = tk == 0 ? rep0 : tk == 1 ? rep1 : tk == 2 ? rep2
                                            : (rep0 ? rep0 - 1 : 0);
                        const uint32_t off = nrep ? ov - 3 : rsel;
                        const bool shift1 = nrep || tk >= 1, shift2 = nrep || tk >= 2;
                        rep2 = shift2 ? rep1 : rep2;
                        rep1 = shift1 ? rep0 : rep1;
                        rep0 = shift1 ? off : rep0;
                        if (lane == k) {
                            m_ll = ll;
                            m_off = off;
                            m_ml = ml;
                            m_zero = !nrep && off == 0;
                        }
                    }
                    if (bp < 0) return CUDEC_ERR_CORRUPT_INPUT;
                    if (exec != CUDEC_OK) continue;  // keep decoding for stream faults
                    // Positions by warp scans and the driver's per-sequence
                    // checks lane-parallel, each in its order; the first
                    // failing lane's verdict is the serial decoder's first
                    // verdict (nothing after a failure is used).
                    m_has = lane < cnt;
                    uint32_t lsum = m_has ? m_ll : 0u, tsum = m_has ? m_ll + m_ml : 0u;
#pragma unroll
                    for (uint32_t d = 1; d < 32; d <<= 1) {
                        const uint32_t a = __shfl_up_sync(0xffffffffu, lsum, d);
                        const uint32_t b2 = __shfl_up_sync(0xffffffffu, tsum, d);
                        if (lane >= d) {
                            lsum += a;
                            tsum += b2;
                        }
                    }
                    m_lsrc = lp + lsum - (m_has ? m_ll : 0u);
                    m_o = cur + tsum - (m_has ? m_ll + m_ml : 0u);
                    const uint64_t cur2 = m_o + m_ll;
                    const int v = !m_has ? CUDEC_OK
                                : static_cast<uint64_t>(m_lsrc) + m_ll > regen ? CUDEC_ERR_CORRUPT_INPUT
                                : m_zero ? CUDEC_ERR_CORRUPT_INPUT
                                : (m_off > cur2 || m_off > window) ? CUDEC_ERR_CORRUPT_INPUT
                                : (cur2 > cap || m_ml > cap - cur2) ? CUDEC_ERR_OUTPUT_TOO_SMALL
                                : CUDEC_OK;
                    const unsigned fails = __ballot_sync(0xffffffffu, v != CUDEC_OK);
                    if (fails) {
                        exec = __shfl_sync(0xffffffffu, v, __ffs(fails) - 1);
                        continue;  // keep decoding for stream faults
                    }
                    lp += __shfl_sync(0xffffffffu, lsum, 31);
                    cur += __shfl_sync(0xffffffffu, tsum, 31);
                    ZS_ADD(3, t_dec);
                    ZS_T(t_exe);
                    // ---- execute the batch ---------------------------------
                    // literal runs: short ones per lane, long ones by the warp
                    const bool lit_long = m_has && m_ll > kLaneCopyMax;
                    if (m_has && m_ll && !lit_long) {
                        if (ltype == 1) lane_fill(dst + m_o, lit_byte, m_ll);
                        else lane_copy(dst + m_o, lit_src + m_lsrc, m_ll);
                    }
                    for (unsigned lm = __ballot_sync(0xffffffffu, lit_long); lm; lm &= lm - 1) {
                        const int l = __ffs(lm) - 1;
                        const uint64_t o = __shfl_sync(0xffffffffu, m_o, l);
                        const uint64_t n = __shfl_sync(0xffffffffu, m_ll, l);
                        const uint64_t sr = __shfl_sync(0xffffffffu, m_lsrc, l);
                        if (ltype == 1) warp_fill(dst + o, lit_byte, n, lane);
                        else warp_copy(dst + o, lit_src + sr, n, lane);
                    }
                    __syncwarp();
                    // matches in rounds: a match goes once no unfinished
                    // match's output overlaps the bytes its source reads in
                    // this batch ([rs, re), relative to the batch start b0;
                    // earlier output and every literal are written). Match
                    // starts grow with the lane, so the unfinished matches
                    // starting below re are the pending lanes among a prefix
                    // of lanes, and the last of them ending by rs clears the
                    // source. The lowest unfinished match always clears.
                    bool pend = m_has && m_ml != 0;
                    const uint64_t ms = m_o + m_ll;
                    const uint64_t b0 = __shfl_sync(0xffffffffu, m_o, 0);
                    const uint32_t rms = m_has ? static_cast<uint32_t>(ms - b0) : ~0u;
                    const uint32_t rme = rms + static_cast<uint32_t>(m_ml);
                    uint32_t rs = 0, re = 0;
                    if (pend) {
                        const uint64_t s0 = ms - m_off;
                        const uint64_t e0 = s0 + m_ml < ms ? s0 + m_ml : ms;
                        rs = s0 > b0 ? static_cast<uint32_t>(s0 - b0) : 0u;
                        re = e0 > b0 ? static_cast<uint32_t>(e0 - b0) : 0u;
                    }
                    while (__any_sync(0xffffffffu, pend)) {
                        const unsigned pm = __ballot_sync(0xffffffffu, pend);
                        uint32_t l = 0;  // the last lane whose match starts below re
#pragma unroll
                        for (uint32_t st = 16; st; st >>= 1) {
                            const uint32_t c = l + st;
                            if (__shfl_sync(0xffffffffu, rms, c) < re) l = c;
                        }
                        const bool below = __shfl_sync(0xffffffffu, rms, 0) < re;
                        const unsigned cand =
                            below ? pm & (l == 31 ? 0xffffffffu : ((2u << l) - 1)) : 0u;
                        const uint32_t last = cand ? 31 - __clz(cand) : 0u;
                        const uint32_t last_end = __shfl_sync(0xffffffffu, rme, last);
                        const bool ready = pend && (re <= rs || cand == 0 || last_end <= rs);
                        if (ready && m_ml <= kLaneCopyMax) {
                            lane_match(dst, ms, m_ml, m_off);
                            pend = false;
                        }
                        for (unsigned lm = __ballot_sync(0xffffffffu, ready && pend); lm;
                             lm &= lm - 1) {
                            const int l = __ffs(lm) - 1;
                            lzw::coop_match(dst, __shfl_sync(0xffffffffu, ms, l),
                                            __shfl_sync(0xffffffffu, m_ml, l),
                                            static_cast<uint32_t>(__shfl_sync(0xffffffffu, m_off, l)),
                                            w.period, lane);
                            if (lane == static_cast<uint32_t>(l)) pend = false;
                        }
                        __syncwarp();
                    }
                    ZS_ADD(4, t_exe);
                }
                if (bp != 0) return CUDEC_ERR_CORRUPT_INPUT;
                if (exec != CUDEC_OK) return exec;
                out = cur;
            }
            // trailing literals
            const uint64_t tail = regen - lp;
            if (out > cap || tail > cap - out) return CUDEC_ERR_OUTPUT_TOO_SMALL;
            if (ltype == 1) warp_fill(dst + out, lit_byte, tail, lane);
            else warp_copy(dst + out, lit_src + lp, tail, lane);
            out += tail;
            __syncwarp();
        }
        __syncwarp();  // this block's bytes are visible to every lane
        pos += 3 + body;
        if (last) break;
    }
    if (has_fcs && out != fcs) return CUDEC_ERR_CORRUPT_INPUT;
    if (csum) {
        if (N - pos < 4) return CUDEC_ERR_CORRUPT_INPUT;
        __syncwarp();
        uint32_t h = 0;
        ZS_T(t_ck);
        if (lane == 0) h = static_cast<uint32_t>(xxh64_dev(dst, out));
        ZS_ADD(6, t_ck);
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h != static_cast<uint32_t>(rd_le(f + pos, 4))) return CUDEC_ERR_CORRUPT_INPUT;
        pos += 4;
    }
    *written = out;
    *consumed = pos;
    return CUDEC_OK;
}

// One frame per chunk, the reference's rule (src/zstd_frame.h:196-409):
// bytes after the frame are CORRUPT_INPUT, a skippable frame UNSUPPORTED.
__device__ inline int decode_frame(const uint8_t* f, uint64_t N, uint8_t* dst, uint64_t cap,
                                   WarpSmem& w, uint8_t* litbuf, uint32_t lane,
                                   uint64_t* written) {
    uint64_t out = 0, used = 0;
    *written = 0;
    const int st = decode_frame_part<false>(f, N, dst, cap, w, litbuf, lane, &out, &used);
    if (st != CUDEC_OK) return st;
    if (used != N) return CUDEC_ERR_CORRUPT_INPUT;
    *written = out;
    return CUDEC_OK;
}

// A chunk of concatenated frames, as libzstd's ZSTD_decompress reads a
// buffer with its default limits (the reference's subset ladder,
// docs/MASTERPLAN.md:1286-1296, rungs 1-3 up to that limit): skippable
// frames (magic 0x184D2A50-5F, 4-byte size) are skipped, and each Zstd frame
// decodes after the previous one's output, with or without a content size,
// with any window up to a log of kMaxWindowLogSeq (a dictionary id stays
// UNSUPPORTED);
// fewer than 4 bytes left, or a skippable frame running past the chunk, is
// CORRUPT_INPUT.
__device__ inline int decode_frames(const uint8_t* f, uint64_t N, uint8_t* dst, uint64_t cap,
                                    WarpSmem& w, uint8_t* litbuf, uint32_t lane,
                                    uint64_t* written) {
    *written = 0;
    uint64_t pos = 0, out = 0;
    while (pos < N) {
        if (N - pos < 4) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t magic = static_cast<uint32_t>(rd_le(f + pos, 4));
        if (magic >= 0x184D2A50u && magic <= 0x184D2A5Fu) {
            if (N - pos < 8) return CUDEC_ERR_CORRUPT_INPUT;
            const uint64_t sz = rd_le(f + pos + 4, 4);
            if (sz > N - pos - 8) return CUDEC_ERR_CORRUPT_INPUT;
            pos += 8 + sz;
            continue;
        }
        uint64_t fo = 0, used = 0;
        const int st = decode_frame_part<true>(f + pos, N - pos, dst + out, cap - out, w,
                                               litbuf, lane, &fo, &used);
        if (st != CUDEC_OK) return st;
        out += fo;
        pos += used;
    }
    *written = out;
    return CUDEC_OK;
}

}  // namespace zstd
}  // namespace cdb
