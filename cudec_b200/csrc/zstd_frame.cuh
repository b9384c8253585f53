// One Zstd frame decoded by one warp: the frame loop, literals, sequence
// batches and their execution (RFC 8878 subset of the reference, statuses as
// iderex/cudec tests/zstd_twin_driver.h:178-390 maps them). Shared by the
// Zstd batch entry and the mixed-format persistent kernel.
#pragma once

#include <cstdint>

#include "cudec.h"
#include "zstd_kernel.cuh"

namespace cdb {
namespace zstd {

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

__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
#pragma unroll
    for (int d = 16; d; d >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, v, d);
        v = o < v ? o : v;
    }
    return v;
}

// Warp-strided byte copy / fill (no overlap between src and dst ranges).
__device__ __forceinline__ void warp_copy(uint8_t* dst, const uint8_t* src, uint64_t n,
                                          uint32_t lane) {
    for (uint64_t i = lane; i < n; i += 32) dst[i] = src[i];
}
__device__ __forceinline__ void warp_fill(uint8_t* dst, uint8_t b, uint64_t n, uint32_t lane) {
    for (uint64_t i = lane; i < n; i += 32) dst[i] = b;
}

// Decode one frame; every lane returns the same status and *written.
__device__ inline int decode_frame(const uint8_t* f, uint64_t N, uint8_t* dst, uint64_t cap,
                            WarpSmem& w, uint8_t* litbuf, uint32_t lane, uint64_t* written) {
    *written = 0;
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
    if (fcs_size == 0) return CUDEC_ERR_UNSUPPORTED;
    const unsigned wbytes = single ? 0 : 1;
    const uint64_t hsz = 5 + wbytes + fcs_size;
    if (N < hsz) return CUDEC_ERR_CORRUPT_INPUT;
    uint64_t fcs = rd_le(f + 5 + wbytes, fcs_size);
    if (fcs_size == 2) fcs += 256;
    uint64_t window;
    if (single) {
        window = fcs;
    } else {
        const uint64_t e = f[5] >> 3, m = f[5] & 7, base = 1ull << (10 + e);
        window = base + (base / 8) * m;
        if (window > kMaxWindow) return CUDEC_ERR_UNSUPPORTED;
    }
    if (fcs > cap) return CUDEC_ERR_OUTPUT_TOO_SMALL;
    const uint64_t bmax = window < kLitSlot ? window : kLitSlot;

    Tables t;
    for (int k = 0; k < 3; ++k) {
        t.size[k] = 0;
        t.log[k] = 0;
        t.present[k] = false;
    }
    t.huf_log = 0;
    t.huf_present = false;
    uint64_t rep0 = 1, rep1 = 4, rep2 = 8;
    uint64_t pos = hsz, out = 0;
    for (;;) {
        if (N - pos < 3) return CUDEC_ERR_CORRUPT_INPUT;
        const uint32_t raw = static_cast<uint32_t>(rd_le(f + pos, 3));
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
                lit_src = litbuf;
                lused = lhs + csize;
            }
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
            uint64_t lp = 0;          // literals consumed
            int exec = CUDEC_OK;      // first execution verdict
            if (nseq) {
                if (nseq > bmax / 3) return CUDEC_ERR_CORRUPT_INPUT;
                if (rem <= cnum) return CUDEC_ERR_CORRUPT_INPUT;
                const unsigned modes = sec[cnum++];
                if (modes & 3) return CUDEC_ERR_CORRUPT_INPUT;
                const unsigned mode[3] = {(modes >> 6) & 3, (modes >> 4) & 3, (modes >> 2) & 3};
                sec += cnum;
                rem -= cnum;
                for (unsigned fld = 0; fld < 3; ++fld) {
                    uint64_t u;
                    if (!seq_table(w, t, fld, mode[fld], sec, rem, &u, lane))
                        return CUDEC_ERR_CORRUPT_INPUT;
                    sec += u;
                    rem -= u;
                }
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
                uint64_t cur = out;   // output position including this batch
                for (uint32_t i0 = 0; i0 < nseq; i0 += 32) {
                    const uint32_t cnt = nseq - i0 < 32 ? nseq - i0 : 32;
                    // my sequence of this batch
                    uint64_t m_o = 0, m_ll = 0, m_lsrc = 0, m_off = 0, m_ml = 0;
                    bool m_has = false;
                    for (uint32_t k = 0; k < cnt; ++k) {
                        const uint32_t i = i0 + k;
                        if (sll >= t.size[0] || sof >= t.size[1] || sml >= t.size[2])
                            return CUDEC_ERR_CORRUPT_INPUT;
                        const uint32_t cl_ = w.fse[0][sll], co_ = w.fse[1][sof], cm_ = w.fse[2][sml];
                        const unsigned cl = (cl_ >> 8) & 0xff, co = (co_ >> 8) & 0xff,
                                       cm = (cm_ >> 8) & 0xff;
                        if (cl > 35 || co > 31 || cm > 52) return CUDEC_ERR_CORRUPT_INPUT;
                        uint64_t eo, em, el;
                        if (!r.read(co, &eo) || !r.read(ml_bits(cm), &em) || !r.read(ll_bits(cl), &el))
                            return CUDEC_ERR_CORRUPT_INPUT;
                        const uint64_t ov = (1ull << co) + eo;
                        const uint64_t ml = kMLBase[cm] + em;
                        const uint64_t ll = kLLBase[cl] + el;
                        if (i + 1 < nseq) {
                            if (!r.read(cl_ & 0xff, &v)) return CUDEC_ERR_CORRUPT_INPUT;
                            sll = (cl_ >> 16) + static_cast<uint32_t>(v);
                            if (!r.read(cm_ & 0xff, &v)) return CUDEC_ERR_CORRUPT_INPUT;
                            sml = (cm_ >> 16) + static_cast<uint32_t>(v);
                            if (!r.read(co_ & 0xff, &v)) return CUDEC_ERR_CORRUPT_INPUT;
                            sof = (co_ >> 16) + static_cast<uint32_t>(v);
                        }
                        if (exec != CUDEC_OK) continue;
                        // the driver's per-sequence checks, in its order
                        if (lp + ll > regen) {
                            exec = CUDEC_ERR_CORRUPT_INPUT;
                            continue;
                        }
                        const uint64_t o = cur, lsrc = lp;
                        lp += ll;
                        cur += ll;
                        uint64_t off;
                        if (ov > 3) {
                            off = ov - 3;
                            rep2 = rep1;
                            rep1 = rep0;
                            rep0 = off;
                        } else {
                            unsigned taken;
                            if (ll != 0) {
                                taken = static_cast<unsigned>(ov) - 1;
                                off = taken == 0 ? rep0 : taken == 1 ? rep1 : rep2;
                            } else if (ov < 3) {
                                taken = static_cast<unsigned>(ov);
                                off = taken == 1 ? rep1 : rep2;
                            } else {
                                taken = 3;
                                off = rep0 ? rep0 - 1 : 0;
                            }
                            if (off == 0) {
                                exec = CUDEC_ERR_CORRUPT_INPUT;
                                continue;
                            }
                            if (taken != 0) {
                                if (taken != 1) rep2 = rep1;
                                rep1 = rep0;
                                rep0 = off;
                            }
                        }
                        if (off > cur || off > window) {
                            exec = CUDEC_ERR_CORRUPT_INPUT;
                            continue;
                        }
                        if (cur > cap || ml > cap - cur) {
                            exec = CUDEC_ERR_OUTPUT_TOO_SMALL;
                            continue;
                        }
                        if (lane == k) {
                            m_o = o;
                            m_ll = ll;
                            m_lsrc = lsrc;
                            m_off = off;
                            m_ml = ml;
                            m_has = true;
                        }
                        cur += ml;
                    }
                    if (exec != CUDEC_OK) continue;  // keep decoding for stream faults
                    // ---- execute the batch ---------------------------------
                    if (m_has && m_ll) {
                        if (ltype == 1) {
                            for (uint64_t j = 0; j < m_ll; ++j) dst[m_o + j] = lit_byte;
                        } else {
                            copy_bytes(dst + m_o, lit_src + m_lsrc, m_ll);
                        }
                    }
                    __syncwarp();
                    bool pend = m_has && m_ml != 0;
                    const uint64_t ms = m_o + m_ll;
                    while (__any_sync(0xffffffffu, pend)) {
                        const uint64_t F = warp_min64(pend ? ms : ~0ull);
                        const uint64_t s0 = ms - m_off;
                        const uint64_t send = s0 + m_ml < ms ? s0 + m_ml : ms;
                        const bool ready = pend && (ms == F || send <= F);
                        if (ready) {
                            for (uint64_t j = 0; j < m_ml; ++j) dst[ms + j] = dst[s0 + j];
                            pend = false;
                        }
                        __syncwarp();
                    }
                }
                if (r.left != 0) return CUDEC_ERR_CORRUPT_INPUT;
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
    if (out != fcs) return CUDEC_ERR_CORRUPT_INPUT;
    if (csum) {
        if (N - pos < 4) return CUDEC_ERR_CORRUPT_INPUT;
        __syncwarp();
        uint32_t h = 0;
        if (lane == 0) h = static_cast<uint32_t>(xxh64_dev(dst, out));
        h = __shfl_sync(0xffffffffu, h, 0);
        if (h != static_cast<uint32_t>(rd_le(f + pos, 4))) return CUDEC_ERR_CORRUPT_INPUT;
        pos += 4;
    }
    if (pos != N) return CUDEC_ERR_CORRUPT_INPUT;
    *written = out;
    return CUDEC_OK;
}

}  // namespace zstd
}  // namespace cdb
