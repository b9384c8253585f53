/* ORACLE — test infrastructure, not part of the product.
 *
 * Plain-C, serial restatement of the reference's Zstd frame decode (the v1
 * subset of iderex/cudec), used by tests/ as the checker for the GPU Zstd
 * path. It follows, unit by unit:
 *   frame/block headers, subset gate, checksum  src/zstd_frame.h:196-409
 *   backward bit reader (strict, no reads past the start)
 *                                               src/zstd_bitstream.h:481-638
 *   FSE description, table spread, 2-state decode  src/zstd_fse.h:259-676
 *   Huffman weights (direct / FSE), table build  src/zstd_huf.h:198-460
 *   literals section (raw/RLE/compressed/treeless, 1 or 4 streams, table log
 *   capped at 11)                               src/zstd_literals.h:211-547
 *   sequences header, tables, 3-state decode    src/zstd_seq.h:320-676
 *   repeat offsets                              src/zstd_repcode.h:98-184
 *   block loop + execution + status mapping     tests/zstd_twin_driver.h:178-390
 * XXH64 is restated from the public xxHash specification.
 *
 * Pinned against the reference's own twin driver (oracle/_ref) and libzstd
 * in tests/test_zstd_oracle.py. Status values are cudec_status.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { Z_OK = 0, Z_CORRUPT = 2, Z_TOO_SMALL = 3, Z_CUDA = 4, Z_UNSUPPORTED = 6 };

static unsigned z_hibit(uint32_t v) {
    unsigned h = 0;
    for (unsigned b = 0; b < 32; b++)
        if ((v >> b) & 1u) h = b;
    return h;
}

static uint64_t z_le(const uint8_t* p, unsigned n) {
    uint64_t v = 0;
    for (unsigned i = 0; i < n; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

/* ---------------- XXH64 ---------------------------------------------- */
static uint64_t x_rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static const uint64_t X1 = 11400714785074694791ull, X2 = 14029467366897019727ull,
                      X3 = 1609587929392839161ull, X4 = 9650029242287828579ull,
                      X5 = 2870177450012600261ull;
static uint64_t x_round(uint64_t acc, uint64_t lane) {
    acc += lane * X2;
    acc = x_rotl(acc, 31);
    return acc * X1;
}
static uint64_t x_merge(uint64_t acc, uint64_t v) {
    acc ^= x_round(0, v);
    return acc * X1 + X4;
}
uint64_t oracle_xxh64(const uint8_t* p, uint64_t n, uint64_t seed) {
    uint64_t i = 0, h;
    if (n >= 32) {
        uint64_t v1 = seed + X1 + X2, v2 = seed + X2, v3 = seed, v4 = seed - X1;
        for (; i + 32 <= n; i += 32) {
            v1 = x_round(v1, z_le(p + i, 8));
            v2 = x_round(v2, z_le(p + i + 8, 8));
            v3 = x_round(v3, z_le(p + i + 16, 8));
            v4 = x_round(v4, z_le(p + i + 24, 8));
        }
        h = x_rotl(v1, 1) + x_rotl(v2, 7) + x_rotl(v3, 12) + x_rotl(v4, 18);
        h = x_merge(h, v1);
        h = x_merge(h, v2);
        h = x_merge(h, v3);
        h = x_merge(h, v4);
    } else {
        h = seed + X5;
    }
    h += n;
    for (; i + 8 <= n; i += 8) {
        h ^= x_round(0, z_le(p + i, 8));
        h = x_rotl(h, 27) * X1 + X4;
    }
    if (i + 4 <= n) {
        h ^= (uint64_t)z_le(p + i, 4) * X1;
        h = x_rotl(h, 23) * X2 + X3;
        i += 4;
    }
    for (; i < n; i++) {
        h ^= p[i] * X5;
        h = x_rotl(h, 11) * X1;
    }
    h ^= h >> 33;
    h *= X2;
    h ^= h >> 29;
    h *= X3;
    h ^= h >> 32;
    return h;
}

/* ---------------- backward bit reader -------------------------------- */
typedef struct {
    const uint8_t* src;
    uint64_t size, total, read;
    unsigned marker;
    int overrun;
} zbr;

static int zbr_start(zbr* r, const uint8_t* src, uint64_t size) {
    r->src = src;
    r->size = size;
    r->read = 0;
    r->overrun = 0;
    if (size == 0) return Z_CORRUPT;
    const uint8_t last = src[size - 1];
    if (last == 0) return Z_CORRUPT;
    r->marker = z_hibit(last);
    r->total = (size - 1) * 8 + r->marker;
    return Z_OK;
}
static uint64_t zbr_left(const zbr* r) { return r->total - r->read; }
static unsigned zbr_bit(const zbr* r, uint64_t idx) {
    if (idx < r->marker) return (r->src[r->size - 1] >> (r->marker - 1 - idx)) & 1u;
    const uint64_t below = idx - r->marker;
    return (r->src[r->size - 2 - below / 8] >> (7 - below % 8)) & 1u;
}
static int zbr_read(zbr* r, unsigned count, uint64_t* v) {
    *v = 0;
    if (r->overrun) return Z_CORRUPT;
    if (count > 57) return Z_CORRUPT;
    if (count == 0) return Z_OK;
    if (count > zbr_left(r)) {
        r->overrun = 1;
        return Z_CORRUPT;
    }
    uint64_t a = 0;
    for (unsigned i = 0; i < count; i++) a = (a << 1) | zbr_bit(r, r->read + i);
    r->read += count;
    *v = a;
    return Z_OK;
}
static uint32_t zbr_peek(const zbr* r, unsigned count) {
    uint32_t a = 0;
    const uint64_t left = zbr_left(r);
    for (unsigned i = 0; i < count; i++)
        a = (a << 1) | (i < left ? zbr_bit(r, r->read + i) : 0u);
    return a;
}

/* ---------------- FSE ------------------------------------------------ */
typedef struct {
    uint16_t next;
    uint8_t sym, bits;
} fse_cell;

/* Forward little-endian bit reader over the description. */
typedef struct {
    const uint8_t* src;
    uint64_t size, byte;
    unsigned bit;
} fdr;
static int fdr_avail(const fdr* r, unsigned count) {
    const unsigned need = r->bit + count;
    return (uint64_t)((need + 7) / 8) <= r->size - r->byte;
}
static uint32_t fdr_peek(const fdr* r, unsigned count) {
    uint32_t v = 0;
    uint64_t by = r->byte;
    unsigned bi = r->bit;
    for (unsigned i = 0; i < count; i++) {
        unsigned t = by < r->size ? (r->src[by] >> bi) & 1u : 0u;
        v |= (uint32_t)t << i;
        if (++bi == 8) { bi = 0; by++; }
    }
    return v;
}
static void fdr_adv(fdr* r, unsigned count) {
    const unsigned t = r->bit + count;
    r->byte += t / 8;
    r->bit = t % 8;
}

/* src/zstd_fse.h ZstdFseReadNCount */
static int fse_ncount(const uint8_t* src, uint64_t size, unsigned max_sym, unsigned max_log,
                      int16_t* counts, unsigned* out_max, unsigned* out_log,
                      uint64_t* used) {
    if (size == 0) return Z_CORRUPT;
    const unsigned nsym = max_sym + 1;
    for (unsigned s = 0; s < nsym; s++) counts[s] = 0;
    fdr r = {src, size, 0, 0};
    if (!fdr_avail(&r, 4)) return Z_CORRUPT;
    const unsigned log = fdr_peek(&r, 4) + 5;
    fdr_adv(&r, 4);
    if (log > max_log) return Z_CORRUPT;
    int32_t remaining = (int32_t)(1u << log) + 1, threshold = (int32_t)(1u << log);
    unsigned nbits = log + 1, sc = 0;
    int prev0 = 0;
    for (unsigned it = 0; it < nsym; it++) {
        if (prev0) {
            int open = 1;
            for (unsigned step = 0; step < nsym && open; step++) {
                if (!fdr_avail(&r, 2)) return Z_CORRUPT;
                const unsigned rep = fdr_peek(&r, 2);
                fdr_adv(&r, 2);
                sc += rep;
                if (rep != 3) open = 0;
                if (sc >= nsym) return Z_CORRUPT;
            }
            if (open) return Z_CORRUPT;
            prev0 = 0;
        }
        const int32_t small = (2 * threshold - 1) - remaining;
        const uint32_t pk = fdr_peek(&r, nbits);
        const int32_t narrow = (int32_t)(pk & (uint32_t)(threshold - 1));
        int32_t prob;
        unsigned w;
        if (narrow < small) {
            prob = narrow;
            w = nbits - 1;
        } else {
            prob = (int32_t)(pk & (uint32_t)(2 * threshold - 1));
            if (prob >= threshold) prob -= small;
            w = nbits;
        }
        if (!fdr_avail(&r, w)) return Z_CORRUPT;
        fdr_adv(&r, w);
        prob--;
        remaining -= prob < 0 ? -prob : prob;
        counts[sc] = (int16_t)prob;
        sc++;
        prev0 = prob == 0;
        if (remaining < threshold) {
            if (remaining <= 1) break;
            nbits = z_hibit((uint32_t)remaining) + 1;
            threshold = (int32_t)(1u << (nbits - 1));
        }
        if (sc >= nsym) break;
    }
    if (remaining != 1) return Z_CORRUPT;
    *out_max = sc - 1;
    *out_log = log;
    *used = r.byte + (r.bit ? 1 : 0);
    return Z_OK;
}

/* src/zstd_fse.h ZstdFseBuildDTable */
static int fse_build(const int16_t* counts, unsigned max_sym, unsigned log, fse_cell* cells) {
    const uint32_t size = 1u << log;
    uint16_t next[256];
    uint32_t claimed = 0;
    for (unsigned s = 0; s <= max_sym; s++) {
        const int16_t p = counts[s];
        if (p < -1) return Z_CORRUPT;
        const uint32_t m = p < 0 ? 1u : (uint32_t)p;
        if (m > size - claimed) return Z_CORRUPT;
        claimed += m;
    }
    if (claimed != size) return Z_CORRUPT;
    uint32_t high = size - 1;
    for (unsigned s = 0; s <= max_sym; s++) {
        if (counts[s] < 0) {
            cells[high].sym = (uint8_t)s;
            high--;
            next[s] = 1;
        } else {
            next[s] = (uint16_t)counts[s];
        }
    }
    const uint32_t mask = size - 1, step = (size >> 1) + (size >> 3) + 3;
    uint32_t pos = 0;
    for (unsigned s = 0; s <= max_sym; s++) {
        for (int16_t k = 0; k < counts[s]; k++) {
            cells[pos].sym = (uint8_t)s;
            pos = (pos + step) & mask;
            uint32_t fuel = size;
            while (pos > high) {
                if (fuel == 0) return Z_CORRUPT;
                fuel--;
                pos = (pos + step) & mask;
            }
        }
    }
    for (uint32_t c = 0; c < size; c++) {
        const uint8_t s = cells[c].sym;
        const uint16_t ns = next[s]++;
        const unsigned b = log - z_hibit(ns);
        cells[c].bits = (uint8_t)b;
        cells[c].next = (uint16_t)((ns << b) - size);
    }
    return Z_OK;
}

/* ---------------- Huffman ------------------------------------------- */
typedef struct {
    uint8_t sym, bits;
} huf_cell;

/* src/zstd_huf.h ZstdHufReadWeights + ZstdFseDecode2State, max table log 11 */
static int huf_weights(const uint8_t* src, uint64_t size, uint8_t* w, unsigned* count,
                       unsigned* table_log, uint64_t* used) {
    const unsigned max_count = 256, max_log = 11;
    if (size == 0) return Z_CORRUPT;
    const unsigned hdr = src[0];
    unsigned written = 0;
    if (hdr >= 128) {
        written = hdr - 127;
        const uint64_t pay = (written + 1u) / 2u;
        if (pay + 1 > size) return Z_CORRUPT;
        if (written + 1 > max_count) return Z_CORRUPT;
        for (unsigned i = 0; i < written; i++) {
            const unsigned b = src[1 + i / 2];
            w[i] = (uint8_t)((i % 2) == 0 ? (b >> 4) : (b & 15));
        }
        *used = pay + 1;
    } else {
        const uint64_t pay = hdr;
        if (pay + 1 > size) return Z_CORRUPT;
        int16_t counts[13];
        unsigned fmax, flog;
        uint64_t desc;
        if (fse_ncount(src + 1, pay, 12, 6, counts, &fmax, &flog, &desc)) return Z_CORRUPT;
        fse_cell cells[64];
        if (fse_build(counts, fmax, flog, cells)) return Z_CORRUPT;
        zbr r;
        if (zbr_start(&r, src + 1 + desc, pay - desc)) return Z_CORRUPT;
        const uint32_t tsize = 1u << flog, cap = max_count - 1;
        uint64_t b;
        uint32_t st[2];
        if (zbr_read(&r, flog, &b)) return Z_CORRUPT;
        st[0] = (uint32_t)b;
        if (zbr_read(&r, flog, &b)) return Z_CORRUPT;
        st[1] = (uint32_t)b;
        uint32_t produced = 0;
        int done = 0;
        for (uint32_t step = 0; step < cap; step++) {
            uint32_t* act = &st[step % 2];
            uint32_t* oth = &st[(step + 1) % 2];
            if (*act >= tsize) return Z_CORRUPT;
            const fse_cell c = cells[*act];
            w[produced++] = c.sym;
            if (c.bits > zbr_left(&r)) {
                if (produced == cap) return Z_CORRUPT;  /* too many weights */
                if (*oth >= tsize) return Z_CORRUPT;
                w[produced++] = cells[*oth].sym;
                done = 1;
                break;
            }
            if (zbr_read(&r, c.bits, &b)) return Z_CORRUPT;
            *act = c.next + (uint32_t)b;
        }
        if (!done) return Z_CORRUPT;
        written = produced;
        *used = pay + 1;
    }
    uint32_t total = 0;
    for (unsigned i = 0; i < written; i++) {
        if (w[i] > max_log) return Z_CORRUPT;
        total += (1u << w[i]) >> 1;
    }
    if (total == 0) return Z_CORRUPT;
    const unsigned tl = z_hibit(total) + 1;
    if (tl > max_log) return Z_CORRUPT;
    const uint32_t rest = (1u << tl) - total;
    const unsigned last = z_hibit(rest) + 1;
    if ((1u << (last - 1)) != rest) return Z_CORRUPT;
    w[written] = (uint8_t)last;
    unsigned deep = 0;
    for (unsigned i = 0; i <= written; i++)
        if (w[i] == 1) deep++;
    if (deep < 2) return Z_CORRUPT;
    *count = written + 1;
    *table_log = tl;
    return Z_OK;
}

static int huf_build(const uint8_t* w, unsigned count, unsigned tl, huf_cell* cells) {
    const uint32_t size = 1u << tl;
    uint32_t rc[13] = {0}, claimed = 0;
    for (unsigned i = 0; i < count; i++) {
        if (w[i] > tl) return Z_CORRUPT;
        rc[w[i]]++;
        claimed += (1u << w[i]) >> 1;
    }
    if (claimed != size) return Z_CORRUPT;
    uint32_t start[13] = {0}, nx = 0;
    for (unsigned k = 1; k <= tl; k++) {
        start[k] = nx;
        nx += rc[k] * ((1u << k) >> 1);
    }
    for (unsigned s = 0; s < count; s++) {
        const unsigned k = w[s];
        if (!k) continue;
        const uint32_t span = (1u << k) >> 1;
        for (uint32_t j = 0; j < span; j++) {
            cells[start[k] + j].sym = (uint8_t)s;
            cells[start[k] + j].bits = (uint8_t)(tl + 1 - k);
        }
        start[k] += span;
    }
    return Z_OK;
}

static int huf_stream(const uint8_t* src, uint64_t size, const huf_cell* cells, unsigned tl,
                      uint8_t* dst, uint64_t count) {
    zbr r;
    if (zbr_start(&r, src, size)) return Z_CORRUPT;
    for (uint64_t i = 0; i < count; i++) {
        const huf_cell c = cells[zbr_peek(&r, tl)];
        uint64_t b;
        if (zbr_read(&r, c.bits, &b)) return Z_CORRUPT;
        dst[i] = c.sym;
    }
    return r.read == r.total ? Z_OK : Z_CORRUPT;
}

/* ---------------- per-frame state ------------------------------------- */
typedef struct {
    huf_cell huf[1 << 11];
    unsigned huf_log;
    int huf_present;
    fse_cell seq[3][512];
    uint32_t seq_size[3];
    unsigned seq_log[3];
    int seq_present[3];
    uint64_t rep[3];
} zstate;

/* src/zstd_literals.h ZstdDecodeLiterals; `cap` = block maximum */
static int z_literals(zstate* z, const uint8_t* src, uint64_t size, uint64_t window,
                      uint8_t* dst, uint64_t cap, uint64_t* produced, uint64_t* consumed) {
    if (size == 0) return Z_CORRUPT;
    const unsigned type = src[0] & 3, fmt = (src[0] >> 2) & 3;
    uint64_t regen, csize = 0, hsize;
    unsigned streams = 0;
    if (type < 2) {
        unsigned hs = 1, sh = 3;
        if (fmt == 1) { hs = 2; sh = 4; }
        else if (fmt == 3) { hs = 3; sh = 4; }
        if (size < hs) return Z_CORRUPT;
        regen = z_le(src, hs) >> sh;
        hsize = hs;
    } else {
        unsigned hs = 3, fb = 10;
        if (fmt == 2) { hs = 4; fb = 14; }
        else if (fmt == 3) { hs = 5; fb = 18; }
        if (size < hs) return Z_CORRUPT;
        const uint64_t raw = z_le(src, hs), m = (1ull << fb) - 1;
        regen = (raw >> 4) & m;
        csize = (raw >> (4 + fb)) & m;
        hsize = hs;
        streams = fmt == 0 ? 1 : 4;
    }
    const uint64_t bmax = window < 131072 ? window : 131072;
    if (regen > bmax) return Z_CORRUPT;
    if (regen > cap) return Z_TOO_SMALL;
    const uint64_t after = size - hsize;
    if (type == 0) {
        if (regen > after) return Z_CORRUPT;
        memcpy(dst, src + hsize, regen);
        *produced = regen;
        *consumed = hsize + regen;
        return Z_OK;
    }
    if (type == 1) {
        if (after < 1) return Z_CORRUPT;
        memset(dst, src[hsize], regen);
        *produced = regen;
        *consumed = hsize + 1;
        return Z_OK;
    }
    if (csize > after) return Z_CORRUPT;
    const uint8_t* pay = src + hsize;
    uint64_t psize = csize;
    if (type == 2) {
        uint8_t w[257];
        unsigned cnt, tl;
        uint64_t used;
        if (huf_weights(pay, psize, w, &cnt, &tl, &used)) return Z_CORRUPT;
        if (huf_build(w, cnt, tl, z->huf)) return Z_CORRUPT;
        z->huf_log = tl;
        z->huf_present = 1;
        pay += used;
        psize -= used;
    } else if (!z->huf_present) {
        return Z_CORRUPT;
    }
    if (psize == 0) return Z_CORRUPT;
    if (streams == 1) {
        if (huf_stream(pay, psize, z->huf, z->huf_log, dst, regen)) return Z_CORRUPT;
    } else {
        if (psize < 10) return Z_CORRUPT;
        if (regen < 6) return Z_CORRUPT;
        uint64_t cs[4], tot = 0;
        for (int s = 0; s < 3; s++) {
            cs[s] = z_le(pay + 2 * s, 2);
            tot += cs[s];
        }
        const uint64_t sb = psize - 6;
        if (tot >= sb) return Z_CORRUPT;
        cs[3] = sb - tot;
        const uint64_t seg = (regen + 3) / 4;
        uint64_t rg[4] = {seg, seg, seg, regen - 3 * seg};
        const uint8_t* st = pay + 6;
        uint8_t* o = dst;
        for (int s = 0; s < 4; s++) {
            if (huf_stream(st, cs[s], z->huf, z->huf_log, o, rg[s])) return Z_CORRUPT;
            st += cs[s];
            o += rg[s];
        }
    }
    *produced = regen;
    *consumed = hsize + csize;
    return Z_OK;
}

/* Sequence code tables (RFC 8878 3.1.1.3.2.1.1) restated: extra bits and
 * baselines of the literal-length and match-length codes. */
static unsigned ll_bits(unsigned c) {
    static const unsigned mid[9] = {1, 1, 1, 1, 2, 2, 3, 3, 4};
    if (c < 16) return 0;
    if (c >= 25) return c - 19;
    return mid[c - 16];
}
static unsigned ml_bits(unsigned c) {
    static const unsigned mid[11] = {1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5};
    if (c < 32) return 0;
    if (c >= 43) return c - 36;
    return mid[c - 32];
}
static uint32_t ll_base(unsigned c) {
    uint32_t b = 0;
    for (unsigned k = 0; k < c; k++) b += 1u << ll_bits(k);
    return b;
}
static uint32_t ml_base(unsigned c) {
    uint32_t b = 3;
    for (unsigned k = 0; k < c; k++) b += 1u << ml_bits(k);
    return b;
}

static const int16_t k_ll_pre[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                     2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
static const int16_t k_of_pre[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                     1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};
static const int16_t k_ml_pre[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                     1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                     1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};

/* field 0 = literal lengths, 1 = offsets, 2 = match lengths */
static int z_table(zstate* z, unsigned field, unsigned mode, const uint8_t* src, uint64_t size,
                   uint64_t* used) {
    static const unsigned symmax[3] = {35, 31, 52}, logmax[3] = {9, 8, 9};
    *used = 0;
    if (mode == 3) return z->seq_present[field] ? Z_OK : Z_CORRUPT;
    if (mode == 1) {
        if (size == 0) return Z_CORRUPT;
        if (src[0] > symmax[field]) return Z_CORRUPT;
        z->seq[field][0].next = 0;
        z->seq[field][0].sym = src[0];
        z->seq[field][0].bits = 0;
        z->seq_size[field] = 1;
        z->seq_log[field] = 0;
        z->seq_present[field] = 1;
        *used = 1;
        return Z_OK;
    }
    int16_t counts[53];
    unsigned dmax, log;
    if (mode == 0) {
        const int16_t* pre = field == 0 ? k_ll_pre : field == 1 ? k_of_pre : k_ml_pre;
        dmax = field == 0 ? 35 : field == 1 ? 28 : 52;
        log = field == 1 ? 5 : 6;
        for (unsigned s = 0; s <= dmax; s++) counts[s] = pre[s];
    } else {
        uint64_t u;
        if (fse_ncount(src, size, symmax[field], logmax[field], counts, &dmax, &log, &u))
            return Z_CORRUPT;
        *used = u;
    }
    if (fse_build(counts, dmax, log, z->seq[field])) {
        *used = 0;
        return Z_CORRUPT;
    }
    z->seq_size[field] = 1u << log;
    z->seq_log[field] = log;
    z->seq_present[field] = 1;
    return Z_OK;
}

typedef struct {
    uint32_t ll, ml;
    uint64_t ov;
} zseq;

/* src/zstd_repcode.h ZstdRepcodeResolve */
static int z_repcode(uint64_t* rep, uint64_t ov, uint32_t ll, uint64_t* out) {
    uint64_t res;
    unsigned taken = 3;
    if (ov > 3) {
        res = ov - 3;
    } else if (ll != 0) {
        taken = (unsigned)ov - 1;
        res = rep[taken];
    } else if (ov < 3) {
        taken = (unsigned)ov;
        res = rep[taken];
    } else {
        res = rep[0];
        if (res) res -= 1;
    }
    if (res == 0) return Z_CORRUPT;
    if (taken != 0) {
        if (taken != 1) rep[2] = rep[1];
        rep[1] = rep[0];
        rep[0] = res;
    }
    *out = res;
    return Z_OK;
}

/* One frame at the start of f[0, n); *consumed is its length in bytes and
 * bytes after it are not looked at. wide: the frame-sequence reading, which
 * also takes a frame without a content size (output bounded by cap) and any
 * window whose log is at most 31 (libzstd's one-shot limit, ZSTD_WINDOWLOG_MAX
 * on 64-bit hosts). */
static int z_frame(const uint8_t* f, uint64_t n, uint8_t* dst, uint64_t cap,
                   uint64_t* written, uint64_t* consumed, int wide) {
    *written = 0;
    *consumed = 0;
    if (n < 4) return Z_CORRUPT;
    const uint32_t magic = (uint32_t)z_le(f, 4);
    if (magic != 0xFD2FB528u) {
        if (magic >= 0x184D2A50u && magic <= 0x184D2A5Fu) return Z_UNSUPPORTED;
        return Z_CORRUPT;
    }
    if (n < 5) return Z_CORRUPT;
    const unsigned d = f[4], fcs_flag = d >> 6, single = (d >> 5) & 1, csum = (d >> 2) & 1,
                   did = d & 3;
    if (d & 8) return Z_CORRUPT;
    if (did) return Z_UNSUPPORTED;
    const unsigned fcs_size = fcs_flag == 0 ? (single ? 1 : 0) : fcs_flag == 1 ? 2 : fcs_flag == 2 ? 4 : 8;
    const int has_fcs = fcs_size != 0; /* single segment implies a content size */
    if (!has_fcs && !wide) return Z_UNSUPPORTED;
    const unsigned wbytes = single ? 0 : 1;
    const uint64_t hsz = 5 + wbytes + fcs_size;
    if (n < hsz) return Z_CORRUPT;
    uint64_t fcs = has_fcs ? z_le(f + 5 + wbytes, fcs_size) : 0;
    if (fcs_size == 2) fcs += 256;
    uint64_t window;
    if (single) {
        window = fcs;
    } else {
        const uint64_t e = f[5] >> 3, m = f[5] & 7, base = 1ull << (10 + e);
        window = base + (base / 8) * m;
        if (!wide && window > (8ull << 20)) return Z_UNSUPPORTED;
        if (wide && 10 + e > 31) return Z_UNSUPPORTED;
    }
    if (has_fcs && fcs > cap) return Z_TOO_SMALL;

    zstate* z = (zstate*)calloc(1, sizeof(zstate));
    const uint64_t bmax = window < 131072 ? window : 131072;
    uint8_t* lit = (uint8_t*)malloc(bmax ? bmax : 1);
    zseq* seqs = (zseq*)malloc(sizeof(zseq) * (bmax / 3 + 1));
    if (!z || !lit || !seqs) {
        free(z); free(lit); free(seqs);
        return Z_CUDA;
    }
    z->rep[0] = 1;
    z->rep[1] = 4;
    z->rep[2] = 8;
    int st = Z_OK;
    uint64_t pos = hsz, out = 0;
    for (;;) {
        if (n - pos < 3) { st = Z_CORRUPT; goto done; }
        const uint32_t raw = (uint32_t)z_le(f + pos, 3);
        const int last = raw & 1;
        const unsigned btype = (raw >> 1) & 3;
        const uint32_t bsize = raw >> 3;
        if (btype == 3) { st = Z_CORRUPT; goto done; }
        if (bsize > bmax) { st = Z_CORRUPT; goto done; }
        const uint32_t body = btype == 1 ? 1 : bsize;
        if (n - pos < 3ull + body) { st = Z_CORRUPT; goto done; }
        const uint8_t* b = f + pos + 3;
        if (btype == 0) {
            if (bsize > cap - out) { st = Z_TOO_SMALL; goto done; }
            memcpy(dst + out, b, bsize);
            out += bsize;
        } else if (btype == 1) {
            if (bsize > cap - out) { st = Z_TOO_SMALL; goto done; }
            memset(dst + out, b[0], bsize);
            out += bsize;
        } else {
            uint64_t lits = 0, used = 0;
            if (z_literals(z, b, body, window, lit, bmax, &lits, &used)) { st = Z_CORRUPT; goto done; }
            const uint8_t* sec = b + used;
            uint64_t rem = body - used;
            /* sequences section header */
            if (rem == 0) { st = Z_CORRUPT; goto done; }
            uint32_t nseq;
            uint64_t c = 1;
            if (sec[0] < 128) {
                nseq = sec[0];
            } else if (sec[0] < 255) {
                if (rem < 2) { st = Z_CORRUPT; goto done; }
                nseq = ((uint32_t)(sec[0] - 128) << 8) + sec[1];
                c = 2;
            } else {
                if (rem < 3) { st = Z_CORRUPT; goto done; }
                nseq = (uint32_t)sec[1] + ((uint32_t)sec[2] << 8) + 0x7F00u;
                c = 3;
            }
            if (nseq) {
                if (nseq > bmax / 3) { st = Z_CORRUPT; goto done; }
                if (rem <= c) { st = Z_CORRUPT; goto done; }
                const unsigned modes = sec[c++];
                if (modes & 3) { st = Z_CORRUPT; goto done; }
                const unsigned mode[3] = {(modes >> 6) & 3, (modes >> 4) & 3, (modes >> 2) & 3};
                sec += c;
                rem -= c;
                for (unsigned fld = 0; fld < 3; fld++) {
                    uint64_t u;
                    if (z_table(z, fld, mode[fld], sec, rem, &u)) { st = Z_CORRUPT; goto done; }
                    sec += u;
                    rem -= u;
                }
                if (rem == 0) { st = Z_CORRUPT; goto done; }
                zbr r;
                if (zbr_start(&r, sec, rem)) { st = Z_CORRUPT; goto done; }
                uint64_t v;
                uint32_t s_ll, s_of, s_ml;
                if (zbr_read(&r, z->seq_log[0], &v)) { st = Z_CORRUPT; goto done; }
                s_ll = (uint32_t)v;
                if (zbr_read(&r, z->seq_log[1], &v)) { st = Z_CORRUPT; goto done; }
                s_of = (uint32_t)v;
                if (zbr_read(&r, z->seq_log[2], &v)) { st = Z_CORRUPT; goto done; }
                s_ml = (uint32_t)v;
                for (uint32_t i = 0; i < nseq; i++) {
                    if (s_ll >= z->seq_size[0] || s_of >= z->seq_size[1] || s_ml >= z->seq_size[2]) {
                        st = Z_CORRUPT; goto done;
                    }
                    const unsigned cl = z->seq[0][s_ll].sym, co = z->seq[1][s_of].sym,
                                   cm = z->seq[2][s_ml].sym;
                    if (cl > 35 || co > 31 || cm > 52) { st = Z_CORRUPT; goto done; }
                    uint64_t eo, em, el;
                    if (zbr_read(&r, co, &eo) || zbr_read(&r, ml_bits(cm), &em) ||
                        zbr_read(&r, ll_bits(cl), &el)) { st = Z_CORRUPT; goto done; }
                    seqs[i].ov = (1ull << co) + eo;
                    seqs[i].ml = ml_base(cm) + (uint32_t)em;
                    seqs[i].ll = ll_base(cl) + (uint32_t)el;
                    if (i + 1 == nseq) continue;
                    const fse_cell a = z->seq[0][s_ll];
                    if (zbr_read(&r, a.bits, &v)) { st = Z_CORRUPT; goto done; }
                    s_ll = a.next + (uint32_t)v;
                    if (s_ml >= z->seq_size[2]) { st = Z_CORRUPT; goto done; }
                    const fse_cell m = z->seq[2][s_ml];
                    if (zbr_read(&r, m.bits, &v)) { st = Z_CORRUPT; goto done; }
                    s_ml = m.next + (uint32_t)v;
                    if (s_of >= z->seq_size[1]) { st = Z_CORRUPT; goto done; }
                    const fse_cell o = z->seq[1][s_of];
                    if (zbr_read(&r, o.bits, &v)) { st = Z_CORRUPT; goto done; }
                    s_of = o.next + (uint32_t)v;
                }
                if (r.read != r.total) { st = Z_CORRUPT; goto done; }
            }
            /* execute (tests/zstd_twin_driver.h:292-348) */
            uint64_t lp = 0;
            for (uint32_t i = 0; i < nseq; i++) {
                const zseq q = seqs[i];
                if (lp + q.ll > lits) { st = Z_CORRUPT; goto done; }
                /* literals: bytes past the capacity are not stored (the
                 * capacity verdict is taken after the match, as the twin
                 * does) */
                for (uint32_t k = 0; k < q.ll; k++)
                    if (out + k < cap) dst[out + k] = lit[lp + k];
                out += q.ll;
                lp += q.ll;
                uint64_t off;
                if (z_repcode(z->rep, q.ov, q.ll, &off)) { st = Z_CORRUPT; goto done; }
                if (off > out || off > window) { st = Z_CORRUPT; goto done; }
                if (out > cap || q.ml > cap - out) { st = Z_TOO_SMALL; goto done; }
                for (uint32_t k = 0; k < q.ml; k++) dst[out + k] = dst[out - off + k];
                out += q.ml;
            }
            if (lits - lp > cap - (out < cap ? out : cap) || out > cap) { st = Z_TOO_SMALL; goto done; }
            memcpy(dst + out, lit + lp, lits - lp);
            out += lits - lp;
        }
        if (out > cap) { st = Z_TOO_SMALL; goto done; }
        pos += 3 + body;
        if (last) break;
    }
    if (has_fcs && out != fcs) { st = Z_CORRUPT; goto done; }
    if (csum) {
        if (n - pos < 4) { st = Z_CORRUPT; goto done; }
        if ((uint32_t)oracle_xxh64(dst, out, 0) != (uint32_t)z_le(f + pos, 4)) {
            st = Z_CORRUPT; goto done;
        }
        pos += 4;
    }
    *written = out;
    *consumed = pos;
done:
    free(z);
    free(lit);
    free(seqs);
    return st;
}

/* One frame per input, the reference's rule (src/zstd_frame.h:196-409):
 * trailing bytes are CORRUPT, a skippable frame UNSUPPORTED. */
int oracle_zstd_decode(const uint8_t* f, uint64_t n, uint8_t* dst, uint64_t cap,
                       uint64_t* written) {
    uint64_t out = 0, used = 0;
    *written = 0;
    const int st = z_frame(f, n, dst, cap, &out, &used, 0);
    if (st != Z_OK) return st;
    if (used != n) return Z_CORRUPT;
    *written = out;
    return Z_OK;
}

/* Concatenated frames as libzstd's ZSTD_decompress reads them with its
 * default limits (the reference's subset ladder, docs/MASTERPLAN.md:
 * 1286-1296, rungs 1-3 up to that limit): skippable frames (magic
 * 0x184D2A50-5F, 4-byte little-endian size) are skipped, each Zstd frame
 * decodes after the previous one's output, with or without a content size,
 * with any window up to a log of 31 (a dictionary id stays UNSUPPORTED);
 * fewer than 4 bytes left, or a skippable frame past the end, is CORRUPT. */
int oracle_zstd_decode_multi(const uint8_t* f, uint64_t n, uint8_t* dst, uint64_t cap,
                             uint64_t* written) {
    uint64_t pos = 0, out = 0;
    *written = 0;
    while (pos < n) {
        if (n - pos < 4) return Z_CORRUPT;
        const uint32_t magic = (uint32_t)z_le(f + pos, 4);
        if (magic >= 0x184D2A50u && magic <= 0x184D2A5Fu) {
            if (n - pos < 8) return Z_CORRUPT;
            const uint64_t sz = z_le(f + pos + 4, 4);
            if (sz > n - pos - 8) return Z_CORRUPT;
            pos += 8 + sz;
            continue;
        }
        uint64_t fo = 0, used = 0;
        const int st = z_frame(f + pos, n - pos, dst + out, cap - out, &fo, &used, 1);
        if (st != Z_OK) return st;
        out += fo;
        pos += used;
    }
    *written = out;
    return Z_OK;
}
