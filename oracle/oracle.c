/* ORACLE — test infrastructure, not part of the product.
 *
 * A plain-C, byte-serial restatement of the reference decoders' accept/reject
 * ladders, used only by tests/, by __graft_entry__.smoke() and by bench.py's
 * CPU-baseline leg as a checker. The shipped library never links, loads or
 * calls anything in this directory.
 *
 * Parity pins: tests/test_oracle.py checks every function here against
 * (a) the reference's own golden seeds (fuzz/corpus/<target>/ of iderex/cudec,
 *     framing per fuzz/fuzz_lz4_block.cpp:69-74 and
 *     fuzz/fuzz_snappy_block.cpp), committed as tests/golden/*.json,
 * (b) the reference's host twins compiled from its sources into oracle/_ref
 *     (tests/lz4_twin.h, tests/snappy_twin.h over src/lz4_block.h and
 *     src/snappy_block.h), and
 * (c) the codec libraries (liblz4 LZ4_decompress_safe, snappy via pyarrow)
 *     on seeded corpora and mutants.
 *
 * Status values are cudec_status (include/cudec.h).
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum {
    ST_OK = 0,
    ST_INVALID_ARGUMENT = 1,
    ST_CORRUPT = 2,
    ST_TOO_SMALL = 3,
    ST_CUDA = 4,
    ST_UNSUPPORTED = 6
};

/* ------------------------------------------------------------------------
 * LZ4 block. Follows src/lz4_block.h:139-258 (Lz4Parser::Next) and
 * :95-128 (AccumulateLength), executed sequentially as tests/lz4_twin.h:41-86
 * does (chasing byte copy).
 * ---------------------------------------------------------------------- */

/* One 255-continued length extension; mirrors lz4_block.h:95-128. `margin`
 * is liblz4's read limit before the input end (15 for literal lengths, 4 for
 * match lengths); `pre` is the extra guard taken before the literal loop. */
static int lz4_extend(const uint8_t* s, uint64_t n, uint64_t* q,
                      uint64_t* len, uint64_t room, uint64_t margin, int pre) {
    if (pre && *q + margin >= n) return ST_CORRUPT;
    uint8_t b;
    do {
        if (*q >= n) return ST_CORRUPT;
        if (*len > room) return ST_TOO_SMALL;
        b = s[(*q)++];
        *len += b;
        if (*q + margin > n) return ST_CORRUPT;
    } while (b == 255);
    return ST_OK;
}

/* Decodes one LZ4 block into dst[0, cap). Returns a status; on ST_OK the
 * decoded size is in *written. dst is always bounded by cap. */
int oracle_lz4_decode(const uint8_t* s, uint64_t n, uint8_t* dst, uint64_t cap,
                      uint64_t* written) {
    uint64_t p = 0, d = 0;
    *written = 0;
    for (;;) {
        if (p >= n) return ST_CORRUPT; /* a token must be present */
        const uint8_t tok = s[p++];
        uint64_t lit = tok >> 4;
        if (lit == 15) {
            int st = lz4_extend(s, n, &p, &lit, cap - d, 15, 1);
            if (st) return st;
        }
        if (lit > n - p) return ST_CORRUPT;
        if (lit > cap - d) return ST_TOO_SMALL;
        /* End-of-block rule (lz4_block.h:161-199): a run ending within 12
         * bytes of the capacity or within 8 bytes of the input end is the
         * last one and must consume the input exactly. */
        if (cap - d - lit < 12 || n - p - lit < 8) {
            if (p + lit != n) return ST_CORRUPT;
            if (cap == 0 && tok != 0) return ST_CORRUPT;
            memcpy(dst + d, s + p, lit);
            *written = d + lit;
            return ST_OK;
        }
        memcpy(dst + d, s + p, lit);
        p += lit;
        d += lit;
        const uint64_t off = (uint64_t)s[p] | ((uint64_t)s[p + 1] << 8);
        p += 2;
        /* Offset zero is refused (stricter than liblz4, lz4_block.h:212-225). */
        if (off == 0) return ST_CORRUPT;
        if (off > d) return ST_CORRUPT;
        uint64_t ml = (uint64_t)(tok & 15) + 4;
        if ((tok & 15) == 15) {
            int st = lz4_extend(s, n, &p, &ml, cap - d, 4, 0);
            if (st) return st;
        }
        if (ml > cap - d) return ST_TOO_SMALL;
        if (ml > cap - d - 5) return ST_CORRUPT; /* last 5 bytes are literals */
        for (uint64_t i = 0; i < ml; i++) dst[d + i] = dst[d - off + i];
        d += ml;
    }
}

/* ------------------------------------------------------------------------
 * Snappy raw block. Follows src/snappy_block.h:172-223 (preamble) and
 * :249-435 (Begin/Next), executed as tests/snappy_twin.h does.
 * ---------------------------------------------------------------------- */

/* Varint32 preamble; returns status, *declared and *used on success. */
int oracle_snappy_declared(const uint8_t* s, uint64_t n, uint64_t* declared,
                           uint64_t* used) {
    uint64_t v = 0;
    for (uint64_t g = 0; g < 5; g++) {
        if (g >= n) return ST_CORRUPT;
        const uint8_t b = s[g];
        if (g == 4 && b >= 16) return ST_CORRUPT;
        v |= (uint64_t)(b & 0x7f) << (7 * g);
        if (!(b & 0x80)) {
            *declared = v;
            *used = g + 1;
            return ST_OK;
        }
    }
    return ST_CORRUPT; /* unreachable: the fifth byte either ends or fails */
}

int oracle_snappy_decode(const uint8_t* s, uint64_t n, uint8_t* dst,
                         uint64_t cap, uint64_t* written) {
    uint64_t declared = 0, p = 0, d = 0;
    *written = 0;
    int st = oracle_snappy_declared(s, n, &declared, &p);
    if (st) return st;
    if (declared > cap) return ST_TOO_SMALL;
    while (p < n) {
        const uint8_t tag = s[p];
        const unsigned kind = tag & 3;
        if (kind == 0) {
            uint64_t len = tag >> 2, hdr = 1;
            if (len > 59) {
                const uint64_t extra = len - 59;
                hdr += extra;
                if (hdr > n - p) return ST_CORRUPT;
                len = 0;
                for (uint64_t i = 0; i < extra; i++)
                    len |= (uint64_t)s[p + 1 + i] << (8 * i);
            }
            len += 1; /* 64-bit: the 0xFFFFFFFF spelling does not wrap */
            p += hdr;
            if (len > n - p) return ST_CORRUPT;
            if (len > declared - d) return ST_CORRUPT;
            memcpy(dst + d, s + p, len);
            p += len;
            d += len;
            continue;
        }
        const uint64_t ob = kind == 1 ? 1 : (kind == 2 ? 2 : 4);
        if (1 + ob > n - p) return ST_CORRUPT;
        uint64_t off = 0, len;
        for (uint64_t i = 0; i < ob; i++) off |= (uint64_t)s[p + 1 + i] << (8 * i);
        if (kind == 1) {
            off |= (uint64_t)(tag >> 5) << 8;
            len = 4 + ((tag >> 2) & 7);
        } else {
            len = (uint64_t)(tag >> 2) + 1;
        }
        p += 1 + ob;
        if (off == 0) return ST_CORRUPT;
        if (off > d) return ST_CORRUPT;
        if (len > declared - d) return ST_CORRUPT;
        for (uint64_t i = 0; i < len; i++) dst[d + i] = dst[d - off + i];
        d += len;
    }
    if (d != declared) return ST_CORRUPT; /* under-production */
    *written = d;
    return ST_OK;
}

/* ------------------------------------------------------------------------
 * Batch drivers over a host thread pool (the CPU-baseline leg). Chunks are
 * taken from an atomic cursor, like the reference bench's CPU harness.
 * ---------------------------------------------------------------------- */

typedef int (*decode_fn)(const uint8_t*, uint64_t, uint8_t*, uint64_t,
                         uint64_t*);

struct batch_job {
    decode_fn fn;
    const uint8_t* const* src;
    const uint64_t* src_sizes;
    uint8_t* const* dst;
    const uint64_t* caps;
    uint64_t n;
    int32_t* status;
    uint64_t* written;
    _Atomic uint64_t cursor;
};

static void* batch_worker(void* arg) {
    struct batch_job* j = (struct batch_job*)arg;
    for (;;) {
        const uint64_t i = atomic_fetch_add(&j->cursor, 1);
        if (i >= j->n) break;
        uint64_t w = 0;
        j->status[i] = j->fn(j->src[i], j->src_sizes[i], j->dst[i], j->caps[i], &w);
        j->written[i] = w;
    }
    return NULL;
}

static int run_batch(decode_fn fn, const uint8_t* const* src,
                     const uint64_t* src_sizes, uint8_t* const* dst,
                     const uint64_t* caps, uint64_t n, int32_t* status,
                     uint64_t* written, int threads) {
    struct batch_job j = {fn, src, src_sizes, dst, caps, n, status, written, 0};
    if (threads < 1) threads = 1;
    if (threads > 1024) threads = 1024;
    pthread_t tids[1024];
    int started = 0;
    for (int t = 1; t < threads; t++) {
        if (pthread_create(&tids[started], NULL, batch_worker, &j) == 0) started++;
    }
    batch_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(tids[t], NULL);
    return started + 1;
}

int oracle_lz4_decode_batch(const uint8_t* const* src, const uint64_t* src_sizes,
                            uint8_t* const* dst, const uint64_t* caps, uint64_t n,
                            int32_t* status, uint64_t* written, int threads) {
    return run_batch(oracle_lz4_decode, src, src_sizes, dst, caps, n, status,
                     written, threads);
}

int oracle_snappy_decode_batch(const uint8_t* const* src,
                               const uint64_t* src_sizes, uint8_t* const* dst,
                               const uint64_t* caps, uint64_t n, int32_t* status,
                               uint64_t* written, int threads) {
    return run_batch(oracle_snappy_decode, src, src_sizes, dst, caps, n, status,
                     written, threads);
}

/* ------------------------------------------------------------------------
 * LZ4 frame. Follows src/frame.cpp:282-397 (DecodeFrame) and :53-278
 * (DecodeAndAssemble: every block reject is CORRUPT; capacity checked before
 * any byte is placed). XXH32 restated from the public xxHash specification.
 * ---------------------------------------------------------------------- */

static uint32_t o_rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
static uint32_t o_rd32(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
           ((uint32_t)p[3] << 24);
}

uint32_t oracle_xxh32(const uint8_t* p, uint64_t len, uint32_t seed) {
    const uint32_t P1 = 2654435761u, P2 = 2246822519u, P3 = 3266489917u,
                   P4 = 668265263u, P5 = 374761393u;
    uint64_t i = 0;
    uint32_t h;
    if (len >= 16) {
        uint32_t v[4] = {seed + P1 + P2, seed + P2, seed, seed - P1};
        for (; i + 16 <= len; i += 16)
            for (int k = 0; k < 4; k++) v[k] = o_rotl(v[k] + o_rd32(p + i + 4 * k) * P2, 13) * P1;
        h = o_rotl(v[0], 1) + o_rotl(v[1], 7) + o_rotl(v[2], 12) + o_rotl(v[3], 18);
    } else {
        h = seed + P5;
    }
    h += (uint32_t)len;
    for (; i + 4 <= len; i += 4) h = o_rotl(h + o_rd32(p + i) * P3, 17) * P4;
    for (; i < len; i++) h = o_rotl(h + p[i] * P5, 11) * P1;
    h ^= h >> 15;
    h *= P2;
    h ^= h >> 13;
    h *= P3;
    h ^= h >> 16;
    return h;
}

int oracle_lz4f_decode(const uint8_t* f, uint64_t n, uint8_t* out, uint64_t cap,
                       uint64_t* written) {
    *written = 0;
    if (n < 7 || o_rd32(f) != 0x184D2204u) return ST_CORRUPT;
    const unsigned flg = f[4], bd = f[5];
    if (((flg >> 6) & 3) != 1 || (flg & 2)) return ST_CORRUPT;
    if (bd & 0x8F) return ST_CORRUPT;
    const unsigned bmax = (bd >> 4) & 7;
    if (bmax < 4 || bmax > 7) return ST_CORRUPT;
    const uint64_t block_max = (uint64_t)65536 << ((bmax - 4) * 2);
    if (!((flg >> 5) & 1) || (flg & 1)) return ST_UNSUPPORTED;
    uint64_t pos = 6, declared = 0;
    const int has_size = (flg >> 3) & 1, bsum = (flg >> 4) & 1, csum = (flg >> 2) & 1;
    if (has_size) {
        if (n < pos + 8) return ST_CORRUPT;
        declared = (uint64_t)o_rd32(f + pos) | ((uint64_t)o_rd32(f + pos + 4) << 32);
        pos += 8;
    }
    if (n < pos + 1) return ST_CORRUPT;
    if (((oracle_xxh32(f + 4, pos - 4, 0) >> 8) & 0xFF) != f[pos]) return ST_CORRUPT;
    pos++;
    /* first pass: the block table with checksums (no output yet) */
    uint64_t bpos = pos;
    int end = 0;
    for (uint64_t fuel = n / 4 + 1; fuel; fuel--) {
        if (n < bpos + 4) return ST_CORRUPT;
        const uint32_t bs = o_rd32(f + bpos);
        bpos += 4;
        if (bs == 0) { end = 1; break; }
        const uint64_t blen = bs & 0x7FFFFFFFu;
        if (blen == 0 || blen > block_max || n < bpos + blen) return ST_CORRUPT;
        if (bsum) {
            if (n < bpos + blen + 4) return ST_CORRUPT;
            if (oracle_xxh32(f + bpos, blen, 0) != o_rd32(f + bpos + blen)) return ST_CORRUPT;
        }
        bpos += blen + (bsum ? 4 : 0);
    }
    if (!end) return ST_CORRUPT;
    /* second pass: decode every compressed block into a scratch slot first
     * (all block rejects win over the capacity check), then place. */
    uint64_t total = 0;
    int too_small = 0;
    uint64_t p2 = pos;
    uint8_t* scratch = (uint8_t*)malloc(block_max ? block_max : 1);
    if (!scratch) return ST_CUDA;
    /* pass 2a: validate all blocks and sum sizes */
    for (;;) {
        const uint32_t bs = o_rd32(f + p2);
        p2 += 4;
        if (bs == 0) break;
        const uint64_t blen = bs & 0x7FFFFFFFu;
        uint64_t len = blen;
        if (!(bs >> 31)) {
            uint64_t w = 0;
            if (oracle_lz4_decode(f + p2, blen, scratch, block_max, &w) != ST_OK) {
                free(scratch);
                return ST_CORRUPT;
            }
            len = w;
        }
        if (len > cap - total) too_small = 1;
        if (!too_small) total += len;
        p2 += blen + (bsum ? 4 : 0);
    }
    if (too_small) { free(scratch); return ST_TOO_SMALL; }
    /* pass 2b: place */
    p2 = pos;
    uint64_t off = 0;
    for (;;) {
        const uint32_t bs = o_rd32(f + p2);
        p2 += 4;
        if (bs == 0) break;
        const uint64_t blen = bs & 0x7FFFFFFFu;
        if (bs >> 31) {
            memcpy(out + off, f + p2, blen);
            off += blen;
        } else {
            uint64_t w = 0;
            oracle_lz4_decode(f + p2, blen, out + off, cap - off < block_max ? cap - off : block_max, &w);
            off += w;
        }
        p2 += blen + (bsum ? 4 : 0);
    }
    free(scratch);
    if (has_size && declared != total) return ST_CORRUPT;
    if (csum) {
        if (n < bpos + 4) return ST_CORRUPT;
        if (oracle_xxh32(out, total, 0) != o_rd32(f + bpos)) return ST_CORRUPT;
    }
    *written = total;
    return ST_OK;
}
