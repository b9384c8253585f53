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
