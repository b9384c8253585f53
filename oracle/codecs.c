/* ORACLE — test infrastructure, not part of the product.
 *
 * Multithreaded CPU decode through the system codec libraries, for the
 * CPU-baseline leg of bench.py and for parity tests: liblz4
 * (LZ4_decompress_safe) and libzstd (ZSTD_decompressDCtx), reached by dlopen
 * with self-declared public prototypes, as the reference's CPU harness does
 * (bench/bench_lz4.cpp; pinned liblz4 1.10.0 / zstd 1.5.7 there, whatever
 * version the host carries here — the caller records it). A chunk that the
 * codec rejects reports status 2 (corrupt).
 */
#include <dlfcn.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stddef.h>
#include <stdint.h>

typedef int (*lz4_dec_t)(const char*, char*, int, int);
typedef int (*lz4_ver_t)(void);
typedef size_t (*zstd_dec_t)(void*, void*, size_t, const void*, size_t);
typedef void* (*zstd_create_t)(void);
typedef size_t (*zstd_free_t)(void*);
typedef unsigned (*zstd_iserr_t)(size_t);
typedef unsigned (*zstd_ver_t)(void);

static void* g_lz4;
static void* g_zstd;

static void* lz4_lib(void) {
    if (!g_lz4) g_lz4 = dlopen("liblz4.so.1", RTLD_NOW | RTLD_LOCAL);
    return g_lz4;
}
static void* zstd_lib(void) {
    if (!g_zstd) g_zstd = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
    return g_zstd;
}

int codec_lz4_version(void) {
    void* h = lz4_lib();
    lz4_ver_t f = h ? (lz4_ver_t)dlsym(h, "LZ4_versionNumber") : NULL;
    return f ? f() : -1;
}

int codec_zstd_version(void) {
    void* h = zstd_lib();
    zstd_ver_t f = h ? (zstd_ver_t)dlsym(h, "ZSTD_versionNumber") : NULL;
    return f ? (int)f() : -1;
}

struct codec_job {
    int kind; /* 0 = lz4, 1 = zstd */
    const uint8_t* const* src;
    const uint64_t* src_sizes;
    uint8_t* const* dst;
    const uint64_t* caps;
    uint64_t n;
    int32_t* status;
    uint64_t* written;
    _Atomic uint64_t cursor;
    lz4_dec_t lz4_dec;
    zstd_dec_t zstd_dec;
    zstd_create_t zstd_create;
    zstd_free_t zstd_free;
    zstd_iserr_t zstd_iserr;
};

static void* codec_worker(void* arg) {
    struct codec_job* j = (struct codec_job*)arg;
    void* dctx = (j->kind == 1) ? j->zstd_create() : NULL;
    for (;;) {
        const uint64_t i = atomic_fetch_add(&j->cursor, 1);
        if (i >= j->n) break;
        if (j->kind == 0) {
            int r = -1;
            if (j->src_sizes[i] > 0 && j->src_sizes[i] <= 0x7fffffff &&
                j->caps[i] <= 0x7fffffff)
                r = j->lz4_dec((const char*)j->src[i], (char*)j->dst[i],
                               (int)j->src_sizes[i], (int)j->caps[i]);
            j->status[i] = r < 0 ? 2 : 0;
            j->written[i] = r < 0 ? 0 : (uint64_t)r;
        } else {
            size_t r = j->zstd_dec(dctx, j->dst[i], j->caps[i], j->src[i],
                                   j->src_sizes[i]);
            int bad = j->zstd_iserr(r) != 0;
            j->status[i] = bad ? 2 : 0;
            j->written[i] = bad ? 0 : (uint64_t)r;
        }
    }
    if (dctx) j->zstd_free(dctx);
    return NULL;
}

/* Decodes n chunks with `threads` workers; returns the worker count used, or
 * -1 when the codec library is absent. */
int codec_decode_batch(int kind, const uint8_t* const* src,
                       const uint64_t* src_sizes, uint8_t* const* dst,
                       const uint64_t* caps, uint64_t n, int32_t* status,
                       uint64_t* written, int threads) {
    struct codec_job j = {0};
    j.kind = kind;
    j.src = src;
    j.src_sizes = src_sizes;
    j.dst = dst;
    j.caps = caps;
    j.n = n;
    j.status = status;
    j.written = written;
    if (kind == 0) {
        void* h = lz4_lib();
        if (!h) return -1;
        j.lz4_dec = (lz4_dec_t)dlsym(h, "LZ4_decompress_safe");
        if (!j.lz4_dec) return -1;
    } else {
        void* h = zstd_lib();
        if (!h) return -1;
        j.zstd_dec = (zstd_dec_t)dlsym(h, "ZSTD_decompressDCtx");
        j.zstd_create = (zstd_create_t)dlsym(h, "ZSTD_createDCtx");
        j.zstd_free = (zstd_free_t)dlsym(h, "ZSTD_freeDCtx");
        j.zstd_iserr = (zstd_iserr_t)dlsym(h, "ZSTD_isError");
        if (!j.zstd_dec || !j.zstd_create || !j.zstd_free || !j.zstd_iserr)
            return -1;
    }
    if (threads < 1) threads = 1;
    if (threads > 1024) threads = 1024;
    pthread_t tids[1024];
    int started = 0;
    for (int t = 1; t < threads; t++)
        if (pthread_create(&tids[started], NULL, codec_worker, &j) == 0) started++;
    codec_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(tids[t], NULL);
    return started + 1;
}
