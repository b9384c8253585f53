/* Seeded synthetic content for the benchmark and test workloads.
 *
 * The reference measures on Silesia/enwik8, which are not available here; the
 * workloads are instead synthetic chunks with the headline configurations'
 * sizes and the same statistics for every run: literal runs (geometric length) over a small
 * alphabet with Zipf frequencies, alternating with back-references (geometric
 * length, uniform offset), optionally with runs of one repeated byte, or whole
 * chunks of uniform random bytes. Deterministic in (seed, chunk index): the
 * stream is SplitMix64 and all sampling goes through it, as the reference's
 * fixture generator does (tests/fixtures.cpp:15-21 SplitMix64).
 *
 * Host-only; compiled into libcudec_workload.so. Not part of the decode ABI.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct gen_params {
    double copy_prob;    /* probability that an event is a back-reference */
    int alphabet;        /* literal symbols (<= 256) */
    double zipf_s;       /* Zipf exponent over the alphabet */
    double mean_lit;     /* geometric mean of a literal run (>= 1) */
    double mean_match;   /* geometric mean of a back-reference length */
    uint32_t min_match;  /* clamp */
    uint32_t max_match;  /* clamp */
    uint64_t max_offset; /* offsets are uniform in [1, min(pos, max_offset)] */
    double rle_prob;     /* probability that an event is a repeated-byte run */
    double mean_rle;     /* geometric mean of such a run */
    int random_bytes;    /* whole chunk is uniform random bytes */
} gen_params;

static inline uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double unit(uint64_t* s) { /* [0, 1) with 53 bits */
    return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
}

static inline uint64_t geometric(uint64_t* s, double mean) {
    if (mean <= 1.0) return 1;
    const double q = 1.0 / mean;
    const double u = unit(s);
    return 1 + (uint64_t)floor(log1p(-u) / log1p(-q));
}

/* Cumulative Zipf weights, alphabet <= 256. */
static void zipf_cdf(double* cdf, int a, double s) {
    double acc = 0;
    for (int k = 0; k < a; k++) {
        acc += 1.0 / pow((double)(k + 1), s);
        cdf[k] = acc;
    }
    for (int k = 0; k < a; k++) cdf[k] /= acc;
}

static inline uint8_t zipf_symbol(uint64_t* s, const double* cdf, int a) {
    const double u = unit(s);
    int lo = 0, hi = a - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] > u) hi = mid; else lo = mid + 1;
    }
    return (uint8_t)((lo * 167 + 13) & 255); /* rank -> byte, a bijection */
}

void gen_chunk(uint64_t seed, uint8_t* out, uint64_t size, const gen_params* p) {
    uint64_t s = seed;
    if (p->random_bytes) {
        uint64_t i = 0;
        for (; i + 8 <= size; i += 8) {
            uint64_t v = splitmix(&s);
            memcpy(out + i, &v, 8);
        }
        if (i < size) {
            uint64_t v = splitmix(&s);
            memcpy(out + i, &v, size - i);
        }
        return;
    }
    double cdf[256];
    const int a = p->alphabet < 1 ? 1 : (p->alphabet > 256 ? 256 : p->alphabet);
    zipf_cdf(cdf, a, p->zipf_s);
    uint64_t pos = 0;
    int first = 1;
    while (pos < size) {
        const double u = first ? 1.0 : unit(&s);
        first = 0;
        if (pos > 0 && u < p->rle_prob) {
            uint64_t len = geometric(&s, p->mean_rle);
            if (len > size - pos) len = size - pos;
            memset(out + pos, zipf_symbol(&s, cdf, a), len);
            pos += len;
        } else if (pos > 0 && u < p->rle_prob + p->copy_prob) {
            uint64_t len = geometric(&s, p->mean_match);
            if (len < p->min_match) len = p->min_match;
            if (len > p->max_match) len = p->max_match;
            if (len > size - pos) len = size - pos;
            const uint64_t span = pos < p->max_offset ? pos : p->max_offset;
            const uint64_t off = 1 + splitmix(&s) % span;
            for (uint64_t i = 0; i < len; i++) out[pos + i] = out[pos - off + i];
            pos += len;
        } else {
            uint64_t len = geometric(&s, p->mean_lit);
            if (len > size - pos) len = size - pos;
            for (uint64_t i = 0; i < len; i++) out[pos + i] = zipf_symbol(&s, cdf, a);
            pos += len;
        }
    }
}

/* Batch generation over a thread pool: chunk i is gen_chunk(seeds[i],
 * base + offsets[i], sizes[i], &params[param_idx[i]]). */
struct gen_job {
    const uint64_t* seeds;
    uint8_t* base;
    const uint64_t* offsets;
    const uint64_t* sizes;
    const gen_params* params;
    const int32_t* param_idx;
    uint64_t n;
    _Atomic uint64_t cursor;
};

static void* gen_worker(void* arg) {
    struct gen_job* j = (struct gen_job*)arg;
    for (;;) {
        uint64_t i = atomic_fetch_add(&j->cursor, 1);
        if (i >= j->n) break;
        gen_chunk(j->seeds[i], j->base + j->offsets[i], j->sizes[i],
                  &j->params[j->param_idx[i]]);
    }
    return NULL;
}

void gen_batch(const uint64_t* seeds, uint8_t* base, const uint64_t* offsets,
               const uint64_t* sizes, const gen_params* params,
               const int32_t* param_idx, uint64_t n, int threads) {
    struct gen_job j = {seeds, base, offsets, sizes, params, param_idx, n, 0};
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t t[256];
    int started = 0;
    for (int k = 1; k < threads; k++)
        if (pthread_create(&t[started], NULL, gen_worker, &j) == 0) started++;
    gen_worker(&j);
    for (int k = 0; k < started; k++) pthread_join(t[k], NULL);
}
