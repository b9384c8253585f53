/* GDeflate page encoder and TileStream writer: synthetic-input generation for
 * the tests and the benchmark (built into libcudec_workload.so, never into
 * the decode library).
 *
 * The reference holds no GDeflate encoder (its dossier records the NVIDIA
 * libdeflate fork as the oracle it would fetch), so pages are produced here
 * from the format description: LZ77 parsing with hash chains, one Huffman
 * block per group of tokens (dynamic, static or stored, whichever is
 * smallest), and the 32-lane interleaving. Every field is appended to the bit
 * stream of the lane that will read it, in the decoder's round structure (the
 * decisions listed in the decoder's header comment), and the page's word
 * order is then laid out by replaying the decoder's refill schedule: the
 * priming round takes word 0 of every lane, and after each round every lane
 * below 32 buffered bits, in lane order, takes its next word.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GL 32
#define MAXLIT 288
#define MAXDIST 32

typedef struct {
    uint8_t* b;
    size_t cap, bits;
} lanebuf;

typedef struct {
    lanebuf lane[GL];
    uint32_t round_bits[GL], left[GL], nw[GL];
    uint32_t* order;
    size_t norder, ocap;
    int err;
} genc;

static void lb_put(lanebuf* l, uint32_t v, int n, int* err) {
    for (int i = 0; i < n; ++i) {
        const size_t byte = l->bits >> 3;
        if (byte >= l->cap) {
            const size_t nc = l->cap ? l->cap * 2 : 256;
            uint8_t* nb = (uint8_t*)realloc(l->b, nc);
            if (!nb) {
                *err = 1;
                return;
            }
            memset(nb + l->cap, 0, nc - l->cap);
            l->b = nb;
            l->cap = nc;
        }
        if ((v >> i) & 1u) l->b[byte] |= (uint8_t)(1u << (l->bits & 7));
        l->bits++;
    }
}

static void put(genc* e, int lane, uint32_t v, int n) {
    lb_put(&e->lane[lane], v, n, &e->err);
    e->round_bits[lane] += (uint32_t)n;
}

static void push_word(genc* e, uint32_t lane) {
    if (e->norder == e->ocap) {
        const size_t nc = e->ocap ? e->ocap * 2 : 1024;
        uint32_t* no = (uint32_t*)realloc(e->order, nc * sizeof(uint32_t));
        if (!no) {
            e->err = 1;
            return;
        }
        e->order = no;
        e->ocap = nc;
    }
    e->order[e->norder++] = (lane << 24) | e->nw[lane]++;
}

/* The decoder's refill turns after a round, in lane order. */
static void round_end(genc* e) {
    for (uint32_t l = 0; l < GL; ++l) {
        e->left[l] -= e->round_bits[l];
        e->round_bits[l] = 0;
        if (e->left[l] < 32) {
            push_word(e, l);
            e->left[l] += 32;
        }
    }
}

/* ---- Huffman ------------------------------------------------------- */

typedef struct {
    uint32_t f;
    int s;
} leaf;

static int cmp_leaf(const void* a, const void* b) {
    const leaf* x = (const leaf*)a;
    const leaf* y = (const leaf*)b;
    if (x->f != y->f) return x->f < y->f ? -1 : 1;
    return x->s - y->s;
}

/* Length-limited code lengths: Huffman by two queues, frequencies halved
 * (kept non-zero) until the longest code fits `limit`. */
static void huff_lengths(const uint32_t* freq_in, int n, int limit, uint8_t* lens) {
    uint32_t freq[MAXLIT];
    memcpy(freq, freq_in, sizeof(uint32_t) * (size_t)n);
    memset(lens, 0, (size_t)n);
    for (;;) {
        leaf lv[MAXLIT];
        int m = 0;
        for (int s = 0; s < n; ++s)
            if (freq[s]) {
                lv[m].f = freq[s];
                lv[m].s = s;
                ++m;
            }
        if (m == 0) return;
        if (m == 1) {
            lens[lv[0].s] = 1;
            return;
        }
        qsort(lv, (size_t)m, sizeof(leaf), cmp_leaf);
        /* nodes: 0..m-1 leaves, m.. internal */
        uint64_t w[2 * MAXLIT];
        int parent[2 * MAXLIT];
        for (int i = 0; i < m; ++i) w[i] = lv[i].f;
        int li = 0, ii = m, next = m;
        for (int k = 0; k < m - 1; ++k) {
            int pick[2];
            for (int t = 0; t < 2; ++t) {
                if (li < m && (ii >= next || w[li] <= w[ii])) pick[t] = li++;
                else pick[t] = ii++;
            }
            w[next] = w[pick[0]] + w[pick[1]];
            parent[pick[0]] = parent[pick[1]] = next;
            ++next;
        }
        int depth[2 * MAXLIT];
        depth[next - 1] = 0;
        for (int i = next - 2; i >= 0; --i) depth[i] = depth[parent[i]] + 1;
        int maxd = 0;
        for (int i = 0; i < m; ++i) maxd = depth[i] > maxd ? depth[i] : maxd;
        if (maxd <= limit) {
            for (int i = 0; i < m; ++i) lens[lv[i].s] = (uint8_t)depth[i];
            return;
        }
        for (int s = 0; s < n; ++s)
            if (freq[s]) freq[s] = (freq[s] >> 1) | 1u;
    }
}

static uint32_t rev(uint32_t c, int n) {
    uint32_t r = 0;
    for (int i = 0; i < n; ++i) r |= ((c >> i) & 1u) << (n - 1 - i);
    return r;
}

/* Canonical codes (RFC 1951 section 3.2.2), bit-reversed for LSB-first output. */
static void canon(const uint8_t* lens, int n, uint32_t* codes) {
    uint32_t cnt[16] = {0}, nxt[16];
    for (int s = 0; s < n; ++s) cnt[lens[s]]++;
    cnt[0] = 0;
    uint32_t code = 0;
    for (int b = 1; b < 16; ++b) {
        code = (code + cnt[b - 1]) << 1;
        nxt[b] = code;
    }
    for (int s = 0; s < n; ++s)
        codes[s] = lens[s] ? rev(nxt[lens[s]]++, lens[s]) : 0;
}

static const uint16_t kLBase[29] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  13,
                                    15, 17, 19, 23, 27, 31, 35, 43,  51,  59,
                                    67, 83, 99, 115, 131, 163, 195, 227, 3};
static const uint8_t kLExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                    2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 16};
static const uint32_t kDBase[32] = {1,     2,     3,     4,     5,     7,    9,    13,
                                    17,    25,    33,    49,    65,    97,   129,  193,
                                    257,   385,   513,   769,   1025,  1537, 2049, 3073,
                                    4097,  6145,  8193,  12289, 16385, 24577, 32769, 49153};
static const uint8_t kDExtra[32] = {0, 0, 0, 0, 1, 1, 2, 2, 3,  3,  4,  4,  5,  5,  6,  6,
                                    7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14};
static const uint8_t kPerm[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 11, 12, 13, 14, 15, 5, 4, 3, 2, 1};

static int len_code(uint32_t L) {
    if (L > 258) return 28;
    int c = 27;
    while (c > 0 && kLBase[c] > L) --c;
    return c;
}

static int dist_code(uint32_t d) {
    int c = 31;
    while (c > 0 && kDBase[c] > d) --c;
    return c;
}

/* ---- LZ77 ---------------------------------------------------------- */

typedef struct {
    uint32_t len, dist;  /* len 0: literal `dist` */
} tok;

static size_t lz77(const uint8_t* in, size_t n, tok* t, int level, uint32_t window) {
    const int chain = level <= 3 ? 16 : level <= 8 ? 128 : 1024;
    const int lazy = level >= 4;
    int32_t head[1 << 15];
    int32_t* prev = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    for (int i = 0; i < (1 << 15); ++i) head[i] = -1;
    size_t nt = 0, i = 0;
#define HASH(p) ((((uint32_t)in[p] << 10) ^ ((uint32_t)in[(p) + 1] << 5) ^ in[(p) + 2]) & 0x7FFF)
#define INSERT(p)                          \
    do {                                   \
        if ((p) + 3 <= n) {                \
            const uint32_t h_ = HASH(p);   \
            prev[p] = head[h_];            \
            head[h_] = (int32_t)(p);       \
        }                                  \
    } while (0)
    while (i < n) {
        uint32_t bl = 0, bd = 0;
        if (i + 3 <= n) {
            int32_t c = head[HASH(i)];
            int steps = chain;
            const uint32_t maxl = (uint32_t)(n - i < 258 ? n - i : 258);
            while (c >= 0 && steps-- > 0 && i - (size_t)c <= window) {
                uint32_t l = 0;
                while (l < maxl && in[(size_t)c + l] == in[i + l]) ++l;
                if (l > bl) {
                    bl = l;
                    bd = (uint32_t)(i - (size_t)c);
                    if (l == maxl) break;
                }
                c = prev[c];
            }
        }
        if (bl >= 3 && lazy && i + 4 <= n) {
            /* one-step lazy evaluation */
            INSERT(i);
            int32_t c = head[HASH(i + 1)];
            int steps = chain / 4 + 1;
            const uint32_t maxl = (uint32_t)(n - i - 1 < 258 ? n - i - 1 : 258);
            uint32_t bl2 = 0;
            while (c >= 0 && steps-- > 0 && i + 1 - (size_t)c <= window) {
                uint32_t l = 0;
                while (l < maxl && in[(size_t)c + l] == in[i + 1 + l]) ++l;
                if (l > bl2) bl2 = l;
                c = prev[c];
            }
            if (bl2 > bl + 1) {
                t[nt].len = 0;
                t[nt].dist = in[i];
                ++nt;
                ++i;
                continue;
            }
            t[nt].len = bl;
            t[nt].dist = bd;
            ++nt;
            for (size_t k = 1; k < bl; ++k) INSERT(i + k);
            i += bl;
            continue;
        }
        if (bl >= 3) {
            t[nt].len = bl;
            t[nt].dist = bd;
            ++nt;
            for (size_t k = 0; k < bl; ++k) INSERT(i + k);
            i += bl;
        } else {
            t[nt].len = 0;
            t[nt].dist = in[i];
            ++nt;
            INSERT(i);
            ++i;
        }
    }
#undef HASH
#undef INSERT
    free(prev);
    return nt;
}

/* ---- blocks -------------------------------------------------------- */

typedef struct {
    uint8_t llen[MAXLIT], dlen[MAXDIST], plen[19];
    uint32_t lcode[MAXLIT], dcode[MAXDIST], pcode[19];
    int hlit, hdist, hclen;
    uint8_t rle_sym[MAXLIT + MAXDIST];
    uint8_t rle_extra[MAXLIT + MAXDIST];
    int nrle;
} dyn;

static void rle_lengths(dyn* d) {
    uint8_t all[MAXLIT + MAXDIST];
    const int total = d->hlit + d->hdist;
    memcpy(all, d->llen, (size_t)d->hlit);
    memcpy(all + d->hlit, d->dlen, (size_t)d->hdist);
    int i = 0;
    d->nrle = 0;
    while (i < total) {
        int run = 1;
        while (i + run < total && all[i + run] == all[i]) ++run;
        if (all[i] == 0 && run >= 3) {
            int r = run;
            while (r >= 3) {
                if (r >= 11) {
                    const int k = r > 138 ? 138 : r;
                    d->rle_sym[d->nrle] = 18;
                    d->rle_extra[d->nrle++] = (uint8_t)(k - 11);
                    r -= k;
                } else {
                    const int k = r > 10 ? 10 : r;
                    d->rle_sym[d->nrle] = 17;
                    d->rle_extra[d->nrle++] = (uint8_t)(k - 3);
                    r -= k;
                }
            }
            while (r-- > 0) {
                d->rle_sym[d->nrle] = 0;
                d->rle_extra[d->nrle++] = 0;
            }
            i += run;
        } else if (all[i] != 0 && run >= 4) {
            d->rle_sym[d->nrle] = all[i];
            d->rle_extra[d->nrle++] = 0;
            int r = run - 1;
            while (r >= 3) {
                const int k = r > 6 ? 6 : r;
                d->rle_sym[d->nrle] = 16;
                d->rle_extra[d->nrle++] = (uint8_t)(k - 3);
                r -= k;
            }
            while (r-- > 0) {
                d->rle_sym[d->nrle] = all[i];
                d->rle_extra[d->nrle++] = 0;
            }
            i += run;
        } else {
            d->rle_sym[d->nrle] = all[i];
            d->rle_extra[d->nrle++] = 0;
            ++i;
        }
    }
}

static const int kRleExtraBits[19] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                      0, 0, 0, 0, 0, 0, 2, 3, 7};

static uint64_t data_bits(const tok* t, size_t a, size_t b, const uint8_t* ll, const uint8_t* dl) {
    uint64_t bits = ll[256];
    for (size_t k = a; k < b; ++k) {
        if (t[k].len == 0) {
            bits += ll[t[k].dist];
        } else {
            const int lc = len_code(t[k].len), dc = dist_code(t[k].dist);
            bits += ll[257 + lc] + kLExtra[lc] + dl[dc] + kDExtra[dc];
        }
    }
    return bits;
}

static void emit_data(genc* e, const tok* t, size_t a, size_t b, const uint32_t* lc_,
                      const uint8_t* ll, const uint32_t* dc_, const uint8_t* dl) {
    long pend[GL];
    for (int l = 0; l < GL; ++l) pend[l] = -1;
    size_t ti = a;
    int eob = 0, npend = 0;
    for (;;) {
        int eob_now = 0;
        for (int l = 0; l < GL; ++l) {
            if (pend[l] >= 0) {
                const tok* x = &t[pend[l]];
                const int dc = dist_code(x->dist);
                put(e, l, dc_[dc], dl[dc]);
                put(e, l, x->dist - kDBase[dc], kDExtra[dc]);
                pend[l] = -1;
                --npend;
            } else if (!eob && !eob_now) {
                if (ti < b) {
                    const tok* x = &t[ti];
                    if (x->len == 0) {
                        put(e, l, lc_[x->dist], ll[x->dist]);
                    } else {
                        const int c = len_code(x->len);
                        put(e, l, lc_[257 + c], ll[257 + c]);
                        put(e, l, x->len - kLBase[c], kLExtra[c]);
                        pend[l] = (long)ti;
                        ++npend;
                    }
                    ++ti;
                } else {
                    put(e, l, lc_[256], ll[256]);
                    eob_now = 1;
                }
            }
        }
        round_end(e);
        if (eob_now) eob = 1;
        if (eob && npend == 0) break;
    }
}

static void emit_block(genc* e, const uint8_t* raw, size_t raw_a, size_t raw_b, const tok* t,
                       size_t a, size_t b, int final) {
    uint32_t lf[MAXLIT] = {0}, df[MAXDIST] = {0};
    for (size_t k = a; k < b; ++k) {
        if (t[k].len == 0) {
            lf[t[k].dist]++;
        } else {
            lf[257 + len_code(t[k].len)]++;
            df[dist_code(t[k].dist)]++;
        }
    }
    lf[256] = 1;
    dyn d;
    huff_lengths(lf, MAXLIT, 15, d.llen);
    huff_lengths(df, MAXDIST, 15, d.dlen);
    int anyd = 0;
    for (int s = 0; s < MAXDIST; ++s) anyd |= d.dlen[s];
    if (!anyd) d.dlen[0] = 1;
    d.hlit = 286;
    while (d.hlit > 257 && d.llen[d.hlit - 1] == 0) --d.hlit;
    d.hdist = 32;
    while (d.hdist > 1 && d.dlen[d.hdist - 1] == 0) --d.hdist;
    rle_lengths(&d);
    uint32_t pf[19] = {0};
    for (int k = 0; k < d.nrle; ++k) pf[d.rle_sym[k]]++;
    huff_lengths(pf, 19, 7, d.plen);
    d.hclen = 19;
    while (d.hclen > 4 && d.plen[kPerm[d.hclen - 1]] == 0) --d.hclen;
    canon(d.llen, MAXLIT, d.lcode);
    canon(d.dlen, MAXDIST, d.dcode);
    canon(d.plen, 19, d.pcode);

    uint8_t sl[MAXLIT], sd[MAXDIST];
    for (int s = 0; s < MAXLIT; ++s) sl[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
    for (int s = 0; s < MAXDIST; ++s) sd[s] = 5;
    uint64_t dyn_bits = 17 + 3ull * (uint64_t)d.hclen + data_bits(t, a, b, d.llen, d.dlen);
    for (int k = 0; k < d.nrle; ++k)
        dyn_bits += d.plen[d.rle_sym[k]] + (uint64_t)kRleExtraBits[d.rle_sym[k]];
    const uint64_t st_bits = 3 + data_bits(t, a, b, sl, sd);
    const size_t raw_len = raw_b - raw_a;
    const uint64_t stored_bits = raw_len <= 65535 ? 19 + 8ull * raw_len : ~0ull;

    if (stored_bits <= dyn_bits && stored_bits <= st_bits) {
        put(e, 0, (uint32_t)final, 1);
        put(e, 0, 0, 2);
        round_end(e);
        put(e, 0, (uint32_t)raw_len, 16);
        round_end(e);
        for (size_t r = 0; r * GL < raw_len; ++r) {
            for (size_t l = 0; l < GL; ++l)
                if (r * GL + l < raw_len) put(e, (int)l, raw[raw_a + r * GL + l], 8);
            round_end(e);
        }
        return;
    }
    if (st_bits <= dyn_bits) {
        uint32_t lc[MAXLIT], dc[MAXDIST];
        canon(sl, MAXLIT, lc);
        canon(sd, MAXDIST, dc);
        put(e, 0, (uint32_t)final, 1);
        put(e, 0, 1, 2);
        round_end(e);
        emit_data(e, t, a, b, lc, sl, dc, sd);
        return;
    }
    put(e, 0, (uint32_t)final, 1);
    put(e, 0, 2, 2);
    round_end(e);
    put(e, 0, (uint32_t)(d.hlit - 257), 5);
    put(e, 0, (uint32_t)(d.hdist - 1), 5);
    put(e, 0, (uint32_t)(d.hclen - 4), 4);
    round_end(e);
    for (int l = 0; l < d.hclen; ++l) put(e, l, d.plen[kPerm[l]], 3);
    round_end(e);
    for (int k = 0; k < d.nrle;) {
        for (int l = 0; l < GL && k < d.nrle; ++l, ++k) {
            const int s = d.rle_sym[k];
            put(e, l, d.pcode[s], d.plen[s]);
            put(e, l, d.rle_extra[k], kRleExtraBits[s]);
        }
        round_end(e);
    }
    emit_data(e, t, a, b, d.lcode, d.llen, d.dcode, d.dlen);
}

/* One page (n <= 65536 input bytes). Returns the page size in bytes, or 0 if
 * it does not fit out_cap (or on allocation failure). level 1..12 sets the
 * match search effort; window is the farthest match distance used. */
size_t gdeflate_compress_page(const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                              int level, uint32_t window) {
    if (n > 65536 || window == 0 || window > 65536) return 0;
    tok* t = (tok*)malloc(sizeof(tok) * (n ? n : 1));
    if (!t) return 0;
    const size_t nt = lz77(in, n, t, level, window);
    genc e;
    memset(&e, 0, sizeof(e));
    for (uint32_t l = 0; l < GL; ++l) {
        push_word(&e, l);
        e.left[l] = 32;
    }
    const size_t per_block = 16384;
    size_t ta = 0, ra = 0;
    do {
        const size_t tb = nt - ta > per_block ? ta + per_block : nt;
        size_t rb = ra;
        for (size_t k = ta; k < tb; ++k) rb += t[k].len ? t[k].len : 1;
        emit_block(&e, in, ra, rb, t, ta, tb, tb == nt);
        ta = tb;
        ra = rb;
    } while (ta < nt);
    size_t bytes = 0;
    if (!e.err && e.norder * 4 <= out_cap) {
        for (size_t k = 0; k < e.norder; ++k) {
            const uint32_t lane = e.order[k] >> 24, w = e.order[k] & 0xFFFFFFu;
            uint32_t v = 0;
            for (int j = 0; j < 4; ++j) {
                const size_t byte = (size_t)w * 4 + (size_t)j;
                const uint32_t b = byte < e.lane[lane].cap ? e.lane[lane].b[byte] : 0;
                v |= b << (8 * j);
            }
            out[4 * k] = (uint8_t)v;
            out[4 * k + 1] = (uint8_t)(v >> 8);
            out[4 * k + 2] = (uint8_t)(v >> 16);
            out[4 * k + 3] = (uint8_t)(v >> 24);
        }
        bytes = e.norder * 4;
    }
    for (int l = 0; l < GL; ++l) free(e.lane[l].b);
    free(e.order);
    free(t);
    return bytes;
}

/* TileStream container of gdeflate pages for n input bytes: header (id 4,
 * magic 0xFB, tile count, 64 KiB tile size index, last tile size), the table
 * (entry 0 = last tile's compressed size, then tile offsets) and the pages.
 * Returns the stream size, or 0 if it does not fit. */
size_t gdeflate_compress_tilestream(const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                                    int level, uint32_t window) {
    const size_t tiles = n ? (n + 65535) / 65536 : 1;
    if (tiles > 65535) return 0;
    const size_t toc = 8 + 4 * tiles;
    if (out_cap < toc) return 0;
    size_t at = toc, last_src = 0;
    for (size_t k = 0; k < tiles; ++k) {
        const size_t a = k * 65536, len = n - a < 65536 ? n - a : 65536;
        const size_t got = gdeflate_compress_page(in + a, len, out + at, out_cap - at, level, window);
        if (got == 0) return 0;
        if (k > 0) {
            const uint32_t off = (uint32_t)at;
            memcpy(out + 8 + 4 * k, &off, 4);
        }
        if (k == tiles - 1) last_src = got;
        at += got;
    }
    const size_t last_dst = n - (tiles - 1) * 65536;
    const uint32_t packed = 1u | ((uint32_t)(last_dst == 65536 ? 0 : last_dst) << 2);
    out[0] = 4;
    out[1] = 0xFB;
    out[2] = (uint8_t)tiles;
    out[3] = (uint8_t)(tiles >> 8);
    memcpy(out + 4, &packed, 4);
    const uint32_t ls = (uint32_t)last_src;
    memcpy(out + 8, &ls, 4);
    return at;
}
