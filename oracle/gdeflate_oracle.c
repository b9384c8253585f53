/* GDeflate page decoder and TileStream envelope parser: a plain-C CPU
 * restatement used only as test infrastructure (the checker for the CUDA
 * decoder), never as a product path.
 *
 * PARITY STATUS. The 32-lane refill schedule below restates iderex/cudec
 * src/gdeflate_schedule.h:108-268 (priming round, refill-current-lane-then-
 * rotate, 32-bit watermark, sticky failure, refusals on a refill past the last
 * word and on a pop wider than the lane) and is pinned against that header,
 * compiled from the reference's sources, on random pages and operation traces.
 * The TileStream envelope restates src/tilestream.h:117-261 and is pinned on
 * the reference's fuzz seeds. The symbol layer has no reference decoder and no
 * golden vectors anywhere in the reference: it follows the format description
 * the reference records (docs/MASTERPLAN.md:861-960, draft sections 5-11,
 * divergences D1-D6 from RFC 1951) plus the decisions listed at
 * `oracle_gdeflate_decode`. Symbol-level parity with the GDeflate reference decoder is
 * therefore UNPINNED.
 */
#include <stdint.h>
#include <string.h>

enum { G_OK = 0, G_CORRUPT = 2, G_TOO_SMALL = 3, G_INVALID = 1 };

/* ---------------------------------------------------------------------
 * Schedule (src/gdeflate_schedule.h:74-268). */
#define G_LANES 32u
#define G_WATERMARK 32u
#define G_MAX_POP 32u

typedef struct {
    uint64_t buf[G_LANES];
    uint32_t left[G_LANES];
    uint32_t idx;
    uint64_t cursor, words;
    int failed;
    const uint8_t* page;
} gsched;

static uint32_t gs_word(const uint8_t* p, uint64_t w) {
    const uint8_t* q = p + w * 4u;
    return (uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16) |
           ((uint32_t)q[3] << 24);
}

static void gs_ensure(gsched* s) {
    if (s->failed || s->left[s->idx] >= G_WATERMARK) return;
    if (s->cursor >= s->words) {
        s->failed = 1;
        return;
    }
    s->buf[s->idx] |= (uint64_t)gs_word(s->page, s->cursor) << s->left[s->idx];
    s->cursor += 1;
    s->left[s->idx] += 32u;
}

static void gs_advance(gsched* s) {
    if (s->failed) return;
    gs_ensure(s);
    if (s->failed) return;
    s->idx = (s->idx + 1u) % G_LANES;
}

static void gs_reset(gsched* s) {
    if (!s->failed) s->idx = 0;
}

static int gs_init(gsched* s, const uint8_t* page, uint64_t bytes) {
    for (uint32_t n = 0; n < G_LANES; ++n) {
        s->buf[n] = 0;
        s->left[n] = 0;
    }
    s->idx = 0;
    s->cursor = 0;
    s->failed = 0;
    s->page = page;
    s->words = bytes / 4u;
    if (bytes % 4u != 0u || s->words < G_LANES) {
        s->failed = 1;
        return 0;
    }
    for (uint32_t n = 0; n < G_LANES; ++n) gs_advance(s);
    return !s->failed;
}

static uint32_t gs_peek(const gsched* s, uint32_t n) {
    if (n == 0 || n > G_MAX_POP) return 0;
    return (uint32_t)(s->buf[s->idx] & (((uint64_t)1 << n) - 1));
}

static void gs_remove(gsched* s, uint32_t n) {
    if (s->failed) return;
    if (n > s->left[s->idx]) {
        s->failed = 1;
        return;
    }
    s->buf[s->idx] >>= n;
    s->left[s->idx] -= n;
}

static uint32_t gs_pop(gsched* s, uint32_t n) {
    if (s->failed) return 0;
    if (n > G_MAX_POP || n > s->left[s->idx]) {
        s->failed = 1;
        return 0;
    }
    const uint32_t v = gs_peek(s, n);
    gs_remove(s, n);
    return v;
}

/* Schedule trace for pinning against the reference header: ops[i] = 0
 * advance, 1..64 pop of that width, 100 reset, 200 ensure, 300 remove of
 * ops[i+1] bits (two slots). trace gets 4 words per op: cursor, idx, failed,
 * value (the pop's result, else 0). Returns the op count executed. */
int oracle_gdeflate_schedule_trace(const uint8_t* page, uint64_t bytes, const uint32_t* ops,
                                   uint64_t n_ops, uint64_t* trace) {
    gsched s;
    const int ok = gs_init(&s, page, bytes);
    trace[0] = s.cursor;
    trace[1] = s.idx;
    trace[2] = (uint64_t)s.failed;
    trace[3] = (uint64_t)ok;
    uint64_t t = 4, i = 0;
    while (i < n_ops) {
        const uint32_t op = ops[i++];
        uint64_t v = 0;
        if (op == 0) gs_advance(&s);
        else if (op <= 64) v = gs_pop(&s, op);
        else if (op == 100) gs_reset(&s);
        else if (op == 200) gs_ensure(&s);
        else if (op == 300 && i < n_ops) gs_remove(&s, ops[i++]);
        trace[t++] = s.cursor;
        trace[t++] = s.idx;
        trace[t++] = (uint64_t)s.failed;
        trace[t++] = v;
    }
    return (int)(t / 4);
}

/* ---------------------------------------------------------------------
 * Canonical Huffman codes, read most-significant code bit first from the
 * lane's least-significant end (RFC 1951 section 3.1.1 bit order). */
#define G_MAXBITS 15
#define G_PAGE_MAX 65536u /* a page never produces more */

typedef struct {
    uint16_t count[G_MAXBITS + 1];
    uint16_t symbol[320];
} ghuff;

/* 0 = usable (complete or incomplete), -1 = over-subscribed. */
static int gh_build(ghuff* h, const uint8_t* lens, int n) {
    uint16_t offs[G_MAXBITS + 2];
    memset(h->count, 0, sizeof(h->count));
    for (int s = 0; s < n; ++s) h->count[lens[s]]++;
    int left = 1;
    for (int len = 1; len <= G_MAXBITS; ++len) {
        left <<= 1;
        left -= h->count[len];
        if (left < 0) return -1;
    }
    offs[1] = 0;
    for (int len = 1; len < G_MAXBITS; ++len) offs[len + 1] = offs[len] + h->count[len];
    for (int s = 0; s < n; ++s)
        if (lens[s]) h->symbol[offs[lens[s]]++] = (uint16_t)s;
    return 0;
}

/* One code from the current lane; -1 for a code no symbol has. The lane holds
 * at least 32 bits whenever this runs, so single-bit pops cannot fail. */
static int gh_decode(gsched* s, const ghuff* h) {
    int code = 0, first = 0, index = 0;
    for (int len = 1; len <= G_MAXBITS; ++len) {
        code |= (int)gs_pop(s, 1);
        const int count = h->count[len];
        if (code - count < first) return h->symbol[index + (code - first)];
        index += count;
        first += count;
        first <<= 1;
        code <<= 1;
    }
    return -1;
}

/* Length codes 257..285 (D1: 285 = 3 + 16 extra bits) and distance codes
 * 0..31 (D2: 30, 31 = 32769 / 49153 + 14 extra bits). */
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

/* Ends a round: every lane after the ones that acted gets its refill turn, in
 * lane order, ending back at lane 0 (the schedule's Advance, 32 times from
 * lane 0). */
static void round_rest(gsched* s) {
    while (!s->failed) {
        gs_advance(s);
        if (s->idx == 0) break;
    }
}

/* Decodes one page. Decisions for the points the format description leaves
 * open (all mirrored by the CUDA decoder and the encoder):
 *   - rounds: every round gives each of the 32 lanes, in lane order, at most
 *     one operation on its own bits followed by its refill turn (Advance);
 *     a block header is its own round on lane 0 (BFINAL 1 bit, BTYPE 2);
 *     stored and dynamic blocks then take a second lane-0 round (stored: a
 *     16-bit LEN; dynamic: HLIT 5, HDIST 5, HCLEN 4);
 *   - dynamic tables: one round with lanes 0..HCLEN+3 reading a 3-bit precode
 *     length each (RFC permutation order), then rounds of up to 32 code-length
 *     symbols, lane l active while fewer than HLIT+HDIST lengths are known;
 *     repeat runs may not cross the end (CORRUPT), code 16 needs a previous
 *     length; over-subscribed codes are CORRUPT, incomplete ones usable (a
 *     code with no symbol is CORRUPT when read); litlen length of 256 must
 *     be non-zero; HLIT+257 <= 288 and HDIST+1 <= 32;
 *   - data rounds: a lane with a pending copy reads its distance symbol (and
 *     its extra bits) in the next round; other lanes read one litlen symbol
 *     each while no lane before them (this round) or in an earlier round of
 *     the block read end-of-block; the block ends after the round where
 *     end-of-block has been read and no distance is pending; symbols 286/287
 *     are CORRUPT;
 *   - stored blocks: LEN bytes as 8-bit atoms, byte 32r+l on lane l of round r;
 *   - checks per operation in this order: symbol, extra bits, the page's
 *     64 KiB output limit (CORRUPT), output room (OUTPUT_TOO_SMALL),
 *     distance within the page output (CORRUPT); a refill with no word left
 *     is CORRUPT at that lane's refill turn;
 *   - the page must be consumed exactly: after the final block's last round
 *     the schedule's word cursor must equal the page's word count.
 * cap is the output capacity (bytes_written <= cap). */
int oracle_gdeflate_decode(const uint8_t* page, uint64_t size, uint8_t* out, uint64_t cap,
                           uint64_t* written) {
    *written = 0;
    gsched s;
    if (!gs_init(&s, page, size)) return G_CORRUPT;
    uint64_t pos = 0;
    ghuff lit, dist, pre;
    int final = 0;
    while (!final) {
        gs_reset(&s);
        final = (int)gs_pop(&s, 1);
        const uint32_t btype = gs_pop(&s, 2);
        round_rest(&s);
        if (s.failed) return G_CORRUPT;
        if (btype == 3) return G_CORRUPT;
        if (btype == 0) {
            const uint32_t len = gs_pop(&s, 16);
            round_rest(&s);
            if (s.failed) return G_CORRUPT;
            for (uint32_t r = 0; r * 32u < len; ++r) {
                for (uint32_t l = 0; l < G_LANES; ++l) {
                    if (r * 32u + l < len) {
                        const uint32_t b = gs_pop(&s, 8);
                        if (pos >= G_PAGE_MAX) return G_CORRUPT;
                        if (pos >= cap) return G_TOO_SMALL;
                        out[pos++] = (uint8_t)b;
                    }
                    gs_advance(&s);
                    if (s.failed) return G_CORRUPT;
                }
            }
            continue;
        }
        if (btype == 1) {
            uint8_t l[320];
            int i = 0;
            for (; i < 144; ++i) l[i] = 8;
            for (; i < 256; ++i) l[i] = 9;
            for (; i < 280; ++i) l[i] = 7;
            for (; i < 288; ++i) l[i] = 8;
            gh_build(&lit, l, 288);
            for (i = 0; i < 32; ++i) l[i] = 5;
            gh_build(&dist, l, 32);
        } else {
            const uint32_t hlit = gs_pop(&s, 5) + 257, hdist = gs_pop(&s, 5) + 1,
                           hclen = gs_pop(&s, 4) + 4;
            round_rest(&s);
            if (s.failed) return G_CORRUPT;
            if (hlit > 288 || hdist > 32) return G_CORRUPT;
            uint8_t plen[19];
            memset(plen, 0, sizeof(plen));
            for (uint32_t l = 0; l < G_LANES; ++l) {
                if (l < hclen) plen[kPerm[l]] = (uint8_t)gs_pop(&s, 3);
                gs_advance(&s);
                if (s.failed) return G_CORRUPT;
            }
            if (gh_build(&pre, plen, 19) != 0) return G_CORRUPT;
            uint8_t lens[320];
            const uint32_t total = hlit + hdist;
            uint32_t have = 0;
            while (have < total) {
                for (uint32_t l = 0; l < G_LANES; ++l) {
                    if (have < total) {
                        const int sym = gh_decode(&s, &pre);
                        if (sym < 0) return G_CORRUPT;
                        if (sym < 16) {
                            lens[have++] = (uint8_t)sym;
                        } else {
                            uint32_t rep;
                            uint8_t val = 0;
                            if (sym == 16) {
                                if (have == 0) return G_CORRUPT;
                                val = lens[have - 1];
                                rep = 3 + gs_pop(&s, 2);
                            } else if (sym == 17) {
                                rep = 3 + gs_pop(&s, 3);
                            } else {
                                rep = 11 + gs_pop(&s, 7);
                            }
                            if (have + rep > total) return G_CORRUPT;
                            while (rep--) lens[have++] = val;
                        }
                    }
                    gs_advance(&s);
                    if (s.failed) return G_CORRUPT;
                }
            }
            if (lens[256] == 0) return G_CORRUPT;
            if (gh_build(&lit, lens, (int)hlit) != 0) return G_CORRUPT;
            if (gh_build(&dist, lens + hlit, (int)hdist) != 0) return G_CORRUPT;
        }
        /* data rounds */
        uint64_t pend_pos[G_LANES], pend_len[G_LANES];
        int pend[G_LANES];
        for (uint32_t l = 0; l < G_LANES; ++l) pend[l] = 0;
        int eob = 0, npend = 0;
        for (;;) {
            int eob_now = 0;
            for (uint32_t l = 0; l < G_LANES; ++l) {
                if (pend[l]) {
                    const int d = gh_decode(&s, &dist);
                    if (d < 0 || d >= 32) return G_CORRUPT;
                    const uint64_t dd = kDBase[d] + gs_pop(&s, kDExtra[d]);
                    if (dd > pend_pos[l]) return G_CORRUPT;
                    for (uint64_t k = 0; k < pend_len[l]; ++k)
                        out[pend_pos[l] + k] = out[pend_pos[l] + k - dd];
                    pend[l] = 0;
                    --npend;
                } else if (!eob && !eob_now) {
                    const int sym = gh_decode(&s, &lit);
                    if (sym < 0 || sym > 285) return G_CORRUPT;
                    if (sym < 256) {
                        if (pos >= G_PAGE_MAX) return G_CORRUPT;
                        if (pos >= cap) return G_TOO_SMALL;
                        out[pos++] = (uint8_t)sym;
                    } else if (sym == 256) {
                        eob_now = 1;
                    } else {
                        const uint64_t L = kLBase[sym - 257] + gs_pop(&s, kLExtra[sym - 257]);
                        if (L > G_PAGE_MAX - pos) return G_CORRUPT;
                        if (L > cap - pos) return G_TOO_SMALL;
                        pend_pos[l] = pos;
                        pend_len[l] = L;
                        pend[l] = 1;
                        ++npend;
                        pos += L;
                    }
                }
                gs_advance(&s);
                if (s.failed) return G_CORRUPT;
            }
            if (eob_now) eob = 1;
            if (eob && npend == 0) break;
        }
    }
    if (s.cursor != s.words) return G_CORRUPT;
    *written = pos;
    return G_OK;
}

/* ---------------------------------------------------------------------
 * TileStream envelope (src/tilestream.h:117-261): 8-byte header (id =
 * magic ^ 0xFF, u16 tile count, packed u32: 2-bit tile size index = 1 for
 * 64 KiB, 18-bit last tile size with 0 = full, 12 reserved bits = 0), then
 * a u32 table whose entry 0 is the last tile's compressed size and entries
 * 1.. the other tiles' offsets (strictly increasing, after the table).
 * tiles[3*i] = src offset, [3*i+1] = src size, [3*i+2] = dst size. */
static uint32_t rd32(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
           ((uint32_t)p[3] << 24);
}

int oracle_tilestream_parse(const uint8_t* st, uint64_t size, uint64_t* tiles,
                            uint64_t tiles_cap, uint64_t* count, uint64_t* total) {
    if (st == NULL || tiles == NULL || count == NULL || total == NULL) return G_INVALID;
    if (size < 8) return G_CORRUPT;
    if (st[0] != (uint8_t)(st[1] ^ 0xFFu)) return G_CORRUPT;
    const uint64_t n = (uint64_t)st[2] | ((uint64_t)st[3] << 8);
    if (n == 0) return G_CORRUPT;
    const uint32_t packed = rd32(st + 4);
    const uint64_t last = (packed >> 2) & 0x3FFFFu;
    if ((packed & 3u) != 1u || ((packed >> 20) & 0xFFFu) != 0 || last >= 65536) return G_CORRUPT;
    if (tiles_cap < n) return G_INVALID;
    const uint64_t toc_end = 8 + 4 * n;
    if (size < toc_end) return G_CORRUPT;
    const uint64_t last_src = rd32(st + 8);
    if (last_src == 0) return G_CORRUPT;
    uint64_t prev = toc_end;
    for (uint64_t i = 1; i < n; ++i) {
        const uint64_t off = rd32(st + 8 + 4 * i);
        if (off <= prev) return G_CORRUPT;
        tiles[3 * i] = off;
        prev = off;
    }
    tiles[0] = toc_end;
    for (uint64_t i = 0; i + 1 < n; ++i) tiles[3 * i + 1] = tiles[3 * (i + 1)] - tiles[3 * i];
    tiles[3 * (n - 1) + 1] = last_src;
    if (tiles[3 * (n - 1)] + last_src > size) return G_CORRUPT;
    for (uint64_t i = 0; i + 1 < n; ++i) tiles[3 * i + 2] = 65536;
    tiles[3 * (n - 1) + 2] = last == 0 ? 65536 : last;
    *count = n;
    *total = n * 65536 - (last == 0 ? 0 : 65536 - last);
    return G_OK;
}
