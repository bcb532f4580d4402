/* galn_oracle.c -- test infrastructure: the CPU restatement of the `bwa aln` search, of samse's coordinate
 * step and of the bwa index files (parity oracle).
 * See galn_oracle.h for what it covers and which reference lines each part follows. Compiled with
 * -ffp-contract=off so that bwa_cal_maxdiff rounds as the reference does (CMakeLists.txt:24-25).
 */
#define _GNU_SOURCE
#include "galn_oracle.h"

#include <ctype.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

enum { MODE_GAPE = 0x01, MODE_LOGGAP = 0x04, MODE_NONSTOP = 0x10 };
enum { ST_M = 0, ST_I = 1, ST_D = 2 };
enum { ERR_SCORE = -3 };
#define BATCH_READS 0x40000        /* bwa_read_seq batch size (host_io.h:16) */
#define FNV_OFFSET 1469598103934665603ULL
#define FNV_PRIME  1099511628211ULL

/* ------------------------------------------------------------------------------------------------ */
/* the index: BWA .bwt layout (idxcommon.h:6). Header: primary, C[1..4]; body: per 128 symbols, 4 u64
 * counts of each base before the block, then 8 u32 words of 2-bit symbols (first symbol in the top bits). */

typedef struct {
    uint64_t primary, L2[5], seq_len, words;
    uint32_t *body;
    int borrowed;                  /* body is the caller's memory (orc_index_borrow) */
} oindex_t;

/* the index over a .bwt file image already in memory (header words first), without a copy: the memory
 * must outlive the index and end with the four totals (as every .bwt does) */
void *orc_index_borrow(const uint32_t *file_words, uint64_t n_words, int *err)
{
    if (n_words < 10 + 8) { *err = -2; return NULL; }
    uint64_t hdr[5];
    memcpy(hdr, file_words, 40);
    oindex_t *x = (oindex_t*)calloc(1, sizeof(oindex_t));
    x->primary = hdr[0];
    x->L2[0] = 0;
    for (int c = 0; c < 4; ++c) x->L2[c + 1] = hdr[c + 1];
    x->seq_len = x->L2[4];
    x->words = n_words - 10;
    x->body = (uint32_t*)(file_words + 10);
    x->borrowed = 1;
    *err = 0;
    return x;
}

void *orc_index_load(const char *path, int *err)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) { *err = -1; return NULL; }
    uint64_t hdr[5];
    if (fread(hdr, 8, 5, fp) != 5) { fclose(fp); *err = -2; return NULL; }
    fseeko(fp, 0, SEEK_END);
    long long sz = ftello(fp);
    fseeko(fp, 40, SEEK_SET);
    oindex_t *x = (oindex_t*)calloc(1, sizeof(oindex_t));
    x->primary = hdr[0];
    x->L2[0] = 0;
    for (int c = 0; c < 4; ++c) x->L2[c + 1] = hdr[c + 1];
    x->seq_len = x->L2[4];
    x->words = (uint64_t)(sz - 40) / 4;
    x->body = (uint32_t*)malloc(x->words * 4 + 64);
    if (fread(x->body, 4, x->words, fp) != x->words) { fclose(fp); free(x->body); free(x); *err = -2; return NULL; }
    memset(x->body + x->words, 0, 64);
    fclose(fp);
    *err = 0;
    return x;
}

void orc_index_free(void *p)
{
    oindex_t *x = (oindex_t*)p;
    if (x) { if (!x->borrowed) free(x->body); free(x); }
}

int orc_index_meta(const void *p, uint64_t *primary, uint64_t L2[5], uint64_t *words)
{
    const oindex_t *x = (const oindex_t*)p;
    *primary = x->primary;
    memcpy(L2, x->L2, sizeof(x->L2));
    *words = x->words;
    return 0;
}

/* number of symbols equal to c among the first `take` (1..16) symbols of a packed word */
static inline uint32_t count_in_word(uint32_t w, int c, int take)
{
    uint32_t x = w ^ (0x55555555u * (uint32_t)c);             /* matching symbols become 00 */
    uint32_t hit = ~(x | (x >> 1)) & 0x55555555u;             /* low bit of each matching pair */
    if (take < 16) hit &= ~(0xffffffffu >> (2 * take));       /* keep the first `take` pairs */
    return (uint32_t)__builtin_popcount(hit);
}

/* Occ(c, k): occurrences of base c in BWT rows 0..k, the $ row not counted; Occ(c, -1) = 0 */
static uint64_t occ(const oindex_t *x, uint64_t k, int c)
{
    if (k == (uint64_t)-1) return 0;
    uint64_t p = k - (k >= x->primary);             /* index into the symbols with $ taken out */
    const uint32_t *blk = x->body + (p >> 7) * 16;
    uint64_t n;
    memcpy(&n, blk + 2 * c, 8);
    int upto = (int)(p & 127) + 1;                  /* symbols of this block that count */
    for (int w = 0; upto > 0; ++w, upto -= 16)
        n += count_in_word(blk[8 + w], c, upto < 16 ? upto : 16);
    return n;
}

void orc_occ4(const void *index, const uint64_t *rows, int64_t n, uint64_t *out)
{
    const oindex_t *x = (const oindex_t*)index;
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 4; ++c) out[4 * i + c] = occ(x, rows[i], c);
}

/* ------------------------------------------------------------------------------------------------ */
/* positions from suffix-array rows (samse's coordinate step) */

/* the BWT symbol of row k (k != primary): the $-free position k - (k > primary), from the packed words */
static int bwt_symbol(const oindex_t *x, uint64_t k)
{
    uint64_t p = k - (k > x->primary);
    uint32_t w = x->body[(p >> 7) * 16 + 8 + ((p & 127) >> 4)];
    return (int)((w >> ((~p & 15) << 1)) & 3);
}

/* bwt_sa (bwa's bwt.c:86-96 with bwt_invPsi, bwt.c:53-59): step back with invPsi(k) = L2[c] + Occ(c, k),
 * the $ row going to 0, until k is a multiple of intv; samples[k / intv] + steps (samples[0] = -1) */
uint64_t orc_bwt_sa(const void *index, const uint64_t *samples, uint64_t intv, uint64_t k)
{
    const oindex_t *x = (const oindex_t*)index;
    uint64_t sa = 0;
    while (k % intv) {
        ++sa;
        if (k == x->primary) { k = 0; continue; }
        int c = bwt_symbol(x, k);
        k = x->L2[c] + occ(x, k, c);
    }
    return sa + samples[k / intv];
}

/* bwa_sa2pos (src/samse/bwa_upstream/bwase.c:112-125) with bns_depos (bntseq.h:87-90); l_pac = seq_len / 2.
 * Returns the position (or (uint64)-1 for a hit across the forward/reverse boundary), strand = !is_rev. */
uint64_t orc_sa2pos(const void *index, const uint64_t *samples, uint64_t intv, uint64_t k, int ref_len, int *strand)
{
    const oindex_t *x = (const oindex_t*)index;
    uint64_t l_pac = x->seq_len / 2;
    uint64_t pos_f = orc_bwt_sa(index, samples, intv, k);
    *strand = 0;
    if (pos_f < l_pac && l_pac < pos_f + (uint64_t)(int64_t)ref_len) return (uint64_t)-1;
    int is_rev = pos_f >= l_pac;
    if (is_rev) pos_f = (l_pac << 1) - 1 - pos_f;
    *strand = !is_rev;
    if (is_rev) pos_f = pos_f + 1 < (uint64_t)(int64_t)ref_len ? 0 : pos_f - (uint64_t)(int64_t)ref_len + 1;
    return pos_f;
}

/* fetch accounting for the roofline: blocks touched by a lookup of (k', l') under a block size */
static inline uint64_t fetches(const oindex_t *x, uint64_t k, uint64_t l, int shift)
{
    int hk = k != (uint64_t)-1, hl = l != (uint64_t)-1;
    if (!hk || !hl) return (uint64_t)(hk + hl);
    uint64_t pk = k - (k >= x->primary), pl = l - (l >= x->primary);
    return (pk >> shift) == (pl >> shift) ? 1 : 2;
}

/* the same for blocks of `size` symbols that need not be a power of two (the build's 80-symbol layout) */
static inline uint64_t fetches_div(const oindex_t *x, uint64_t k, uint64_t l, uint64_t size)
{
    int hk = k != (uint64_t)-1, hl = l != (uint64_t)-1;
    if (!hk || !hl) return (uint64_t)(hk + hl);
    uint64_t pk = k - (k >= x->primary), pl = l - (l >= x->primary);
    return pk / size == pl / size ? 1 : 2;
}

/* ------------------------------------------------------------------------------------------------ */
/* per-read search state */

typedef struct { uint64_t w; int32_t bid; } width_t;

typedef struct {
    uint64_t k, l;
    uint32_t info;              /* score << 21 | i */
    int32_t last_diff_pos;
    uint8_t n_mm, n_gapo, n_gape, state;
    uint16_t n_ins, n_del;
} entry_t;

typedef struct { entry_t *v; long n, m; } bucket_t;

typedef struct { uint64_t packed, k, l; } rec_t;

typedef struct {
    /* options of this read (the batch's, with the read's max_diff and seed_len) */
    int s_mm, s_gapo, s_gape, mode, indel_end_skip, max_del_occ, max_entries;
    int max_diff, max_gapo, max_gape, max_seed_diff, seed_len, max_top2;
} ropt_t;

typedef struct {
    bucket_t *b;
    int nb, best;
    long n_entries, peak;
    uint64_t pops, trace, f128, f64, f80;
    rec_t *rec; long n_rec, m_rec;
    width_t *w, *sw; int w_cap, sw_cap;
} ws_t;

static inline int score_of(int m, int o, int e, const ropt_t *p)
{
    return m * p->s_mm + o * p->s_gapo + e * p->s_gape;
}

static int push(ws_t *s, const ropt_t *o, int i, uint64_t k, uint64_t l, int n_mm, int n_gapo, int n_gape,
                int n_ins, int n_del, int state, int is_diff)
{
    int sc = score_of(n_mm, n_gapo, n_gape, o);
    if (sc < 0 || sc >= s->nb) return ERR_SCORE;
    bucket_t *q = &s->b[sc];
    if (q->n == q->m) {
        q->m = q->m ? 2 * q->m : 16;
        q->v = (entry_t*)realloc(q->v, (size_t)q->m * sizeof(entry_t));
    }
    entry_t *e = &q->v[q->n++];
    e->k = k; e->l = l;
    e->info = (uint32_t)sc << 21 | (uint32_t)i;
    e->last_diff_pos = is_diff ? i : 0;
    e->n_mm = (uint8_t)n_mm; e->n_gapo = (uint8_t)n_gapo; e->n_gape = (uint8_t)n_gape;
    e->state = (uint8_t)state;
    e->n_ins = (uint16_t)n_ins; e->n_del = (uint16_t)n_del;
    if (++s->n_entries > s->peak) s->peak = s->n_entries;
    if (sc < s->best) s->best = sc;
    return 0;
}

static inline uint64_t mix(uint64_t h, uint64_t v) { return (h ^ v) * FNV_PRIME; }

static void pop(ws_t *s, entry_t *e)
{
    bucket_t *q = &s->b[s->best];
    *e = q->v[--q->n];
    --s->n_entries;
    ++s->pops;
    uint64_t h = s->trace;
    h = mix(h, e->info);
    h = mix(h, e->k);
    h = mix(h, e->l);
    h = mix(h, (uint64_t)(e->n_mm | e->n_gapo << 8 | e->n_gape << 16 | (uint32_t)e->state << 24));
    h = mix(h, (uint64_t)e->n_ins | (uint64_t)e->n_del << 16);
    h = mix(h, (uint64_t)(uint32_t)e->last_diff_pos);
    h = mix(h, (uint64_t)(uint32_t)s->n_entries);
    s->trace = h;
    if (s->n_entries == 0) s->best = s->nb;
    else if (q->n == 0) {
        int b = s->best + 1;
        while (b < s->nb && s->b[b].n == 0) ++b;
        s->best = b;
    }
}

/* (k, l) <- the interval of c prepended to (k, l): [C(c) + Occ(c, k-1) + 1, C(c) + Occ(c, l)] */
static inline void extend1(ws_t *s, const oindex_t *x, int c, uint64_t *k, uint64_t *l)
{
    s->f128 += fetches(x, *k - 1, *l, 7);
    s->f64 += fetches(x, *k - 1, *l, 6);
    s->f80 += fetches_div(x, *k - 1, *l, 80);
    uint64_t ok = occ(x, *k - 1, c), ol = occ(x, *l, c);
    *k = x->L2[c] + ok + 1;
    *l = x->L2[c] + ol;
}

/* bwt_cal_width on the read as the search sees it (reversed and complemented): the complement is undone
 * here, an ambiguous base restarts the interval like a mismatch does */
static int cal_width(ws_t *s, const oindex_t *x, int len, const uint8_t *q, width_t *w)
{
    uint64_t k = 0, l = x->seq_len;
    int bid = 0;
    for (int i = 0; i < len; ++i) {
        int c = q[i] > 3 ? 4 : 3 - q[i];
        if (c < 4) extend1(s, x, c, &k, &l);
        if (k > l || c > 3) { k = 0; l = x->seq_len; ++bid; }
        w[i].w = l - k + 1;
        w[i].bid = bid;
    }
    w[len].w = 0;
    w[len].bid = ++bid;
    return bid;
}

/* bwt_match_exact_alt: backward extension of (k, l) by q[len-1] .. q[0] */
static int match_exact_alt(ws_t *s, const oindex_t *x, int len, const uint8_t *q, uint64_t *k0, uint64_t *l0)
{
    uint64_t k = *k0, l = *l0;
    for (int i = len - 1; i >= 0; --i) {
        if (q[i] > 3) return 0;
        extend1(s, x, q[i], &k, &l);
        if (k > l) return 0;
    }
    *k0 = k; *l0 = l;
    return (int)(l - k + 1);
}

static void shadow(int x, uint64_t max, int last_diff_pos, width_t *w)
{
    int j = 0;
    uint64_t xx = (uint64_t)(int64_t)x;
    for (int i = 0; i < last_diff_pos; ++i) {
        if (w[i].w > xx) w[i].w -= xx;
        else if (w[i].w == xx) { w[i].bid = 1; w[i].w = max - (uint64_t)(++j); }
    }
}

static int ilog2_floor(uint32_t v)
{
    int c = 0;
    while (v >>= 1) ++c;
    return c;
}

#define PUSH(...) do { int r_ = push(s, o, __VA_ARGS__); if (r_) return r_; } while (0)

/* bwt_match_gap for one read; q is the reversed+complemented read. Returns n_aln or ERR_SCORE. */
static int match_gap(ws_t *s, const oindex_t *x, int len, const uint8_t *q, width_t *w, width_t *sw, const ropt_t *o)
{
    int best_score = score_of(o->max_diff + 1, o->max_gapo + 1, o->max_gape + 1, o);
    int max_diff = o->max_diff, best_cnt = 0;
    int gape = (o->mode & MODE_GAPE) != 0;
    s->n_rec = 0;
    int n_amb = 0;
    for (int j = 0; j < len; ++j) n_amb += q[j] > 3;
    if (n_amb > max_diff) return 0;

    for (int b = 0; b < s->nb; ++b) s->b[b].n = 0;
    s->best = s->nb; s->n_entries = 0; s->peak = 0; s->pops = 0; s->trace = FNV_OFFSET;
    PUSH(len, 0, x->seq_len, 0, 0, 0, 0, 0, ST_M, 0);

    while (s->n_entries) {
        entry_t e;
        if (s->n_entries > o->max_entries) break;
        pop(s, &e);
        uint64_t k = e.k, l = e.l;
        int i = (int)(e.info & 0xffff);
        if (!(o->mode & MODE_NONSTOP) && (e.info >> 21) > (uint32_t)(best_score + o->s_mm)) break;

        int diffs = e.n_mm + e.n_gapo + (gape ? e.n_gape : 0);
        int m = max_diff - diffs;
        if (m < 0) continue;
        int m_seed = sw ? o->max_seed_diff - diffs : 0;
        if (i > 0 && m < w[i - 1].bid) continue;

        int hit = 0;
        if (i == 0) hit = 1;
        else if (m == 0 && (e.state == ST_M || gape || e.n_gape == o->max_gape)) {
            if (match_exact_alt(s, x, i, q, &k, &l)) hit = 1;
            else continue;
        }
        if (hit) {
            int sc = score_of(e.n_mm, e.n_gapo, e.n_gape, o);
            if (s->n_rec == 0) {
                best_score = sc;
                int best_diff = diffs;
                if (!(o->mode & MODE_NONSTOP)) max_diff = best_diff + 1 > o->max_diff ? o->max_diff : best_diff + 1;
            }
            if (sc == best_score) best_cnt = (int)(uint32_t)((uint64_t)(int64_t)best_cnt + (l - k + 1));
            else if (best_cnt > o->max_top2) break;
            int add = 1;
            if (e.n_gapo)
                for (long j = 0; j < s->n_rec; ++j)
                    if (s->rec[j].k == k && s->rec[j].l == l) { add = 0; break; }
            if (add) {
                shadow((int)(l - k + 1), x->seq_len, e.last_diff_pos, w);
                if (s->n_rec == s->m_rec) {
                    s->m_rec = s->m_rec ? 2 * s->m_rec : 64;
                    s->rec = (rec_t*)realloc(s->rec, (size_t)s->m_rec * sizeof(rec_t));
                }
                rec_t *r = &s->rec[s->n_rec++];
                r->packed = (uint64_t)(e.n_mm & 0xff) | (uint64_t)(e.n_gapo & 0xff) << 8
                          | (uint64_t)(e.n_gape & 0xff) << 16 | (uint64_t)(sc & 0xfffff) << 24
                          | (uint64_t)(e.n_ins & 0x3ff) << 44 | (uint64_t)(e.n_del & 0x3ff) << 54;
                r->k = k; r->l = l;
            }
            continue;
        }

        --i;
        uint64_t ck[4], cl[4];
        s->f128 += fetches(x, k - 1, l, 7);
        s->f64 += fetches(x, k - 1, l, 6);
        s->f80 += fetches_div(x, k - 1, l, 80);
        for (int c = 0; c < 4; ++c) { ck[c] = occ(x, k - 1, c); cl[c] = occ(x, l, c); }
        uint64_t width_now = l - k + 1;
        int allow_diff = 1, allow_M = 1;
        if (i > 0) {
            if (w[i - 1].bid > m - 1) allow_diff = 0;
            else if (w[i - 1].bid == m - 1 && w[i].bid == m - 1 && w[i - 1].w == w[i].w) allow_M = 0;
            int ii = i - (len - o->seed_len);
            if (sw && ii > 0) {
                if (sw[ii - 1].bid > m_seed - 1) allow_diff = 0;
                else if (sw[ii - 1].bid == m_seed - 1 && sw[ii].bid == m_seed - 1 && sw[ii - 1].w == sw[ii].w) allow_M = 0;
            }
        }
        int gaps = e.n_gapo + e.n_gape;
        int end_gap = (o->mode & MODE_LOGGAP) ? ilog2_floor((uint32_t)gaps) / 2 + 1 : gaps;
        if (allow_diff && i >= o->indel_end_skip + end_gap && len - i >= o->indel_end_skip + end_gap) {
            if (e.state == ST_M) {
                if (e.n_gapo < o->max_gapo) {
                    PUSH(i, k, l, e.n_mm, e.n_gapo + 1, e.n_gape, e.n_ins + 1, e.n_del, ST_I, 1);
                    for (int c = 0; c < 4; ++c) {
                        uint64_t kk = x->L2[c] + ck[c] + 1, ll = x->L2[c] + cl[c];
                        if (kk <= ll) PUSH(i + 1, kk, ll, e.n_mm, e.n_gapo + 1, e.n_gape, e.n_ins, e.n_del + 1, ST_D, 1);
                    }
                }
            } else if (e.state == ST_I) {
                if (e.n_gape < o->max_gape)
                    PUSH(i, k, l, e.n_mm, e.n_gapo, e.n_gape + 1, e.n_ins + 1, e.n_del, ST_I, 1);
            } else if (e.state == ST_D) {
                if (e.n_gape < o->max_gape && (gaps < max_diff || width_now < (uint64_t)(int64_t)o->max_del_occ)) {
                    for (int c = 0; c < 4; ++c) {
                        uint64_t kk = x->L2[c] + ck[c] + 1, ll = x->L2[c] + cl[c];
                        if (kk <= ll) PUSH(i + 1, kk, ll, e.n_mm, e.n_gapo, e.n_gape + 1, e.n_ins, e.n_del + 1, ST_D, 1);
                    }
                }
            }
        }
        int base = q[i];
        if (allow_diff && allow_M) {
            for (int j = 1; j <= 4; ++j) {
                int c = (base + j) & 3;
                int mm = j != 4 || base > 3;
                uint64_t kk = x->L2[c] + ck[c] + 1, ll = x->L2[c] + cl[c];
                if (kk <= ll) PUSH(i, kk, ll, e.n_mm + mm, e.n_gapo, e.n_gape, e.n_ins, e.n_del, ST_M, mm);
            }
        } else if (base < 4) {
            uint64_t kk = x->L2[base] + ck[base] + 1, ll = x->L2[base] + cl[base];
            if (kk <= ll) PUSH(i, kk, ll, e.n_mm, e.n_gapo, e.n_gape, e.n_ins, e.n_del, ST_M, 0);
        }
    }
    return (int)s->n_rec;
}
#undef PUSH

/* ------------------------------------------------------------------------------------------------ */
/* options */

int orc_cal_maxdiff(int l, double err, double thres)
{
    double elambda = exp(-l * err);
    double sum = elambda, y = 1.0;
    int x = 1;
    for (int k = 1; k < 1000; ++k) {
        y *= l * err;
        x = (int)((unsigned)x * (unsigned)k);
        sum += elambda * y / x;
        if (1.0 - sum < thres) return k;
    }
    return 2;
}

/* per-batch options: max_diff from the longest read when -n is a fraction, max_gapo clamped to it;
 * returns n_stacks = score(max_diff+1, max_gapo+1, max_gape+1) */
static int batch_opt(const orc_gap_opt_t *u, int max_len, ropt_t *b)
{
    b->s_mm = u->s_mm; b->s_gapo = u->s_gapo; b->s_gape = u->s_gape; b->mode = u->mode;
    b->indel_end_skip = u->indel_end_skip; b->max_del_occ = u->max_del_occ; b->max_entries = u->max_entries;
    b->max_diff = u->max_diff; b->max_gapo = u->max_gapo; b->max_gape = u->max_gape;
    b->max_seed_diff = u->max_seed_diff; b->seed_len = u->seed_len; b->max_top2 = u->max_top2;
    if (u->fnr > 0.0) b->max_diff = orc_cal_maxdiff(max_len, 0.02, u->fnr);
    if (b->max_diff < b->max_gapo) b->max_gapo = b->max_diff;
    return score_of(b->max_diff + 1, b->max_gapo + 1, b->max_gape + 1, b);
}

/* ------------------------------------------------------------------------------------------------ */
/* search over many reads */

typedef struct {
    int n;
    int32_t *n_aln, *peak, *n_stacks, *max_diff;
    uint64_t *pops, *trace, *f128, *f64, *f80;
    rec_t **rec;
} ores_t;

typedef struct {
    const oindex_t *x;
    const orc_gap_opt_t *u;
    const uint8_t *query;
    const int64_t *off;
    const int32_t *len, *batch;
    const ropt_t *bopt;
    const int *bstacks;
    int n, next;
    pthread_mutex_t mu;
    ores_t *res;
} ojob_t;

static void *worker(void *arg)
{
    ojob_t *J = (ojob_t*)arg;
    ws_t s;
    memset(&s, 0, sizeof(s));
    int nb_cap = 0;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        int r = J->next;
        J->next += 64;
        pthread_mutex_unlock(&J->mu);
        if (r >= J->n) break;
        int r_end = r + 64 < J->n ? r + 64 : J->n;
        for (; r < r_end; ++r) {
            int b = J->batch[r], len = J->len[r];
            const uint8_t *q = J->query + J->off[r];
            ropt_t o = J->bopt[b];
            o.max_diff = J->u->fnr > 0.0 ? orc_cal_maxdiff(len, 0.02, J->u->fnr) : J->bopt[b].max_diff;
            o.seed_len = J->u->seed_len < len ? J->u->seed_len : 0x7fffffff;
            int ns = J->bstacks[b];
            if (ns > nb_cap) {
                s.b = (bucket_t*)realloc(s.b, (size_t)ns * sizeof(bucket_t));
                memset(s.b + nb_cap, 0, (size_t)(ns - nb_cap) * sizeof(bucket_t));
                nb_cap = ns;
            }
            s.nb = ns;
            if (s.w_cap < len + 1) { s.w_cap = len + 1; s.w = (width_t*)realloc(s.w, (size_t)s.w_cap * sizeof(width_t)); }
            int use_seed = len > J->u->seed_len;
            if (use_seed && s.sw_cap < J->u->seed_len + 1) {
                s.sw_cap = J->u->seed_len + 1;
                s.sw = (width_t*)realloc(s.sw, (size_t)s.sw_cap * sizeof(width_t));
            }
            s.f128 = s.f64 = s.f80 = 0;
            cal_width(&s, J->x, len, q, s.w);
            if (use_seed) cal_width(&s, J->x, J->u->seed_len, q + (len - J->u->seed_len), s.sw);
            s.pops = 0; s.trace = FNV_OFFSET; s.peak = 0;
            int ret = match_gap(&s, J->x, len, q, s.w, use_seed ? s.sw : NULL, &o);
            ores_t *R = J->res;
            R->n_aln[r] = ret; R->pops[r] = s.pops; R->trace[r] = s.trace; R->peak[r] = (int32_t)s.peak;
            R->f128[r] = s.f128; R->f64[r] = s.f64; R->f80[r] = s.f80; R->n_stacks[r] = ns; R->max_diff[r] = o.max_diff;
            if (ret > 0) {
                R->rec[r] = (rec_t*)malloc((size_t)ret * sizeof(rec_t));
                memcpy(R->rec[r], s.rec, (size_t)ret * sizeof(rec_t));
            }
        }
    }
    for (int b = 0; b < nb_cap; ++b) free(s.b[b].v);
    free(s.b); free(s.rec); free(s.w); free(s.sw);
    return NULL;
}

void *orc_aln_bmax(const void *index, const orc_gap_opt_t *u, const uint8_t *query, const int64_t *off,
                   const int32_t *len, const int32_t *batch, int n, int n_threads, const int32_t *bmax, int n_bmax)
{
    const oindex_t *x = (const oindex_t*)index;
    int nbatch = 0;
    for (int r = 0; r < n; ++r) if (batch[r] + 1 > nbatch) nbatch = batch[r] + 1;
    if (bmax && n_bmax > nbatch) nbatch = n_bmax;
    int *maxlen = (int*)calloc(nbatch > 0 ? nbatch : 1, sizeof(int));
    for (int r = 0; r < n; ++r) if (len[r] > maxlen[batch[r]]) maxlen[batch[r]] = len[r];
    if (bmax) for (int b = 0; b < n_bmax; ++b) if (bmax[b] > maxlen[b]) maxlen[b] = bmax[b];
    ropt_t *bopt = (ropt_t*)calloc(nbatch > 0 ? nbatch : 1, sizeof(ropt_t));
    int *bstacks = (int*)calloc(nbatch > 0 ? nbatch : 1, sizeof(int));
    for (int b = 0; b < nbatch; ++b) bstacks[b] = batch_opt(u, maxlen[b], &bopt[b]);
    ores_t *R = (ores_t*)calloc(1, sizeof(ores_t));
    size_t nn = n > 0 ? (size_t)n : 1;
    R->n = n;
    R->n_aln = (int32_t*)calloc(nn, 4); R->peak = (int32_t*)calloc(nn, 4);
    R->n_stacks = (int32_t*)calloc(nn, 4); R->max_diff = (int32_t*)calloc(nn, 4);
    R->pops = (uint64_t*)calloc(nn, 8); R->trace = (uint64_t*)calloc(nn, 8);
    R->f128 = (uint64_t*)calloc(nn, 8); R->f64 = (uint64_t*)calloc(nn, 8); R->f80 = (uint64_t*)calloc(nn, 8);
    R->rec = (rec_t**)calloc(nn, sizeof(rec_t*));
    ojob_t J;
    memset(&J, 0, sizeof(J));
    J.x = x; J.u = u; J.query = query; J.off = off; J.len = len; J.batch = batch;
    J.bopt = bopt; J.bstacks = bstacks; J.n = n; J.res = R;
    pthread_mutex_init(&J.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    pthread_t *tid = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
    for (int t = 0; t < n_threads; ++t) pthread_create(&tid[t], NULL, worker, &J);
    for (int t = 0; t < n_threads; ++t) pthread_join(tid[t], NULL);
    free(tid); free(maxlen); free(bopt); free(bstacks);
    return R;
}

void *orc_aln(const void *index, const orc_gap_opt_t *u, const uint8_t *query, const int64_t *off,
              const int32_t *len, const int32_t *batch, int n, int n_threads)
{
    return orc_aln_bmax(index, u, query, off, len, batch, n, n_threads, NULL, 0);
}

int64_t orc_result_total(const void *p)
{
    const ores_t *R = (const ores_t*)p;
    int64_t t = 0;
    for (int r = 0; r < R->n; ++r) if (R->n_aln[r] > 0) t += R->n_aln[r];
    return t;
}

int orc_result_dump(const void *p, int32_t *n_aln, uint64_t *pops, uint64_t *trace, int32_t *peak,
                    uint64_t *f128, uint64_t *f64, int32_t *n_stacks, int32_t *max_diff,
                    int64_t *rec_off, void *records)
{
    const ores_t *R = (const ores_t*)p;
    int64_t t = 0;
    for (int r = 0; r < R->n; ++r) {
        n_aln[r] = R->n_aln[r]; pops[r] = R->pops[r]; trace[r] = R->trace[r]; peak[r] = R->peak[r];
        f128[r] = R->f128[r]; f64[r] = R->f64[r]; n_stacks[r] = R->n_stacks[r]; max_diff[r] = R->max_diff[r];
        rec_off[r] = t;
        if (R->n_aln[r] > 0) {
            memcpy((char*)records + t * 24, R->rec[r], (size_t)R->n_aln[r] * 24);
            t += R->n_aln[r];
        }
    }
    rec_off[R->n] = t;
    return 0;
}

/* "SAI\1", the 64-byte option block, then per read int32 n_aln and n_aln 24-byte records; a read whose
 * search failed is written with 0 records (galn.cu:1250-1263) and the call returns 4 */
/* per-read block fetches under the 80-symbol layout */
int orc_result_fetch80(const void *res, uint64_t *fetch80)
{
    const ores_t *R = (const ores_t *)res;
    for (int r = 0; r < R->n; ++r) fetch80[r] = R->f80[r];
    return 0;
}

int orc_result_write_sai(const void *p, const orc_gap_opt_t *opt, const char *path)
{
    const ores_t *R = (const ores_t*)p;
    FILE *fp = fopen(path, "wb");
    if (!fp) return 5;
    int err = 0;
    fwrite("SAI\1", 1, 4, fp);
    fwrite(opt, sizeof(*opt), 1, fp);
    for (int r = 0; r < R->n; ++r) {
        int32_t na = R->n_aln[r];
        if (na < 0) { err = 4; na = 0; }
        fwrite(&na, 4, 1, fp);
        if (na > 0) fwrite(R->rec[r], 24, (size_t)na, fp);
    }
    if (fclose(fp) != 0) return 5;
    return err;
}

void orc_result_free(void *p)
{
    ores_t *R = (ores_t*)p;
    if (!R) return;
    for (int r = 0; r < R->n; ++r) free(R->rec[r]);
    free(R->rec); free(R->n_aln); free(R->peak); free(R->n_stacks); free(R->max_diff);
    free(R->pops); free(R->trace); free(R->f128); free(R->f64); free(R->f80);
    free(R);
}

/* ------------------------------------------------------------------------------------------------ */
/* FASTQ/FASTA reading with kseq's record rules, and bwa_read_seq's batch rule */

typedef struct { const unsigned char *p; size_t n, i; } instr_t;

static inline int getc_(instr_t *s) { return s->i < s->n ? s->p[s->i++] : -1; }

typedef struct { char *s; size_t l, m; } str_t;

static void str_put(str_t *t, const unsigned char *p, size_t n)
{
    if (t->l + n + 1 > t->m) {
        t->m = (t->l + n + 1) * 2;
        t->s = (char*)realloc(t->s, t->m);
    }
    memcpy(t->s + t->l, p, n);
    t->l += n;
    t->s[t->l] = 0;
}

/* append up to (not including) the next '\n', which is consumed; a trailing '\r' of the whole string is
 * dropped when it is longer than one character. Returns -1 when nothing was left to read. */
static long read_line(instr_t *s, str_t *t)
{
    if (s->i >= s->n) return -1;
    const unsigned char *nl = (const unsigned char*)memchr(s->p + s->i, '\n', s->n - s->i);
    size_t e = nl ? (size_t)(nl - s->p) : s->n;
    str_put(t, s->p + s->i, e - s->i);
    s->i = nl ? e + 1 : e;
    if (t->l > 1 && t->s[t->l - 1] == '\r') t->s[--t->l] = 0;
    return (long)t->l;
}

typedef struct { str_t name, seq, qual; int last; } rec_reader_t;

/* one record: >= 0 sequence length, -1 end of input, -2 malformed (quality missing or of another length) */
static int read_record(instr_t *s, rec_reader_t *R)
{
    int c;
    if (R->last == 0) {
        while ((c = getc_(s)) != -1 && c != '>' && c != '@') ;
        if (c == -1) return -1;
        R->last = c;
    }
    R->seq.l = R->qual.l = R->name.l = 0;
    if (s->i >= s->n) return -1;
    /* name: up to the first white space; the rest of the line is a comment */
    size_t st = s->i;
    while (s->i < s->n && !isspace(s->p[s->i])) ++s->i;
    str_put(&R->name, s->p + st, s->i - st);
    int delim = s->i < s->n ? s->p[s->i++] : 0;
    if (delim != '\n') { str_t tmp = {0, 0, 0}; read_line(s, &tmp); free(tmp.s); }
    while ((c = getc_(s)) != -1 && c != '>' && c != '+' && c != '@') {
        if (c == '\n') continue;
        unsigned char ch = (unsigned char)c;
        str_put(&R->seq, &ch, 1);
        read_line(s, &R->seq);
    }
    if (c == '>' || c == '@') R->last = c;
    if (R->seq.s == NULL) str_put(&R->seq, (const unsigned char*)"", 0);
    if (c != '+') return (int)R->seq.l;
    while ((c = getc_(s)) != -1 && c != '\n') ;
    if (c == -1) return -2;
    while (read_line(s, &R->qual) >= 0 && R->qual.l < R->seq.l) ;
    R->last = 0;
    if (R->seq.l != R->qual.l) return -2;
    return (int)R->seq.l;
}

typedef struct {
    int n;
    uint8_t *query; size_t q_len, q_cap;
    int64_t *off; int32_t *len, *batch; size_t cap;
} oreads_t;

static const unsigned char *nt4_table(void)
{
    static unsigned char t[256];
    static int init = 0;
    if (!init) {
        memset(t, 4, sizeof(t));
        t['A'] = t['a'] = 0; t['C'] = t['c'] = 1; t['G'] = t['g'] = 2; t['T'] = t['t'] = 3; t['-'] = 5;
        init = 1;
    }
    return t;
}

void *orc_reads_load(const char *path, int *n_reads, int64_t *total, int *err)
{
    gzFile fp = gzopen(path, "rb");
    if (!fp) { *err = -1; return NULL; }
    size_t cap = 1 << 20, n = 0;
    unsigned char *buf = (unsigned char*)malloc(cap);
    for (;;) {
        if (cap - n < (1 << 16)) { cap *= 2; buf = (unsigned char*)realloc(buf, cap); }
        int r = gzread(fp, buf + n, (unsigned)(cap - n));
        if (r < 0) { gzclose(fp); free(buf); *err = -3; return NULL; }
        if (r == 0) break;
        n += (size_t)r;
    }
    gzclose(fp);
    const unsigned char *nt4 = nt4_table();
    instr_t s = { buf, n, 0 };
    rec_reader_t R;
    memset(&R, 0, sizeof(R));
    oreads_t *o = (oreads_t*)calloc(1, sizeof(oreads_t));
    int batch = 0, in_batch = 0;
    for (;;) {
        int l = read_record(&s, &R);
        if (l < 0) {
            if (in_batch == 0 || l == -1) break;
            ++batch; in_batch = 0;                 /* a malformed record ends the batch */
            continue;
        }
        if (R.seq.l == 0) continue;
        if ((size_t)o->n + 1 >= o->cap) {
            o->cap = o->cap ? 2 * o->cap : 1024;
            o->off = (int64_t*)realloc(o->off, (o->cap + 1) * 8);
            o->len = (int32_t*)realloc(o->len, o->cap * 4);
            o->batch = (int32_t*)realloc(o->batch, o->cap * 4);
        }
        if (o->q_len + R.seq.l > o->q_cap) {
            o->q_cap = (o->q_len + R.seq.l) * 2 + 1024;
            o->query = (uint8_t*)realloc(o->query, o->q_cap);
        }
        int L = (int)R.seq.l;
        uint8_t *q = o->query + o->q_len;
        for (int j = 0; j < L; ++j) {                /* reverse, then complement (ambiguous -> 4) */
            unsigned b = nt4[(unsigned char)R.seq.s[L - 1 - j]];
            q[j] = b > 3 ? 4 : (uint8_t)(3 - b);
        }
        o->off[o->n] = (int64_t)o->q_len;
        o->len[o->n] = L;
        o->batch[o->n] = batch;
        o->q_len += (size_t)L;
        ++o->n;
        if (++in_batch == BATCH_READS) { ++batch; in_batch = 0; }
    }
    if (o->off == NULL) o->off = (int64_t*)calloc(1, 8);
    o->off[o->n] = (int64_t)o->q_len;
    free(R.name.s); free(R.seq.s); free(R.qual.s);
    free(buf);
    *n_reads = o->n;
    *total = (int64_t)o->q_len;
    *err = 0;
    return o;
}

int orc_reads_get(const void *p, uint8_t *query, int64_t *off, int32_t *len, int32_t *batch)
{
    const oreads_t *o = (const oreads_t*)p;
    if (o->q_len) memcpy(query, o->query, o->q_len);
    memcpy(off, o->off, (size_t)(o->n + 1) * 8);
    if (o->n) { memcpy(len, o->len, (size_t)o->n * 4); memcpy(batch, o->batch, (size_t)o->n * 4); }
    return 0;
}

void orc_reads_free(void *p)
{
    oreads_t *o = (oreads_t*)p;
    if (!o) return;
    free(o->query); free(o->off); free(o->len); free(o->batch); free(o);
}

/* ---- index files (`bwa index` 0.7.19 .bwt and .sa; the reference's src/index/idxcommon.c:72-153) ----
 * Test sizes only: the suffix array of T$ by a comparison sort over the suffixes (memcmp on one code per
 * byte; a suffix that is a prefix of another sorts first, $ being the smallest symbol). */
static const uint8_t *orc_sa_text;
static uint64_t orc_sa_n;

static int orc_suffix_cmp(const void *a, const void *b)
{
    const uint64_t i = *(const uint64_t*)a, j = *(const uint64_t*)b;
    const uint64_t li = orc_sa_n - i, lj = orc_sa_n - j, l = li < lj ? li : lj;
    const int c = memcmp(orc_sa_text + i, orc_sa_text + j, l);
    if (c) return c;
    return li < lj ? -1 : li > lj ? 1 : 0;
}

/* sa[0..n]: row 0 is the $ suffix (position n) */
int orc_suffix_array(const uint8_t *T, uint64_t n, uint64_t *sa)
{
    orc_sa_text = T;
    orc_sa_n = n;
    sa[0] = n;
    for (uint64_t i = 0; i < n; ++i) sa[i + 1] = i;
    qsort(sa + 1, n, sizeof(uint64_t), orc_suffix_cmp);
    return 0;
}

/* <prefix>.bwt and <prefix>.sa for the forward sequence F[0..l_pac) (codes 0..3): the text is
 * T = F . revcomp(F); its BWT drops the $ of the row of suffix 0 (`primary`); the .bwt body holds, every 128
 * symbols, the four 64-bit counts of the symbols before, and 16 symbols per 32-bit word, the first in the
 * top two bits, then the four totals (idxcommon.c:72-112); the .sa holds every 32nd row from row 32 on
 * (idxcommon.c:137-153). Both files start with primary and L2[1..4]; the .sa adds 32 and n. */
int orc_index_files(const uint8_t *F, uint64_t l_pac, const char *prefix)
{
    const uint64_t n = 2 * l_pac;
    uint8_t *T = (uint8_t*)malloc(n ? n : 1);
    uint64_t *sa = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
    uint8_t *L = (uint8_t*)malloc(n ? n : 1);
    if (!T || !sa || !L) { free(T); free(sa); free(L); return -1; }
    for (uint64_t i = 0; i < l_pac; ++i) { T[i] = F[i]; T[n - 1 - i] = (uint8_t)(3 - F[i]); }
    orc_suffix_array(T, n, sa);
    uint64_t primary = 0, m = 0, L2[5] = {0, 0, 0, 0, 0}, cnt[4] = {0, 0, 0, 0};
    for (uint64_t r = 0; r <= n; ++r) {
        if (sa[r] == 0) { primary = r; continue; }
        L[m++] = T[sa[r] - 1];
    }
    for (uint64_t i = 0; i < n; ++i) ++cnt[T[i]];
    for (int c = 0; c < 4; ++c) L2[c + 1] = L2[c] + cnt[c];
    const uint64_t nw = (n + 15) / 16, nb = (n + 127) / 128;
    uint32_t *body = (uint32_t*)calloc(nw + 8 * (nb + 1), sizeof(uint32_t));
    uint64_t run[4] = {0, 0, 0, 0}, k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if ((i & 127) == 0) { memcpy(body + k, run, sizeof run); k += 8; }
        if ((i & 15) == 0) {
            uint32_t w = 0;
            for (uint64_t t = 0; t < 16 && i + t < n; ++t) w |= (uint32_t)L[i + t] << (30 - 2 * t);
            body[k++] = w;
        }
        ++run[L[i]];
    }
    memcpy(body + k, run, sizeof run);
    k += 8;
    char path[4096];
    int rc = 0;
    snprintf(path, sizeof path, "%s.bwt", prefix);
    FILE *f = fopen(path, "wb");
    if (!f) rc = -1;
    else {
        fwrite(&primary, 8, 1, f);
        fwrite(L2 + 1, 8, 4, f);
        fwrite(body, 4, k, f);
        fclose(f);
    }
    snprintf(path, sizeof path, "%s.sa", prefix);
    f = rc ? NULL : fopen(path, "wb");
    if (!f) rc = -1;
    else {
        const uint64_t head[3] = {primary, 32, n};
        fwrite(head, 8, 1, f);
        fwrite(L2 + 1, 8, 4, f);
        fwrite(head + 1, 8, 2, f);
        for (uint64_t r = 32; r <= n; r += 32) fwrite(sa + r, 8, 1, f);
        fclose(f);
    }
    free(T); free(sa); free(L); free(body);
    return rc;
}
