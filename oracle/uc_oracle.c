/*
 * uc_oracle.c — CPU restatement of the reference's unitig-compaction path
 * (euphoricpoptarts/UnitigCoarsening).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Each function restates the behaviour of the reference code it cites.  The
 * reference splits the input into 64 minimizer buckets with duplicated
 * boundary k-mers and stitches the cross-bucket paths afterwards
 * (driver.cpp:479-639); that bookkeeping does not change which edges are kept
 * or which lines are written (every edge u->v is found in the bucket of v's
 * prefix minimizer, which equals u's suffix minimizer, and both degrees are
 * counted there in full), so the restatement applies the edge rule to the
 * whole input at once and walks the resulting paths.
 */
#include "uc_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- packing */

/* char_map of compact_kmers (driver.cpp:228-232): a zeroed 256-entry table
 * with A,C,G,T set, so every other byte packs as A. */
static inline uint32_t base_code(unsigned char c) {
    switch (c) {
    case 'C': return 1u;
    case 'G': return 2u;
    case 'T': return 3u;
    default: return 0u;
    }
}

static inline int comp_words(int k) { return (k + 15) / 16; }

/* Header and line rules of load_kmers (driver.cpp:296-328): the first line
 * holds the count (sscanf "%u"), every later line contributes its first k
 * chars.  The reference hangs when the count disagrees with the number of
 * lines (its chunk loop never reaches total_read == n) and copies past the
 * newline of a line shorter than k; both are reported as ORC_EINPUT here. */
int orc_parse(const char *text, size_t bytes, int k, uint32_t *words,
              int64_t cap_n, int64_t *n_out) {
    if (k < 2 || k > 63) return ORC_EINPUT;
    size_t p = 0;
    while (p < bytes && (text[p] == ' ' || text[p] == '\t' || text[p] == '\r'))
        p++;
    if (p >= bytes || text[p] < '0' || text[p] > '9') return ORC_EINPUT;
    uint64_t hdr = 0;
    while (p < bytes && text[p] >= '0' && text[p] <= '9') {
        hdr = hdr * 10u + (uint64_t)(text[p] - '0');
        if (hdr > 0xFFFFFFFFull) return ORC_EINPUT;
        p++;
    }
    while (p < bytes && text[p] != '\n') p++;
    if (p < bytes) p++; /* past the header's newline */
    const int comp = comp_words(k);
    int64_t n = 0;
    while (p < bytes) {
        size_t e = p;
        while (e < bytes && text[e] != '\n') e++;
        size_t len = e - p;
        if (len == 0) {
            /* a blank line is accepted only at the end of the text */
            size_t q = e;
            while (q < bytes && (text[q] == '\n' || text[q] == '\r')) q++;
            if (q != bytes) return ORC_EINPUT;
            break;
        }
        if (len < (size_t)k) return ORC_EINPUT;
        if (words) {
            if (n >= cap_n) return ORC_EINPUT;
            uint32_t *w = words + (size_t)n * comp;
            for (int i = 0; i < comp; i++) w[i] = 0;
            for (int x = 0; x < k; x++)
                w[x / 16] |= base_code((unsigned char)text[p + x]) << (2 * (x % 16));
        }
        n++;
        p = (e < bytes) ? e + 1 : e;
    }
    if ((uint64_t)n != hdr) return ORC_EINPUT;
    *n_out = n;
    return ORC_OK;
}

/* ------------------------------------------------------------- minimizers */

/* Seeded bijection of [0, 4^l) standing in for the reference's random l-mer
 * permutation (generate_permutation, driver.cpp:356-402): an odd multiplier
 * and an addend drawn from the seed, modulo 4^l. */
uint32_t orc_lmer_priority(uint32_t x, int l, uint64_t seed) {
    const uint32_t b = 2u * (uint32_t)l;
    const uint32_t mask = (b >= 32u) ? 0xFFFFFFFFu : ((1u << b) - 1u);
    const uint32_t mult = (0x9E3779B1u ^ ((uint32_t)seed << 1)) | 1u;
    return (x * mult + (uint32_t)(seed >> 32)) & mask;
}

static inline uint32_t get_char(const uint32_t *w, int x) {
    return (w[x / 16] >> (2 * (x % 16))) & 3u;
}

/* get_double_lmin (lmin_buckets.h:67-94): the l-mer id is built big-endian
 * (lmer_id <<= 2; lmer_id ^= c); l1 is the smallest priority among l-mers
 * inside chars [0, k-1), l2 among l-mers inside chars [1, k). */
void orc_lmin(const uint32_t *words, int64_t n, int k, int l,
              const uint32_t *table, uint64_t seed, uint32_t *l1, uint32_t *l2) {
    const int comp = comp_words(k);
    const uint32_t lmask = (2 * l >= 32) ? 0xFFFFFFFFu : ((1u << (2 * l)) - 1u);
    for (int64_t v = 0; v < n; v++) {
        const uint32_t *w = words + (size_t)v * comp;
        uint32_t id = 0, a = ORC_NONE, b = ORC_NONE;
        for (int i = 0; i < k; i++) {
            id = ((id << 2) ^ get_char(w, i)) & lmask;
            if (i + 1 >= l) {
                uint32_t pr = table ? table[id] : orc_lmer_priority(id, l, seed);
                if (i + 1 < k && a > pr) a = pr;
                if (i + 1 >= l + 1 && b > pr) b = pr;
            }
        }
        l1[v] = a;
        l2[v] = b;
    }
}

/* ------------------------------------------------------------------ edges */

typedef struct {
    uint64_t lo, hi;
} k128;

static inline k128 load_key(const uint32_t *w, int comp) {
    uint32_t t[4] = {0, 0, 0, 0};
    for (int i = 0; i < comp; i++) t[i] = w[i];
    k128 r;
    r.lo = (uint64_t)t[0] | ((uint64_t)t[1] << 32);
    r.hi = (uint64_t)t[2] | ((uint64_t)t[3] << 32);
    return r;
}

/* low 2*(k-1) bits: the (k-1)-prefix (fnv_pref/cmp_pref, assembler.h:8-22,
 * 49-63, whose fixed mask 0x0FFFFFFF keeps exactly these bits when
 * k = 15 mod 16). */
static inline k128 prefix_of(k128 x, int k) {
    const int bits = 2 * (k - 1);
    if (bits >= 128) return x;
    if (bits >= 64) {
        x.hi &= (bits == 64) ? 0 : ((1ull << (bits - 64)) - 1ull);
    } else {
        x.lo &= (1ull << bits) - 1ull;
        x.hi = 0;
    }
    return x;
}

/* chars 1..k-1 shifted down to position 0 (fnv_suf/cmp_suf,
 * assembler.h:26-45, 67-85). */
static inline k128 suffix_of(k128 x, int k) {
    k128 s;
    s.lo = (x.lo >> 2) | (x.hi << 62);
    s.hi = x.hi >> 2;
    return prefix_of(s, k);
}

static inline int k128_eq(k128 a, k128 b) { return a.lo == b.lo && a.hi == b.hi; }
static inline int k128_lt(k128 a, k128 b) {
    return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}

static inline uint64_t mix64(uint64_t z) {
    z ^= z >> 33;
    z *= 0xff51afd7ed558ccdull;
    z ^= z >> 33;
    z *= 0xc4ceb9fe1a85ec53ull;
    z ^= z >> 33;
    return z;
}
static inline uint64_t hash_k128(k128 x) { return mix64(x.lo ^ mix64(x.hi + 0x9e3779b97f4a7c15ull)); }

/* Open-addressing prefix table (init_hashmap/generate_hashmap,
 * assembler.h:113-150): one slot per distinct (k-1)-prefix; a prefix shared
 * by two or more k-mers is "nullified".  Lookup of a k-mer's suffix
 * (find_vtx_from_edge, assembler.h:89-111) yields the unique k-mer with that
 * prefix, "ambiguous" or "none".  Then in-degrees are counted over the unique
 * lookups and u->v is kept iff v was u's unique lookup and v's count is 1
 * (assemble_pruned_graph, assembler.h:180-197). */
int orc_edges(const uint32_t *words, int64_t n, int k, uint32_t *succ,
              uint32_t *pred) {
    const int comp = comp_words(k);
    uint64_t cap = 1;
    while (cap < 2ull * (uint64_t)(n > 0 ? n : 1)) cap <<= 1;
    uint32_t *slot_id = (uint32_t *)malloc(cap * sizeof(uint32_t));
    uint32_t *slot_cnt = (uint32_t *)calloc(cap, sizeof(uint32_t));
    uint32_t *cand = (uint32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(uint32_t));
    uint32_t *indeg = (uint32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(uint32_t));
    if (!slot_id || !slot_cnt || !cand || !indeg) {
        free(slot_id); free(slot_cnt); free(cand); free(indeg);
        return ORC_ENOMEM;
    }
    for (uint64_t i = 0; i < cap; i++) slot_id[i] = ORC_NONE;
    const uint64_t m = cap - 1;
    for (int64_t v = 0; v < n; v++) {
        k128 p = prefix_of(load_key(words + (size_t)v * comp, comp), k);
        uint64_t h = hash_k128(p) & m;
        for (;;) {
            uint32_t s = slot_id[h];
            if (s == ORC_NONE) {
                slot_id[h] = (uint32_t)v;
                slot_cnt[h] = 1;
                break;
            }
            if (k128_eq(prefix_of(load_key(words + (size_t)s * comp, comp), k), p)) {
                slot_cnt[h]++;
                break;
            }
            h = (h + 1) & m;
        }
    }
    for (int64_t u = 0; u < n; u++) {
        k128 s = suffix_of(load_key(words + (size_t)u * comp, comp), k);
        uint64_t h = hash_k128(s) & m;
        cand[u] = ORC_NONE;
        for (;;) {
            uint32_t id = slot_id[h];
            if (id == ORC_NONE) break;
            if (k128_eq(prefix_of(load_key(words + (size_t)id * comp, comp), k), s)) {
                if (slot_cnt[h] == 1) {
                    cand[u] = id;
                    indeg[id]++;
                }
                break;
            }
            h = (h + 1) & m;
        }
    }
    for (int64_t v = 0; v < n; v++) pred[v] = ORC_NONE;
    for (int64_t u = 0; u < n; u++) {
        uint32_t v = cand[u];
        if (v != ORC_NONE && indeg[v] == 1) {
            succ[u] = v;
            pred[v] = (uint32_t)u;
        } else {
            succ[u] = ORC_NONE;
        }
    }
    free(slot_id); free(slot_cnt); free(cand); free(indeg);
    return ORC_OK;
}

/* -------------------------------------------------------------- contract */

/* The reference contracts paths by rounds of heavy-edge coarsening
 * (coarseners.h:437-485, heuristics.h:205-256) and orders each aggregate's
 * members along the path (coarseners.h:182-235); the members of a finished
 * aggregate are one maximal path, first vertex first.  That equals walking
 * each path from its head.  A vertex set with no head is a cycle; the
 * reference leaves its member order unspecified there, the restatement starts
 * it at its smallest packed k-mer. */
int64_t orc_contract(const uint32_t *words, int64_t n, int k,
                     const uint32_t *succ, const uint32_t *pred,
                     uint32_t *head, uint32_t *rank) {
    const int comp = comp_words(k);
    for (int64_t v = 0; v < n; v++) head[v] = ORC_NONE;
    for (int64_t v = 0; v < n; v++) {
        if (pred[v] != ORC_NONE) continue;
        uint32_t r = 0;
        for (uint32_t x = (uint32_t)v; x != ORC_NONE; x = succ[x]) {
            head[x] = (uint32_t)v;
            rank[x] = r++;
        }
    }
    int64_t cycles = 0;
    for (int64_t v = 0; v < n; v++) {
        if (head[v] != ORC_NONE) continue;
        /* v lies on a cycle: find its smallest k-mer, then rank from there */
        uint32_t best = (uint32_t)v;
        k128 bk = load_key(words + (size_t)v * comp, comp);
        for (uint32_t x = succ[v]; x != (uint32_t)v; x = succ[x]) {
            k128 xk = load_key(words + (size_t)x * comp, comp);
            if (k128_lt(xk, bk)) { bk = xk; best = x; }
        }
        uint32_t r = 0, x = best;
        do {
            head[x] = best;
            rank[x] = r++;
            x = succ[x];
        } while (x != best);
        cycles++;
    }
    return cycles;
}

/* ------------------------------------------------------------------- emit */

static const char ACGT[4] = {'A', 'C', 'G', 'T'};

int64_t orc_emit(const uint32_t *words, int64_t n, int k, const uint32_t *succ,
                 const uint32_t *head, const uint32_t *rank, char *out,
                 int64_t cap) {
    (void)rank;
    const int comp = comp_words(k);
    int64_t pos = 0;
    for (int64_t v = 0; v < n; v++) {
        if (head[v] != (uint32_t)v) continue;
        const uint32_t *w = words + (size_t)v * comp;
        if (out && pos + k > cap) return -1;
        for (int x = 0; x < k; x++) {
            if (out) out[pos] = ACGT[get_char(w, x)];
            pos++;
        }
        for (uint32_t x = succ[v]; x != ORC_NONE && x != (uint32_t)v; x = succ[x]) {
            if (out) {
                if (pos + 1 > cap) return -1;
                out[pos] = ACGT[get_char(words + (size_t)x * comp, k - 1)];
            }
            pos++;
        }
        if (out) {
            if (pos + 1 > cap) return -1;
            out[pos] = '\n';
        }
        pos++;
    }
    return pos;
}

int orc_compact(const char *text, size_t bytes, int k, char **out,
                int64_t *out_len, int64_t *n_kmers, int64_t *n_cycles) {
    int64_t n = 0;
    int st = orc_parse(text, bytes, k, NULL, 0, &n);
    if (st) return st;
    const int comp = comp_words(k);
    size_t nn = (size_t)(n > 0 ? n : 1);
    uint32_t *words = (uint32_t *)malloc(nn * comp * sizeof(uint32_t));
    uint32_t *succ = (uint32_t *)malloc(nn * sizeof(uint32_t));
    uint32_t *pred = (uint32_t *)malloc(nn * sizeof(uint32_t));
    uint32_t *head = (uint32_t *)malloc(nn * sizeof(uint32_t));
    uint32_t *rank = (uint32_t *)malloc(nn * sizeof(uint32_t));
    char *buf = NULL;
    int64_t cyc = 0, len = 0;
    st = ORC_ENOMEM;
    if (!words || !succ || !pred || !head || !rank) goto done;
    st = orc_parse(text, bytes, k, words, n, &n);
    if (st) goto done;
    st = orc_edges(words, n, k, succ, pred);
    if (st) goto done;
    cyc = orc_contract(words, n, k, succ, pred, head, rank);
    len = orc_emit(words, n, k, succ, head, rank, NULL, 0);
    buf = (char *)malloc((size_t)(len > 0 ? len : 1));
    st = ORC_ENOMEM;
    if (!buf) goto done;
    orc_emit(words, n, k, succ, head, rank, buf, len);
    st = ORC_OK;
done:
    free(words); free(succ); free(pred); free(head); free(rank);
    if (st == ORC_OK) {
        *out = buf;
        *out_len = len;
        if (n_kmers) *n_kmers = n;
        if (n_cycles) *n_cycles = cyc;
    } else {
        free(buf);
    }
    return st;
}

/* ---------------------------------------------------------- sorted lines */

/* Sort key of a line: its first 16 bytes big-endian (two words), then the
 * rest by memcmp.  Unitig lines start with distinct k-mers, so the words
 * nearly always decide. */
typedef struct {
    uint64_t w0, w1;
    int64_t off, len;
} orc_line;

static const char *g_sort_base;

static inline uint64_t be_word(const char *p, int64_t avail) {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | (uint64_t)(unsigned char)(i < avail ? p[i] : 0);
    return v;
}

static int cmp_line(const void *a, const void *b) {
    const orc_line *x = (const orc_line *)a, *y = (const orc_line *)b;
    if (x->w0 != y->w0) return x->w0 < y->w0 ? -1 : 1;
    if (x->w1 != y->w1) return x->w1 < y->w1 ? -1 : 1;
    int64_t m = x->len < y->len ? x->len : y->len;
    int c = memcmp(g_sort_base + x->off, g_sort_base + y->off, (size_t)m);
    if (c) return c;
    return (x->len > y->len) - (x->len < y->len);
}

int orc_sort_lines(const char *in, int64_t len, char *out, int64_t *n_lines) {
    int64_t n = 0;
    for (int64_t i = 0; i < len; i++) n += in[i] == '\n';
    if (len > 0 && in[len - 1] != '\n') return ORC_EINPUT;
    orc_line *r = (orc_line *)malloc((size_t)(n > 0 ? n : 1) * sizeof(orc_line));
    if (!r) return ORC_ENOMEM;
    int64_t s = 0, j = 0;
    for (int64_t i = 0; i < len; i++) {
        if (in[i] != '\n') continue;
        r[j].off = s;
        r[j].len = i - s;
        r[j].w0 = be_word(in + s, i - s);
        r[j].w1 = be_word(in + s + 8, i - s - 8);
        j++;
        s = i + 1;
    }
    g_sort_base = in;
    qsort(r, (size_t)n, sizeof(orc_line), cmp_line);
    int64_t p = 0;
    for (int64_t t = 0; t < n; t++) {
        memcpy(out + p, in + r[t].off, (size_t)r[t].len);
        p += r[t].len;
        out[p++] = '\n';
    }
    free(r);
    *n_lines = n;
    return ORC_OK;
}

void orc_free(void *p) { free(p); }
