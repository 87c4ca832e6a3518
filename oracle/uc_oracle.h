/*
 * uc_oracle.h — CPU restatement of the reference's unitig-compaction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the parity tests,
 * the smoke check and the CPU-baseline leg of bench.py compare the CUDA path
 * against.  No product code path may link, load or call it.
 *
 * k-mer words use the reference layout (driver.cpp:227-249): comp = ceil(k/16)
 * uint32 words per k-mer, 16 chars per word, char x at bits 2*(x%16) of word
 * x/16, A=0 C=1 G=2 T=3, every other byte -> 0, zero padding.
 */
#ifndef UC_ORACLE_H
#define UC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NONE 0xFFFFFFFFu

/* 0 ok, 1 malformed input (see orc_parse), 2 out of memory */
enum { ORC_OK = 0, ORC_EINPUT = 1, ORC_ENOMEM = 2 };

/* Parse the reference's k-mer text (count header line, then one k-mer per
 * line; only the first k chars of a line are used) and pack it.
 * words may be NULL to only count.  *n_out receives the k-mer count. */
int orc_parse(const char *text, size_t bytes, int k, uint32_t *words,
              int64_t cap_n, int64_t *n_out);

/* Priority of an l-mer (big-endian 2-bit id, first char in the top bits):
 * a seeded bijection of [0, 4^l). */
uint32_t orc_lmer_priority(uint32_t lmer, int l, uint64_t seed);

/* Prefix (l1) and suffix (l2) L-minimizers of every k-mer
 * (lmin_buckets.h:67-94).  table (4^l entries) overrides the seeded priority
 * when not NULL. */
void orc_lmin(const uint32_t *words, int64_t n, int k, int l,
              const uint32_t *table, uint64_t seed, uint32_t *l1, uint32_t *l2);

/* Kept-edge functional graph (assembler.h:113-214 on the whole input):
 * succ[u] = v iff v is the only k-mer whose (k-1)-prefix equals u's
 * (k-1)-suffix and u is the only k-mer whose suffix equals v's prefix.
 * pred is the inverse.  Returns ORC_OK or ORC_ENOMEM. */
int orc_edges(const uint32_t *words, int64_t n, int k, uint32_t *succ,
              uint32_t *pred);

/* Path decomposition: head[v] = first vertex of v's unitig, rank[v] = its
 * position.  A cycle starts at its numerically smallest packed k-mer.
 * Returns the number of cycles. */
int64_t orc_contract(const uint32_t *words, int64_t n, int k,
                     const uint32_t *succ, const uint32_t *pred,
                     uint32_t *head, uint32_t *rank);

/* Spell every unitig (compact.h:161-210): first k-mer in full, then the last
 * char of each later k-mer, then '\n'.  Lines in increasing head id.  out may
 * be NULL to size.  Returns bytes written (or needed). */
int64_t orc_emit(const uint32_t *words, int64_t n, int k, const uint32_t *succ,
                 const uint32_t *head, const uint32_t *rank, char *out,
                 int64_t cap);

/* Whole path: text in, unitig lines out.  *out is malloc'd (free with
 * orc_free).  Returns ORC_OK / ORC_EINPUT / ORC_ENOMEM. */
int orc_compact(const char *text, size_t bytes, int k, char **out,
                int64_t *out_len, int64_t *n_kmers, int64_t *n_cycles);

/* Lines of in[0, len) (each '\n'-terminated) copied to out in byte order;
 * *n_lines receives their count.  Used to digest outputs too large to sort
 * as Python objects.  Returns ORC_OK / ORC_EINPUT (a line without its
 * newline) / ORC_ENOMEM. */
int orc_sort_lines(const char *in, int64_t len, char *out, int64_t *n_lines);

void orc_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
