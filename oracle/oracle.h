/*
 * CPU oracle for the RESET set-intersection path: TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithms (table layout,
 * table build, hash functions, probe rule, hash-order extraction and the four
 * applications: triangle counting, set-similarity search, conjunctive IR and
 * the raw pair intersection).  It is the checker that the CUDA library is
 * compared against; only tests, the smoke check and the CPU-baseline leg of
 * the benchmark may load it.  Nothing in the product links against it.
 *
 * Every function cites the reference file:line it follows (paths relative to
 * the RESET repository root).  Parity of this restatement is pinned against
 * outputs of the reference's own kernels, compiled unchanged for sm_100a and
 * run on identical inputs (fixtures under tests/golden/).
 */
#ifndef RESET_ORACLE_H
#define RESET_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- table layout ------------------------------------------------------ */

/* triangle-count/hashtable.cu:21-36: t=(int)(d/alpha) in float, L=t/b,
 * L==0 -> 8, else next power of two strictly above L, at least 8. */
int32_t ro_calc_len(int32_t degree, float alpha, int32_t bucket);

/* triangle-count/TC.cuh:48-52 */
int32_t ro_hash_normal(int32_t x, int32_t len);
/* triangle-count/TC.cuh:40-46 (shift = ffs(max_len) - ffs(len)) */
int32_t ro_hash_hier(int32_t x, int32_t len, int32_t max_len);

/* triangle-count/hashtable.cu:103-128 (calculate_hash_length + exclusive
 * scan): fills len[n], off64[n+1] (off64[n] = bucket_num), *max_len.
 * Returns bucket_num.  max_len is 8 when n == 0. */
int64_t ro_table_meta(int32_t n, const int32_t *off, float alpha,
                      int32_t bucket, int32_t *len, int64_t *off64,
                      int32_t *max_len);

/* triangle-count/hashtable.cu:53-101 insertion rule, applied sequentially in
 * CSR order (the order of the commented-out host build at
 * information-retrieval/hashtable.cu:102-160).  table has bucket*bucket_num
 * int32 entries; slot k of bucket h of set u is table[off64[u]+h+k*bucket_num].
 * Returns 0, or -1 if some set's table overflowed (cannot happen for
 * alpha <= 1). */
int32_t ro_table_build(int32_t n, const int32_t *off, const int32_t *elems,
                       int32_t bucket, const int32_t *len,
                       const int64_t *off64, int64_t bucket_num,
                       int32_t max_len, int32_t hier, int32_t *table);

/* triangle-count/TC.cu:11-31 probe rule for one key into set u's table. */
int32_t ro_probe(int32_t key, const int32_t *table, int64_t toff,
                 int64_t bucket_num, int32_t len, int32_t max_len,
                 int32_t bucket, int32_t hier);

/* baseline/common/utils.cu:76-146: read every set's table back slot-major
 * within the set (bucket = i / b, slot = i % b), dropping -1. */
void ro_hash_order(int32_t n, const int32_t *off, const int64_t *off64,
                   const int32_t *table, int64_t bucket_num, int32_t bucket,
                   int32_t *cols_out);

/* ---- applications ------------------------------------------------------ */

/* Independent check: sum over oriented edges (u,v) of |N(u) ∩ N(v)| by
 * sorted-row merge.  Rows must be sorted ascending.  OpenMP over vertices. */
uint64_t ro_tc_merge(int32_t n, const int32_t *off, const int32_t *cols,
                     int32_t nthreads);
/* Same, restricted to the vertex range [v0, v1) (bounded CPU samples). */
uint64_t ro_tc_merge_range(int32_t n, const int32_t *off, const int32_t *cols,
                           int32_t v0, int32_t v1, int32_t nthreads);

/* triangle-count/TC.cu:128-190: per edge, the smaller row's keys are probed
 * into the larger row's table (ties keep u as the probing side). */
uint64_t ro_tc_hash(int32_t n, const int32_t *off, const int32_t *cols,
                    const int32_t *len, const int64_t *off64,
                    const int32_t *table, int64_t bucket_num, int32_t max_len,
                    int32_t bucket, int32_t hier, int32_t nthreads);

/* set-similarity-search/sss.cu:93-154 for explicit pairs (a[p], b[p]).
 * inter_out[p] = |smaller ∩ larger| counted by probing.
 * mode 0: reference float rule  (float)I / (float)(|A|+|B|-I) >= thr.
 * mode 1: integer rule          U > 0 && den*I >= num*U.
 * flags_out[p] in {0,1}. */
void ro_sss(int32_t n, const int32_t *off, const int32_t *elems,
            const int32_t *pa, const int32_t *pb, int64_t npairs,
            const int32_t *len, const int64_t *off64, const int32_t *table,
            int64_t bucket_num, int32_t max_len, int32_t bucket, int32_t hier,
            int32_t mode, float thr, int32_t num, int32_t den,
            uint8_t *flags_out, int32_t *inter_out);

/* information-retrieval/ir.cu:94-176: per query, the posting list of the
 * first term (in stored order) filtered by every further term's table.
 * result[res_off[q] .. res_off[q]+count[q]) receives the survivors in
 * first-term order; an empty query yields count 0. */
void ro_ir(int32_t nterms, const int32_t *toff, const int32_t *docs,
           const int32_t *query, const int32_t *qoff, int32_t nq,
           const int64_t *res_off, const int32_t *len, const int64_t *off64,
           const int32_t *table, int64_t bucket_num, int32_t max_len,
           int32_t bucket, int32_t hier, int32_t *result, int32_t *count);

/* set_size/intersection.cu:154-181: number of elements of A (with A's
 * multiplicity) that occur in B. */
int64_t ro_pair_count(const int32_t *a, int64_t na, const int32_t *b,
                      int64_t nb);

/* All pairs a < b of sorted token sets with den*I >= num*U (U > 0); writes
 * at most cap pairs in (a, b) order, returns the full count. */
int64_t ro_jaccard_join(int32_t n, const int32_t *off, const int32_t *tok,
                        int32_t num, int32_t den, int32_t *pa, int32_t *pb,
                        int64_t cap);

/* 4-cliques of an oriented graph with sorted rows (merge intersections). */
uint64_t ro_clique4(int32_t n, const int32_t *off, const int32_t *cols);
/* k-cliques (k >= 3) of an oriented graph with sorted rows, each counted
 * once (SMOG/SMOG_hie/subgraph_match_hie.cu:58-247). */
uint64_t ro_clique_k(int32_t n, const int32_t *off, const int32_t *cols, int32_t k);
/* Embeddings of a pattern in SMOG's encoding (k vertices; backward lists
 * by offsets; restriction / reuse arrays or NULL; flags 1 = restrictions,
 * 2 = distinctness) in a graph with sorted rows, counted by the definition
 * (SMOG/SMOG_hie/subgraph_match_hie.cu:23-42, 58-406); nthreads <= 0 = all
 * cores. */
uint64_t ro_pattern_count(int32_t n, const int32_t *off, const int32_t *cols,
                          int32_t k, int32_t flags, const int32_t *offsets,
                          const int32_t *backward, const int32_t *restriction,
                          const int32_t *reuse, int32_t nthreads);

/* ---- synthetic inputs --------------------------------------------------- */

/* splitmix64 finaliser; the R-MAT draw for edge i uses 16-bit fields of
 * ro_rmat_word(seed, i, g) = mix64(seed ^ mix64(8*i + g)), four levels per
 * word, quadrant by integer thresholds ta < tb < tc on [0, 65536). */
uint64_t ro_mix64(uint64_t z);
void ro_rmat_thresholds(double a, double b, double c, int32_t *ta,
                        int32_t *tb, int32_t *tc);
void ro_rmat_edge(uint64_t seed, int64_t i, int32_t scale, int32_t ta,
                  int32_t tb, int32_t tc, int32_t *u, int32_t *v);

/* Seeded bijection of [0, 2^scale) used to relabel R-MAT vertices (the
 * Graph500 Kronecker generator permutes vertex labels the same way, so that
 * ids carry no trace of the recursive quadrant choice): three rounds of
 * x = (x * M_r) mod 2^scale; x ^= x >> ceil(scale/2); x = (x + A_r) mod 2^scale,
 * M_r = mix64(seed ^ (0x5EC0DE00 + 2r)) | 1, A_r = mix64(seed ^ (0x5EC0DE01 + 2r)). */
uint32_t ro_relabel(uint64_t seed, int32_t scale, uint32_t x);

typedef struct {
  int32_t n;
  int64_t m;
  int32_t *off;  /* n+1 */
  int32_t *cols; /* m */
} ro_csr;

/* R-MAT scale/edge-factor graph, vertices relabeled by ro_relabel (unless
 * mode & 2), self-loops and duplicates removed, symmetrised.  mode & 1 == 0:
 * oriented low-degree -> high-degree (ties by id), the triangle-counting
 * input; mode & 1 == 1: full symmetric adjacency.  Rows sorted ascending. */
ro_csr *ro_rmat_graph(int32_t scale, int32_t edge_factor, uint64_t seed,
                      double a, double b, double c, int32_t mode);
void ro_csr_free(ro_csr *g);

#ifdef __cplusplus
}
#endif
#endif
