/*
 * reset.h -- C ABI of the B200-native RESET set-intersection library
 * (libreset.so, sm_100a).
 *
 * Drop-in boundary for the reference's set-intersection path.  The reference
 * has no FFI of its own: its entry points are C++ free functions over process
 * globals, HashTableBuilder / *Baseline classes, and raw __global__ kernels.
 * Each function below names the reference interface it replaces.
 *
 * Conventions
 *  - extern "C", plain pointers and sizes, int32 status returns; nothing
 *    throws across the boundary.  reset_last_error_string() describes the
 *    last failure on the calling host thread.
 *  - Pointers prefixed d_ are device (HBM) pointers; h_ are host pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Calls are asynchronous on that stream except where noted.
 *  - Tables use the reference layout: set u owns len[u] buckets of
 *    `bucket` slots; slot k of bucket h of set u is
 *        table[off[u] + h + k * bucket_num]        (int32, -1 = empty)
 *    with bucket_num = sum(len) (triangle-count/hashtable.cu:53-76,
 *    triangle-count/TC.cu:18).
 *  - Handles are re-entrant: different tables may be used concurrently from
 *    different threads/streams.  One table may be probed concurrently.
 */
#ifndef RESET_H
#define RESET_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *reset_stream_t; /* cudaStream_t */

typedef enum {
  RESET_OK = 0,
  RESET_ERR_CUDA = 1,        /* a CUDA runtime call failed */
  RESET_ERR_OOM = 2,         /* device allocation failed */
  RESET_ERR_ARG = 3,         /* invalid argument */
  RESET_ERR_TABLE_FULL = 4,  /* a set does not fit its table (alpha > 1) */
  RESET_ERR_PROBE_LIMIT = 5, /* a probe walked a whole table */
  RESET_ERR_TIMEOUT = 6,     /* a bounded wait gave up */
  RESET_ERR_UNSUPPORTED = 7, /* no sm_100 device / feature not built */
  RESET_ERR_BUSY = 8         /* admission refused (serving) */
} reset_status;

#define RESET_ABI_VERSION 1

/* Table parameters.  Defaults (reset_params_default): alpha = 0.2,
 * bucket = 5, the reference defaults of triangle-count/TC.cu:220-221. */
typedef struct reset_params {
  float alpha;      /* load factor (0, 1]                                  */
  int32_t bucket;   /* slots per bucket, 1..16                             */
  int32_t reserved[6];
} reset_params;

void reset_params_default(reset_params *p);

/* Opaque device-resident table (replaces the globals d_hash_table_*,
 * d_hash_length, d_hash_tables_offset, max_length, bucket_num of
 * triangle-count/TC.cuh:23-28 and the HashTableBuilder members of
 * baseline/common/hash_table.cuh:82-94). */
typedef struct reset_table reset_table;

typedef struct reset_table_view {
  int32_t n;            /* number of sets                                  */
  int32_t bucket;       /* slots per bucket                                */
  int32_t max_len;      /* maximum len over all sets                       */
  int32_t hierarchical; /* 1: hierarchical hash, 0: normal hash            */
  int64_t bucket_num;   /* total buckets = sum(len)                        */
  int64_t m;            /* number of elements inserted                     */
  float alpha;
  int32_t pad;
  int32_t *d_table;     /* bucket * bucket_num int32, slot-major           */
  int32_t *d_len;       /* n                                               */
  int64_t *d_off;       /* n + 1, d_off[n] == bucket_num                   */
} reset_table_view;

/* Build one table over the sets of a CSR (d_off[n+1] int32, d_elems[m]
 * int32, element ids >= 0).  Replaces make_hash_table
 * (triangle-count/hashtable.cu:103-183; set-similarity-search/
 * hashtable.cu:100-181; information-retrieval/hashtable.cu:162-249) and
 * HashTableBuilder::build_hash_tables (baseline/common/hash_table.cu:69-192)
 * for one hash function at a time.  len/off/bucket_num/max_len follow
 * calculate_length (triangle-count/hashtable.cu:21-36) exactly.  Keys are
 * placed by the reference insertion rule (hashtable.cu:53-101) applied in
 * CSR order, so the layout is deterministic.  Synchronises `stream` once
 * (to size the table).  If d_hash_order_out is not NULL it receives, in the
 * same pass, every row read back in bucket order (what
 * launch_extract_hashtable_to_csr, baseline/common/utils.cu:148-175,
 * produces). */
reset_status reset_table_build(const int32_t *d_off, const int32_t *d_elems,
                               int32_t n, int64_t m, const reset_params *params,
                               int32_t hierarchical, int32_t *d_hash_order_out,
                               reset_table **out, reset_stream_t stream);

/* Device pointers and sizes of a table (for dumps and for callers that
 * launch their own kernels over the reference layout).  Host-only. */
reset_status reset_table_info(const reset_table *t, reset_table_view *view);

/* Free a table (replaces HashTableBuilder::free_hash_tables,
 * baseline/common/hash_table.cuh:45-72).  Synchronises the device.  Table
 * memory comes from a library-owned stream-ordered pool that keeps freed
 * pages mapped, so the next build of a similar table maps no new memory. */
reset_status reset_table_free(reset_table *t);

/* Stream-ordered free: the table's memory returns to the pool when `stream`
 * reaches this point; no host or device synchronisation.  Every use of the
 * table on other streams must be ordered before it (events) by the caller. */
reset_status reset_table_free_async(reset_table *t, reset_stream_t stream);

/* Returns the pages the table pool keeps for reuse to the device
 * (no counterpart in the reference).  Synchronises the device. */
reset_status reset_release_cached_memory(void);

/* Synchronise `stream` and report device-side errors raised by kernels that
 * used this table since the last call (RESET_ERR_TABLE_FULL,
 * RESET_ERR_PROBE_LIMIT, RESET_ERR_ARG for a row, pair or query id outside
 * [0, n), RESET_ERR_TIMEOUT for a bounded wait that gave up), then clear
 * them. */
reset_status reset_table_check(reset_table *t, reset_stream_t stream);

/* Rows of the table's CSR read back in bucket order (slot-major within each
 * set, -1 dropped).  Replaces launch_extract_hashtable_to_csr
 * (baseline/common/utils.cu:148-175) and the sort by column % max_length
 * of gpu_sort_csr_cols (triangle-count/TC.cu:107-126). */
reset_status reset_csr_hash_order(const reset_table *t, const int32_t *d_off,
                                  int32_t *d_cols_out, reset_stream_t stream);

/* Triangle count over an oriented CSR whose table is `t`:
 *   sum over edges e=(u, d_cols[e]) of |row(u) ∩ row(v)|,
 * the smaller row's keys probed into the larger row's table.  d_cols may be
 * the plain rows or the hash-ordered rows.  *d_count (device u64) is
 * overwritten.  Replaces dynamic_triangle_count (triangle-count/TC.cu:128-190)
 * and TCBaseline::run_{normal,hierarchical} (baseline/tc/tc.cu:165-237). */
reset_status reset_tc_count(const reset_table *t, const int32_t *d_off,
                            const int32_t *d_cols, int64_t m,
                            uint64_t *d_count, reset_stream_t stream);

/* reset_tc_count with an explicit method (same count either way):
 *   0 = default (1, the faster on B200 as measured);
 *   1 = edge-flattened: 32 edges per warp; pairs with at least
 *       warp_pair_min keys (reset_tuning, default 64) probed by the whole
 *       warp, smaller ones flattened across the lanes, both sides read from
 *       HBM (the reference's access pattern);
 *   2 = vertex-staged: each row staged once in shared memory (keys + hash
 *       set) and reused by all its out-edges. */
reset_status reset_tc_count_ex(const reset_table *t, const int32_t *d_off,
                               const int32_t *d_cols, int64_t m,
                               int32_t method, uint64_t *d_count,
                               reset_stream_t stream);

/* reset_tc_count for callers that cannot allocate device memory while they
 * run -- for example a serving process that has reserved nearly all HBM for
 * resident tables, where a cudaMalloc can fail mid-request and a cudaFree
 * synchronises the whole device and stalls every other stream.  It has no
 * counterpart in the reference.  Same count as reset_tc_count (vertex-staged
 * method); it calls no cudaMalloc, cudaFree or allocating library routine.
 * Its scratch (four work counters and up to 2^20 work units, 8 MiB) is one
 * fixed device array inside libreset.so, present on every GPU that loads the
 * library until the process exits.  Limits: at most 134,209,536 edges (m and
 * the table's own edge count), d_off must be NULL or the offsets the table
 * was built from, and m must equal the table's edge count (d_cols is the
 * build CSR's column array, or a row-wise permutation of it such as the
 * hash-ordered rows); otherwise RESET_ERR_ARG.  The first call on a device
 * looks up the array's device address (once per device, kept for the life
 * of the device's primary context: do not call it again after a
 * cudaDeviceReset), so make that first call before any stream capture.  All calls share the array and the array
 * keeps the last call's contents (the counters are cleared at every call):
 * calls that overlap on the GPU -- on different streams, or from different
 * threads -- race on it and must be serialised by the caller. */
/* Batched triangle counting: n_graphs disjoint oriented graphs stored as
 * one block-diagonal CSR (graph g owns the vertices
 * d_graph_off[g] .. d_graph_off[g+1] - 1; d_graph_off[0] = 0, nondecreasing,
 * d_graph_off[n_graphs] = n; edges stay inside their graph) with one table.
 * d_counts[g] (device u64) receives graph g's triangle count -- the
 * reference's dynamic_triangle_count (triangle-count/TC.cu:128-190) run once
 * per graph -- from a single owner-grouped count over the whole batch (each
 * triangle is credited to the graph of the vertex whose table it is found
 * in).  d_off/m must be the CSR the table was built on and d_cols 16-byte
 * aligned.  No host synchronisation. */
reset_status reset_tc_count_batch(const reset_table *t, const int32_t *d_off,
                                  const int32_t *d_cols, int64_t m,
                                  const int32_t *d_graph_off, int32_t n_graphs,
                                  uint64_t *d_counts, reset_stream_t stream);

reset_status reset_tc_count_noalloc(const reset_table *t, const int32_t *d_off,
                                    const int32_t *d_cols, int64_t m,
                                    uint64_t *d_count, reset_stream_t stream);

/* Set-similarity decisions for P explicit pairs (d_pair_a[p], d_pair_b[p])
 * of sets of the table's CSR.  I = |A ∩ B| by probing the smaller set into
 * the larger set's table; U = |A| + |B| - I.
 *   d_flags[p] = U > 0 && den * I >= num * U            (exact, integer)
 * d_inter (optional) receives I; without it the call decides only, and a
 * pair stops probing as soon as its decision is settled (enough hits, or
 * too many misses for the threshold to be reachable).  Replaces
 * set_similarity_search_kernel
 * (set-similarity-search/sss.cu:93-154) and SSSBaseline::run_*
 * (baseline/sss/sss.cu:145-251), whose float rule
 * I / (float)U >= thr is available through reset_sss_float. */
reset_status reset_sss(const reset_table *t, const int32_t *d_off,
                       const int32_t *d_elems, const int32_t *d_pair_a,
                       const int32_t *d_pair_b, int64_t npairs, int32_t num,
                       int32_t den, uint8_t *d_flags, int32_t *d_inter,
                       reset_stream_t stream);

/* The reference's float decision, bit-exact with sss.cu:139-141:
 *   d_flags[p] = (float)I / (float)U >= thr. */
reset_status reset_sss_float(const reset_table *t, const int32_t *d_off,
                             const int32_t *d_elems, const int32_t *d_pair_a,
                             const int32_t *d_pair_b, int64_t npairs,
                             float thr, uint8_t *d_flags, int32_t *d_inter,
                             reset_stream_t stream);

/* Batched set-similarity form.  A reset_batch owns device pair buffers for
 * up to `capacity` pairs over one table and a captured CUDA graph of the
 * persistent pair kernel; reset_batch_run decides the first `npairs` pairs
 * of those buffers with one graph replay (no allocation, no per-batch
 * launch setup).  Decisions are those of reset_sss with the num/den given
 * at creation.  The caller fills *d_pair_a / *d_pair_b (from
 * reset_batch_buffers) on `stream` or before the call; results land in
 * *d_flags / *d_inter.  A batch belongs to one thread at a time.
 * The batched counterpart of the reference's per-call SSS launch
 * (set-similarity-search/sss.cu:93-154 with the host loop of
 * set-similarity-search/main.cu). */
typedef struct reset_batch reset_batch;
reset_status reset_batch_create(const reset_table *t, const int32_t *d_elems,
                                int64_t capacity, int32_t num, int32_t den,
                                reset_batch **out, reset_stream_t stream);
/* Options of reset_batch_create_ex. */
#define RESET_BATCH_DECISIONS_ONLY 1 /* flags only: each pair stops as soon as its
                                        decision is settled; *d_inter is not
                                        written                                 */
#define RESET_BATCH_OWNER_GROUPED 2  /* the replay groups the pairs by the
                                        larger set, stages its table in shared
                                        memory and streams the smaller sets
                                        through it (full sizes, *d_inter
                                        written); d_elems 16-byte aligned.
                                        Faster for many pairs per large set */
reset_status reset_batch_create_ex(const reset_table *t, const int32_t *d_elems,
                                   int64_t capacity, int32_t num, int32_t den,
                                   int32_t options, reset_batch **out,
                                   reset_stream_t stream);
reset_status reset_batch_buffers(reset_batch *b, int32_t **d_pair_a,
                                 int32_t **d_pair_b, uint8_t **d_flags,
                                 int32_t **d_inter);
reset_status reset_batch_run(reset_batch *b, int64_t npairs,
                             reset_stream_t stream);
reset_status reset_batch_destroy(reset_batch *b);

/* Prefix-filter candidates for a Jaccard self-join at threshold num/den
 * over token sets (d_off[n+1], d_tokens; tokens in [0, 2^universe_log2),
 * distinct within a set).  Tokens are ordered globally by (frequency, id);
 * set x's prefix is its first |x| - ceil(num*|x|/den) + 1 tokens in that
 * order.  A pair (a < b) is a candidate iff the prefixes share a token and
 * den*min(|a|,|b|) >= num*max(|a|,|b|); every pair with Jaccard >= num/den
 * is a candidate.  Outputs: distinct pairs sorted by (a, b), allocated with
 * cudaMalloc, owned by the caller.  n < 2^21, set sizes < 2^15.
 * Synchronises `stream`. */
reset_status reset_prefix_candidates(const int32_t *d_off, const int32_t *d_tokens,
                                     int32_t n, int64_t m, int32_t universe_log2,
                                     int32_t num, int32_t den, int32_t **d_pa_out,
                                     int32_t **d_pb_out, int64_t *np_out,
                                     reset_stream_t stream);

/* Conjunctive retrieval.  The table is built over the inverted index
 * (d_toff[nterms+1], d_docs).  Query q is the term list
 * d_query[d_qoff[q] .. d_qoff[q+1]); its result is the posting list of its
 * first term, in d_docs order, filtered by membership in every further
 * term's table.  Survivors go to d_res[d_res_off[q] ...] (the caller sizes
 * slot q for df(first term), as ir.cu:324-330 does); d_cnt[q] receives the
 * count.  Empty queries yield 0.  Replaces ir_kernel
 * (information-retrieval/ir.cu:94-176) and IRBaseline::run_*
 * (baseline/ir/ir.cu:240-343). */
reset_status reset_ir(const reset_table *t, const int32_t *d_toff,
                      const int32_t *d_docs, const int32_t *d_query,
                      const int32_t *d_qoff, int32_t nq,
                      const int64_t *d_res_off, int32_t *d_res,
                      int32_t *d_cnt, reset_stream_t stream);

/* 4-cliques of an oriented graph (rows sorted ascending, oriented as for
 * reset_tc_count) whose table is `t` (built on d_off/d_cols):
 *   sum over edges (u, v) of sum over w in W of |W ∩ N+(w)|,
 * W = N+(u) ∩ N+(v), every intersection by hash probes.  *d_count (device
 * u64) is overwritten.  The depth-4 clique search of SMOG's
 * DFSKernelForClique (SMOG/SMOG_hie/subgraph_match_hie.cu:58-247) over this
 * library's tables.  Synchronises `stream` once (scratch sizing). */
reset_status reset_clique4_count(const reset_table *t, const int32_t *d_off,
                                 const int32_t *d_cols, int64_t m,
                                 uint64_t *d_count, reset_stream_t stream);

/* k-cliques, 3 <= k <= 16, of an oriented graph whose table is `t` (built
 * on d_off/d_cols): SMOG's clique DFS (DFSKernelForClique,
 * SMOG/SMOG_hie/subgraph_match_hie.cu:58-247) with every candidate set
 * C_{j+1} = C_j ∩ N+(w) found by hash probes, starting from
 * C_0 = N+(u) ∩ N+(v) for every edge (u, v); each clique is counted once.
 * k = 3 gives the triangle count, k = 4 the 4-clique count.  *d_count
 * (device u64) is overwritten.  Synchronises `stream` once (scratch
 * sizing: k - 3 rows of the largest out-degree per warp). */
reset_status reset_clique_count(const reset_table *t, const int32_t *d_off,
                                const int32_t *d_cols, int64_t m, int32_t k,
                                uint64_t *d_count, reset_stream_t stream);

/* A query pattern for reset_pattern_count, in the encoding of SMOG's
 * pattern table (SMOG/SMOG_hie/script_hie.py:85-152, which writes it to
 * constants.cpp as intersection_orders, intersection_offset, restriction
 * and reuse, with H and the withRestriction / withDuplicate defines):
 *   k            pattern vertices (H), 3..RESET_PATTERN_MAX; vertices 0 and
 *                1 are the two ends of the start edge;
 *   offsets      k entries: backward[offsets[l-1] .. offsets[l]) are the
 *                earlier pattern vertices adjacent to vertex l (l >= 1;
 *                level 1 must be [0]); -1 stands for the vertices that
 *                the reused level's set already covers;
 *   backward     offsets[k-1] entries;
 *   restriction  k entries or NULL (all -1): r = restriction[l] >= 0
 *                requires m_l < m_r when flags has RESET_PATTERN_RESTRICT;
 *                with RESET_PATTERN_DISTINCT a level whose r is -1
 *                requires m_l to differ from m_0 .. m_{l-1}
 *                (checkRestriction, subgraph_match_hie.cu:23-42);
 *   reuse        k entries or NULL (all -1): reuse[l] = r in [2, l) makes
 *                level l start from level r's candidate set; such a level
 *                lists exactly one -1, every other level none. */
#define RESET_PATTERN_RESTRICT 1
#define RESET_PATTERN_DISTINCT 2
#define RESET_PATTERN_MAX 8
typedef struct reset_pattern {
  int32_t k;
  int32_t flags;
  const int32_t *offsets;
  const int32_t *backward;
  const int32_t *restriction;
  const int32_t *reuse;
} reset_pattern;

/* Embeddings of pattern `p` in the graph whose table is `t` (built on
 * d_off/d_cols): the number of tuples (m_0 .. m_{k-1}) with (m_0, m_1) a
 * stored edge and, for l >= 2, m_l in
 *   C_l = [C_reuse(l) or all vertices] ∩ (∩ over listed j of N(m_j)),
 * each level passing its restriction / distinctness check.  SMOG's
 * DFSKernelForGeneral and DFSKernelForClique
 * (SMOG/SMOG_hie/subgraph_match_hie.cu:58-406) as one warp-level DFS per
 * start edge; C_l starts from the smallest listed row (or the reused set)
 * and probes the other listed rows' tables.  Symmetric CSR for general
 * patterns, oriented for cliques, as the reference loads them
 * (SMOG/SMOG_hie/common_hie.cu:61-85).  Rows in any order; strictly
 * ascending rows take shortcuts (restriction prefixes, counts without a
 * scan).  A reusing k-clique chain without checks runs
 * reset_clique_count.  *d_count (device u64) is overwritten.  Synchronises
 * `stream` once (scratch sizing and the row-order check). */
reset_status reset_pattern_count(const reset_table *t, const int32_t *d_off,
                                 const int32_t *d_cols, int64_t m,
                                 const reset_pattern *p, uint64_t *d_count,
                                 reset_stream_t stream);

/* SMOG's query patterns by name, "Q0" .. "Q8" (SMOG/SMOG_hie/
 * script_hie.py:85-152): *out points at library-owned static arrays;
 * *oriented (if not NULL) is 1 for the patterns SMOG counts on the oriented
 * graph (Q0, Q3, Q5, Q7: begin.bin / adjacent.bin), 0 for those it counts
 * on the symmetric one (generic_*.bin; SMOG/SMOG_hie/common_hie.cu:72-85).
 * RESET_ERR_ARG for another name.  Host-only. */
reset_status reset_pattern_named(const char *name, reset_pattern *out, int32_t *oriented);

/* |A ∩ B| counted with A's multiplicity for one pair of device arrays
 * (keys >= 0).  Builds B's table with `params` and probes A.  *d_count
 * (device i64) is overwritten.  Replaces make_hashtable_kernel +
 * intersection_kernel (set_size/intersection.cu:128-181). */
reset_status reset_intersect_count(const int32_t *d_a, int64_t na,
                                   const int32_t *d_b, int64_t nb,
                                   const reset_params *params,
                                   int64_t *d_count, reset_stream_t stream);

/* ---- element-modulo sharding -------------------------------------------- */
/* Shard `shard` of `shards` of a CSR: every row keeps, in order, its
 * elements x with x % shards == shard (C remainder), the per-device input of
 * the reference's multi-GPU programs (multi-GPU/tc-multi-GPU/main.cu:113-130,
 * multi-GPU/sss-multi-GPU/main.cu:124-136).  d_off_out has n + 1 entries,
 * d_cols_out room for m; *d_m_out (device, optional) receives the shard's
 * element count.  No host synchronisation. */
reset_status reset_csr_shard(const int32_t *d_off, const int32_t *d_cols,
                             int32_t n, int64_t m, int32_t shards,
                             int32_t shard, int32_t *d_off_out,
                             int32_t *d_cols_out, int64_t *d_m_out,
                             reset_stream_t stream);

/* Partial triangle count of one shard, replacing partial_tc
 * (multi-GPU/tc-multi-GPU/tc.cu:264): sum over the edges (u, v) of the
 * full edge CSR of |K(u) ∩ K(v)|, where K is the shard CSR (d_key_off,
 * d_key_cols, 16-byte aligned) that `t` was built on; the smaller shard row
 * probes the larger one's table.  Summed over all shards (on one device or
 * across devices) it equals reset_tc_count of the full graph (rows without
 * repeated entries).  *d_count (device u64) is overwritten. */
reset_status reset_tc_count_shard(const reset_table *t, const int32_t *d_key_off,
                                  const int32_t *d_key_cols, int64_t m_keys,
                                  const int32_t *d_edge_off,
                                  const int32_t *d_edge_cols, int64_t m_edges,
                                  uint64_t *d_count, reset_stream_t stream);

/* Set-similarity decisions from intersection sizes summed over shards
 * (multi-GPU/sss-multi-GPU/main.cu:144-151, with the exact integer rule):
 * d_flags[p] = U > 0 && den * I >= num * U, I = d_inter[p],
 * U = |A| + |B| - I with the full sets' sizes from d_off.  Pair ids outside
 * [0, n) give flag 0 and set bit 4 (an out-of-range id) in *d_status_bits
 * (optional). */
reset_status reset_sss_decide(const int32_t *d_off, int32_t n,
                              const int32_t *d_pair_a, const int32_t *d_pair_b,
                              int64_t npairs, const int32_t *d_inter,
                              int32_t num, int32_t den, uint8_t *d_flags,
                              int32_t *d_status_bits, reset_stream_t stream);

/* ---- synthetic inputs (stand-ins for the reference's datasets) -------- */

/* Options of reset_gen_rmat. */
#define RESET_GEN_SYMMETRIC 1 /* full symmetric adjacency instead of oriented */
#define RESET_GEN_KEEP_IDS 2  /* keep raw R-MAT ids (no relabeling)          */

/* Seeded R-MAT graph on the device: 2^scale vertices, edge_factor*2^scale
 * generated edges, vertex labels relabeled by a seeded bijection (the
 * Graph500 convention; RESET_GEN_KEEP_IDS skips it), self-loops and
 * duplicates removed, symmetrised.  Default: keep u->v iff
 * (deg u, u) < (deg v, v) (triangle-counting input); RESET_GEN_SYMMETRIC:
 * full symmetric adjacency.  Rows sorted ascending.  Outputs are allocated
 * with cudaMalloc and owned by the caller (free with reset_free).
 * Synchronises `stream`. */
reset_status reset_gen_rmat(int32_t scale, int32_t edge_factor, uint64_t seed,
                            double a, double b, double c, int32_t options,
                            int32_t **d_off_out, int32_t **d_cols_out,
                            int64_t *m_out, reset_stream_t stream);

/* Seeded token sets (stand-in for the set-similarity datasets): n sets,
 * set sizes Zipf(size_s) on [size_lo, size_hi], tokens drawn from a
 * Zipf(1)-like law over 2^universe_log2 ranks and relabeled by a seeded
 * bijection; duplicates removed, rows sorted.  With probability dup_frac a
 * set (other than the first) is a near-duplicate of the nearest earlier
 * non-duplicate set within 256: same size, each of that set's draws kept
 * with probability keep ~ U(keep_min, 1), fresh draws otherwise.  Outputs
 * allocated with cudaMalloc, owned by the caller.  n < 2^21,
 * size_hi <= 16384, universe_log2 in 4..24.  Synchronises `stream`. */
reset_status reset_gen_token_sets(int32_t n, int32_t universe_log2, double size_s,
                                  int32_t size_lo, int32_t size_hi, double dup_frac,
                                  double keep_min, uint64_t seed,
                                  int32_t **d_off_out, int32_t **d_tokens_out,
                                  int64_t *m_out, reset_stream_t stream);
/* Seeded inverted index (stand-in for the IR corpora): term t (0-based
 * rank) gets df(t) = clamp(round(df_max * (t+1)^-zipf_s), 1, ndocs) uniform
 * doc-id draws from [0, ndocs); duplicates removed, posting lists sorted.
 * Outputs (d_toff[nterms+1], d_docs[m]) allocated with cudaMalloc, owned by
 * the caller.  Synchronises `stream`. */
reset_status reset_gen_inverted_index(int32_t nterms, int32_t ndocs, double zipf_s,
                                      int64_t df_max, uint64_t seed,
                                      int32_t **d_toff_out, int32_t **d_docs_out,
                                      int64_t *m_out, reset_stream_t stream);
reset_status reset_free(void *d_ptr);

/* ---- served form ----------------------------------------------------------- */

/* A request loop over device-resident indexes with continuous batching: a
 * scheduler thread drains the arrival queue into batches whenever one of
 * `streams` slots is free, admitting requests (FIFO) while their device bytes
 * fit the memory budget; batches on different slots overlap on the GPU.  A
 * result depends only on its request and the index: it is the same whether
 * the request ran alone or in a mix.  No counterpart in the reference (its
 * applications run one offline batch per process: triangle-count/TC.cu:
 * 192-247, set-similarity-search/sss.cu:191-244,
 * information-retrieval/ir.cu:213-267, set_size/intersection.cu:183-192). */
typedef struct reset_server reset_server;

typedef struct {
  int32_t streams;            /* batches in flight at once (default 4)        */
  int32_t max_batch_requests; /* requests per batch at most (default 1024)    */
  int64_t mem_budget_bytes;   /* device bytes for batches; 0 = half the free
                                 device memory when the server starts        */
  int64_t max_batch_cost;     /* estimated probes per batch at most (default
                                 2^22; 0 = no limit).  A request above it runs
                                 in a batch of its own, and such batches hold
                                 at most streams - 1 slots, so lighter requests
                                 never wait behind one (they may pass it)   */
  int64_t pinned_result_bytes; /* pinned host arena that IR results land in
                                 and are handed out from without a copy
                                 until released (default 256 MiB); results
                                 that do not fit are copied out           */
  int32_t reserved[4];
} reset_server_config;

enum {
  RESET_REQ_IR = 1,        /* args: query terms (first term's list filtered
                              by the others, as reset_ir); -> docs          */
  RESET_REQ_PAIRS = 2,     /* args: (a, b) set pairs; num/den threshold;
                              -> values = |A ∩ B|, flags, count = #similar  */
  RESET_REQ_TRIPLES = 3,   /* args: (a, b, c); -> values = |A ∩ B ∩ C|       */
  RESET_REQ_TC_VERTEX = 4, /* args: vertices v of an oriented graph index;
                              -> values = sum over w in N(v) of
                                 |N(v) ∩ N(w)| (triangles with v first)     */
  RESET_REQ_RAW = 5        /* args: A, args2: B (host keys >= 0, no index);
                              -> count = |A ∩ B| with A's multiplicity       */
};

typedef struct {
  int32_t kind;        /* RESET_REQ_*                                        */
  int32_t index;       /* from reset_server_add_index (unused by RAW)        */
  const int32_t *args; /* host array, copied at submit                       */
  int64_t nargs;
  const int32_t *args2;
  int64_t nargs2;
  int32_t num, den;    /* PAIRS: similar iff den*I >= num*U, U > 0           */
  int64_t arrival_ns;  /* reset_now_ns() clock; 0 = the submit time          */
  int32_t reserved[4];
} reset_request;

typedef struct {
  reset_status status;
  int32_t kind;
  int64_t count;          /* IR: #docs; PAIRS: #similar; others: sum        */
  const int32_t *docs;    /* IR result list (ndocs), first-term order       */
  int64_t ndocs;
  const int64_t *values;  /* per pair / triple / vertex (nvalues)           */
  int64_t nvalues;
  const uint8_t *flags;   /* PAIRS decisions (nvalues)                      */
  double queue_us;        /* arrival -> batch launch                        */
  double service_us;      /* batch launch -> results on the host            */
  double latency_us;      /* arrival -> results on the host                 */
  int64_t batch_id;
  int32_t batch_size;
  int32_t reserved;
} reset_result;

typedef struct {
  int64_t completed, batches, max_batch, pending;
  int64_t inflight_batches, max_inflight_batches;
  int64_t budget_bytes, in_use_bytes, max_in_use_bytes;
  double mean_batch;
  double launch_host_us;  /* host time spent packing and launching batches  */
  double batch_us;        /* sum over batches of launch -> results unpacked */
  int64_t arena_bytes;    /* device buffers the slots keep for reuse        */
  double max_launch_us;   /* longest host time packing + launching a batch  */
  double max_finish_us;   /* longest host time handing a batch's results out */
  int64_t reserved[2];
} reset_server_counters;

void reset_server_config_default(reset_server_config *cfg);
int64_t reset_now_ns(void);
reset_status reset_server_create(const reset_server_config *cfg, reset_server **out);
/* Registers a built table as an index; d_off must be the offsets it was
 * built on (their host copy is taken for planning).  The table and arrays
 * must outlive the server. */
reset_status reset_server_add_index(reset_server *s, const reset_table *t,
                                    const int32_t *d_off, const int32_t *d_elems,
                                    int32_t *index_out);
/* Queues a request; invalid ids fail here (RESET_ERR_ARG).  A request that
 * can never fit the memory budget completes with RESET_ERR_OOM. */
reset_status reset_server_submit(reset_server *s, const reset_request *req,
                                 uint64_t *ticket);
/* Waits up to timeout_ms (< 0: no limit; RESET_ERR_TIMEOUT when it runs
 * out).  The result's arrays stay valid until reset_server_release. */
reset_status reset_server_wait(reset_server *s, uint64_t ticket, int32_t timeout_ms,
                               reset_result *out);
reset_status reset_server_release(reset_server *s, uint64_t ticket);
reset_status reset_server_stats(reset_server *s, reset_server_counters *out);
/* Finishes queued requests, then stops. */
reset_status reset_server_destroy(reset_server *s);

/* ---- tuning --------------------------------------------------------------- */

/* Process-wide kernel knobs (no counterpart in the reference, whose launch
 * shapes are compile-time constants).  Results never depend on them. */
typedef struct reset_tuning {
  int32_t probe_rounds;  /* 2, 4 (or 8 with variant 1): probe rounds a warp
                            keeps in flight                                 */
  int32_t warp_pair_min; /* pairs with >= this many keys get a whole warp   */
  int32_t probe_variant; /* whole-warp pair loop: 0 = software-pipelined,
                            1 = lean (branch-free resolve, no prefetch)     */
  int32_t pair_method;   /* reset_sss / reset_sss_float: 0 = default (1),
                            1 = pair-flattened (with early exit when
                            deciding only), 2 = owner-grouped (tables staged
                            in shared memory; 16-byte aligned elements)      */
  int32_t reserved[4];
} reset_tuning;

reset_status reset_get_tuning(reset_tuning *out);
reset_status reset_set_tuning(const reset_tuning *in);

/* ---- misc --------------------------------------------------------------- */

const char *reset_last_error_string(void);
const char *reset_status_string(int32_t status);
int32_t reset_abi_version(void);
/* Number of launches of libreset's own kernels in this process so far
 * (library routines it calls, such as CUB scans, are not counted). */
int64_t reset_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* RESET_H */
