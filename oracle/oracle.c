/*
 * CPU oracle for the RESET set-intersection path: TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the contract; each function cites the reference
 * file:line whose behaviour it restates.  Only tests, the smoke check and
 * the benchmark's CPU-baseline leg may load this code.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* a tiny parallel-for over [0, n) in chunks, pthreads + an atomic cursor    */
/* ------------------------------------------------------------------------ */

typedef void (*ro_body)(void *ctx, int64_t lo, int64_t hi, uint64_t *acc);

typedef struct {
  ro_body body;
  void *ctx;
  int64_t n, chunk;
  int64_t cursor;
  uint64_t total;
  pthread_mutex_t mu;
} ro_pool;

static void *ro_worker(void *arg) {
  ro_pool *p = (ro_pool *)arg;
  uint64_t acc = 0;
  for (;;) {
    int64_t lo = __atomic_fetch_add(&p->cursor, p->chunk, __ATOMIC_RELAXED);
    if (lo >= p->n) break;
    int64_t hi = lo + p->chunk < p->n ? lo + p->chunk : p->n;
    p->body(p->ctx, lo, hi, &acc);
  }
  pthread_mutex_lock(&p->mu);
  p->total += acc;
  pthread_mutex_unlock(&p->mu);
  return NULL;
}

static int ro_threads(int32_t want) {
  if (want > 0) return want;
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

static uint64_t ro_parallel(int64_t n, int64_t chunk, ro_body body, void *ctx,
                            int32_t nthreads) {
  ro_pool p;
  p.body = body;
  p.ctx = ctx;
  p.n = n;
  p.chunk = chunk > 0 ? chunk : 1;
  p.cursor = 0;
  p.total = 0;
  pthread_mutex_init(&p.mu, NULL);
  int nt = ro_threads(nthreads);
  if (nt > 1024) nt = 1024;
  if (nt <= 1 || n <= p.chunk) {
    ro_worker(&p);
  } else {
    pthread_t th[1024];
    int started = 0;
    for (int i = 0; i < nt; i++)
      if (pthread_create(&th[started], NULL, ro_worker, &p) == 0) started++;
    if (started == 0) ro_worker(&p);
    for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
  }
  pthread_mutex_destroy(&p.mu);
  return p.total;
}

/* ------------------------------------------------------------------------ */
/* table layout                                                              */
/* ------------------------------------------------------------------------ */

int32_t ro_calc_len(int32_t degree, float alpha, int32_t bucket) {
  /* triangle-count/hashtable.cu:23: int total_size = degrees / load_factor;
   * a float division (int promoted to float), truncated toward zero. */
  volatile float q = (float)degree / alpha;
  int32_t total = (int32_t)q;
  int32_t length = total / bucket; /* hashtable.cu:24 */
  if (length == 0) return 8;       /* hashtable.cu:25-26 */
  length |= length >> 1;           /* hashtable.cu:27-32: strict next pow2 */
  length |= length >> 2;
  length |= length >> 4;
  length |= length >> 8;
  length |= length >> 16;
  length++;
  if (length < 8) length = 8; /* hashtable.cu:33-34 */
  return length;
}

int32_t ro_hash_normal(int32_t x, int32_t len) { return x & (len - 1); }

int32_t ro_hash_hier(int32_t x, int32_t len, int32_t max_len) {
  int32_t shift = __builtin_ffs(max_len) - __builtin_ffs(len);
  return (x & (max_len - 1)) >> shift;
}

static inline int32_t home_bucket(int32_t x, int32_t len, int32_t max_len,
                                  int32_t hier) {
  return hier ? ro_hash_hier(x, len, max_len) : ro_hash_normal(x, len);
}

int64_t ro_table_meta(int32_t n, const int32_t *off, float alpha,
                      int32_t bucket, int32_t *len, int64_t *off64,
                      int32_t *max_len) {
  int32_t mx = 0;
  int64_t acc = 0;
  for (int32_t u = 0; u < n; u++) {
    int32_t l = ro_calc_len(off[u + 1] - off[u], alpha, bucket);
    len[u] = l;
    if (l > mx) mx = l;
    off64[u] = acc; /* exclusive scan, hashtable.cu:120-122 */
    acc += l;
  }
  off64[n] = acc; /* bucket_num = last_sum + last_len, hashtable.cu:128-131 */
  *max_len = n > 0 ? mx : 8;
  return acc;
}

int32_t ro_table_build(int32_t n, const int32_t *off, const int32_t *elems,
                       int32_t bucket, const int32_t *len,
                       const int64_t *off64, int64_t bucket_num,
                       int32_t max_len, int32_t hier, int32_t *table) {
  int64_t total = (int64_t)bucket * bucket_num;
  for (int64_t i = 0; i < total; i++) table[i] = -1; /* hashtable.cu:142-143 */
  int32_t status = 0;
  for (int32_t u = 0; u < n; u++) {
    int32_t l = len[u];
    int32_t *base = table + off64[u];
    int64_t cap = (int64_t)l * bucket;
    for (int32_t j = off[u]; j < off[u + 1]; j++) {
      int32_t v = elems[j];
      int32_t h = home_bucket(v, l, max_len, hier);
      int32_t k = 0;
      int64_t tries = 0;
      /* hashtable.cu:65-74: first empty slot of the home bucket, then the
       * next bucket (mod len), slot 0 upward. */
      while (base[h + (int64_t)k * bucket_num] != -1) {
        if (++tries >= cap) {
          status = -1;
          break;
        }
        k++;
        if (k == bucket) {
          k = 0;
          h = (h + 1) % l;
        }
      }
      if (tries >= cap) continue;
      base[h + (int64_t)k * bucket_num] = v;
    }
  }
  return status;
}

int32_t ro_probe(int32_t key, const int32_t *table, int64_t toff,
                 int64_t bucket_num, int32_t len, int32_t max_len,
                 int32_t bucket, int32_t hier) {
  /* triangle-count/TC.cu:11-31 */
  const int32_t *base = table + toff;
  int32_t h = home_bucket(key, len, max_len, hier);
  int32_t k = 0;
  int64_t cap = (int64_t)len * bucket;
  for (int64_t t = 0; t < cap; t++) {
    int32_t s = base[h + (int64_t)k * bucket_num];
    if (s == key) return 1;
    if (s == -1) return 0;
    k++;
    if (k == bucket) {
      k = 0;
      h = (h + 1) & (len - 1);
    }
  }
  return 0; /* full table without the key (not reachable for alpha <= 1) */
}

void ro_hash_order(int32_t n, const int32_t *off, const int64_t *off64,
                   const int32_t *table, int64_t bucket_num, int32_t bucket,
                   int32_t *cols_out) {
  /* baseline/common/utils.cu:89-131 */
  for (int32_t u = 0; u < n; u++) {
    if (off[u + 1] - off[u] <= 0) continue;
    int32_t l = (int32_t)(off64[u + 1] - off64[u]);
    const int32_t *base = table + off64[u];
    int32_t w = off[u];
    for (int32_t i = 0; i < l * bucket; i++) {
      int32_t b = i / bucket, s = i % bucket;
      int32_t x = base[b + (int64_t)s * bucket_num];
      if (x != -1) cols_out[w++] = x;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* applications                                                              */
/* ------------------------------------------------------------------------ */

static inline uint64_t merge_count(const int32_t *a, int32_t na,
                                   const int32_t *b, int32_t nb) {
  uint64_t c = 0;
  int32_t i = 0, j = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j])
      i++;
    else if (a[i] > b[j])
      j++;
    else {
      c++;
      i++;
      j++;
    }
  }
  return c;
}

typedef struct {
  const int32_t *off, *cols;
  int32_t v0;
} tc_merge_ctx;

static void tc_merge_body(void *vctx, int64_t lo, int64_t hi, uint64_t *acc) {
  tc_merge_ctx *c = (tc_merge_ctx *)vctx;
  for (int64_t i = lo; i < hi; i++) {
    int32_t u = c->v0 + (int32_t)i;
    const int32_t *nu = c->cols + c->off[u];
    int32_t du = c->off[u + 1] - c->off[u];
    for (int32_t j = 0; j < du; j++) {
      int32_t v = nu[j];
      *acc += merge_count(nu, du, c->cols + c->off[v], c->off[v + 1] - c->off[v]);
    }
  }
}

uint64_t ro_tc_merge_range(int32_t n, const int32_t *off, const int32_t *cols,
                           int32_t v0, int32_t v1, int32_t nthreads) {
  if (v0 < 0) v0 = 0;
  if (v1 > n) v1 = n;
  if (v1 <= v0) return 0;
  tc_merge_ctx c = {off, cols, v0};
  return ro_parallel(v1 - v0, 64, tc_merge_body, &c, nthreads);
}

uint64_t ro_tc_merge(int32_t n, const int32_t *off, const int32_t *cols,
                     int32_t nthreads) {
  return ro_tc_merge_range(n, off, cols, 0, n, nthreads);
}

typedef struct {
  const int32_t *off, *cols, *len, *table;
  const int64_t *off64;
  int64_t bucket_num;
  int32_t max_len, bucket, hier;
} tc_hash_ctx;

static void tc_hash_body(void *vctx, int64_t lo, int64_t hi, uint64_t *acc) {
  tc_hash_ctx *x = (tc_hash_ctx *)vctx;
  const int32_t *off = x->off, *cols = x->cols;
  for (int64_t wi = lo; wi < hi; wi++) {
    int32_t w = (int32_t)wi;
    uint64_t c = 0;
    for (int32_t e = off[w]; e < off[w + 1]; e++) {
      /* TC.cu:144-157 */
      int32_t u = w, v = cols[e];
      int32_t us = off[u + 1] - off[u], vs = off[v + 1] - off[v];
      if (us > vs) {
        int32_t t = u;
        u = v;
        v = t;
        t = us;
        us = vs;
        vs = t;
      }
      for (int32_t j = 0; j < us; j++)
        c += (uint64_t)ro_probe(cols[off[u] + j], x->table, x->off64[v],
                                x->bucket_num, x->len[v], x->max_len,
                                x->bucket, x->hier);
    }
    *acc += c;
  }
}

uint64_t ro_tc_hash(int32_t n, const int32_t *off, const int32_t *cols,
                    const int32_t *len, const int64_t *off64,
                    const int32_t *table, int64_t bucket_num, int32_t max_len,
                    int32_t bucket, int32_t hier, int32_t nthreads) {
  tc_hash_ctx x = {off, cols, len, table, off64, bucket_num, max_len, bucket,
                   hier};
  return ro_parallel(n, 64, tc_hash_body, &x, nthreads);
}

void ro_sss(int32_t n, const int32_t *off, const int32_t *elems,
            const int32_t *pa, const int32_t *pb, int64_t npairs,
            const int32_t *len, const int64_t *off64, const int32_t *table,
            int64_t bucket_num, int32_t max_len, int32_t bucket, int32_t hier,
            int32_t mode, float thr, int32_t num, int32_t den,
            uint8_t *flags_out, int32_t *inter_out) {
  (void)n;
  for (int64_t p = 0; p < npairs; p++) {
    /* sss.cu:104-136 */
    int32_t u = pa[p], v = pb[p];
    int32_t us = off[u + 1] - off[u], vs = off[v + 1] - off[v];
    if (us > vs) {
      int32_t t = u;
      u = v;
      v = t;
      t = us;
      us = vs;
      vs = t;
    }
    int32_t inter = 0;
    for (int32_t j = 0; j < us; j++)
      inter += ro_probe(elems[off[u] + j], table, off64[v], bucket_num, len[v],
                        max_len, bucket, hier);
    int32_t uni = us + vs - inter;
    int32_t flag;
    if (mode == 0) {
      /* sss.cu:139-140: result_num / (float)(u_size + v_size - result_num) */
      volatile float jac = (float)inter / (float)uni;
      flag = jac >= thr;
    } else {
      flag = uni > 0 && (int64_t)den * inter >= (int64_t)num * uni;
    }
    if (flags_out) flags_out[p] = (uint8_t)flag;
    if (inter_out) inter_out[p] = inter;
  }
}

void ro_ir(int32_t nterms, const int32_t *toff, const int32_t *docs,
           const int32_t *query, const int32_t *qoff, int32_t nq,
           const int64_t *res_off, const int32_t *len, const int64_t *off64,
           const int32_t *table, int64_t bucket_num, int32_t max_len,
           int32_t bucket, int32_t hier, int32_t *result, int32_t *count) {
  (void)nterms;
  for (int32_t q = 0; q < nq; q++) {
    int32_t qs = qoff[q], ql = qoff[q + 1] - qoff[q];
    if (ql <= 0) {
      count[q] = 0;
      continue;
    }
    /* ir.cu:119-128: copy term0's list, then filter in place per term */
    int32_t t0 = query[qs];
    int32_t *r = result + res_off[q];
    int32_t rn = toff[t0 + 1] - toff[t0];
    memcpy(r, docs + toff[t0], sizeof(int32_t) * (size_t)rn);
    for (int32_t i = 1; i < ql; i++) {
      int32_t t = query[qs + i];
      int32_t w = 0;
      for (int32_t j = 0; j < rn; j++) {
        int32_t x = r[j];
        if (ro_probe(x, table, off64[t], bucket_num, len[t], max_len, bucket,
                     hier))
          r[w++] = x;
      }
      rn = w;
    }
    count[q] = rn;
  }
}

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

int64_t ro_pair_count(const int32_t *a, int64_t na, const int32_t *b,
                      int64_t nb) {
  int32_t *sb = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nb > 0 ? nb : 1));
  memcpy(sb, b, sizeof(int32_t) * (size_t)nb);
  qsort(sb, (size_t)nb, sizeof(int32_t), cmp_i32);
  int64_t c = 0;
  for (int64_t i = 0; i < na; i++)
    if (nb > 0 && bsearch(&a[i], sb, (size_t)nb, sizeof(int32_t), cmp_i32))
      c++;
  free(sb);
  return c;
}

/* Brute-force Jaccard self-join over sorted token sets: every pair a < b
 * with |A| + |B| - I > 0 and den * I >= num * (|A| + |B| - I), I by a merge
 * of the two sorted rows.  Writes at most `cap` pairs; returns the number of
 * qualifying pairs (which may exceed cap).  Test-size inputs only
 * (quadratic).  The set-similarity rule of set-similarity-search/sss.cu:
 * 139-141 in its integer form, applied to all pairs. */
int64_t ro_jaccard_join(int32_t n, const int32_t *off, const int32_t *tok,
                        int32_t num, int32_t den, int32_t *pa, int32_t *pb,
                        int64_t cap) {
  int64_t k = 0;
  for (int32_t a = 0; a < n; a++) {
    const int32_t *ra = tok + off[a];
    const int64_t na = off[a + 1] - off[a];
    for (int32_t b = a + 1; b < n; b++) {
      const int32_t *rb = tok + off[b];
      const int64_t nb = off[b + 1] - off[b];
      if (na + nb == 0) continue;
      int64_t i = 0, j = 0, inter = 0;
      while (i < na && j < nb) {
        if (ra[i] < rb[j]) i++;
        else if (ra[i] > rb[j]) j++;
        else { inter++; i++; j++; }
      }
      const int64_t uni = na + nb - inter;
      if ((int64_t)den * inter >= (int64_t)num * uni) {
        if (k < cap) { pa[k] = a; pb[k] = b; }
        k++;
      }
    }
  }
  return k;
}

/* 4-cliques of an oriented graph with sorted rows: for every edge (u, v),
 * W = N+(u) ∩ N+(v) by merging, then for every w in W, |W ∩ N+(w)| by
 * merging (each 4-clique counted once from its two lowest vertices; the
 * multi-way intersections of SMOG/SMOG_hie/subgraph_match_hie.cu:58-247 at
 * depth 4).  Test sizes only. */
uint64_t ro_clique4(int32_t n, const int32_t *off, const int32_t *cols) {
  int32_t maxd = 0;
  for (int32_t u = 0; u < n; u++)
    if (off[u + 1] - off[u] > maxd) maxd = off[u + 1] - off[u];
  int32_t *W = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxd > 0 ? maxd : 1));
  uint64_t total = 0;
  for (int32_t u = 0; u < n; u++) {
    for (int32_t e = off[u]; e < off[u + 1]; e++) {
      const int32_t v = cols[e];
      int32_t i = off[u], j = off[v], nw = 0;
      while (i < off[u + 1] && j < off[v + 1]) {
        if (cols[i] < cols[j]) i++;
        else if (cols[i] > cols[j]) j++;
        else { W[nw++] = cols[i]; i++; j++; }
      }
      for (int32_t t = 0; t < nw; t++) {
        const int32_t w = W[t];
        int32_t a = 0, b = off[w];
        while (a < nw && b < off[w + 1]) {
          if (W[a] < cols[b]) a++;
          else if (W[a] > cols[b]) b++;
          else { total++; a++; b++; }
        }
      }
    }
  }
  free(W);
  return total;
}

/* k-cliques of an oriented graph with sorted rows: the clique search of
 * SMOG's DFSKernelForClique (SMOG/SMOG_hie/subgraph_match_hie.cu:58-247),
 * where the candidates of level l+1 are those of level l intersected with
 * the out-row of the vertex picked at level l (orientation breaks the
 * symmetry, so every clique is counted once).  Depth-first, candidate sets
 * by sorted merge; level 2 starts from every edge (u, v). */
static uint64_t ro_clique_level(const int32_t *off, const int32_t *cols, int32_t *buf,
                                int32_t maxd, const int32_t *C, int32_t nc, int32_t left) {
  /* left: vertices still to pick from C */
  if (left == 1) return (uint64_t)nc;
  uint64_t total = 0;
  int32_t *D = buf;
  for (int32_t t = 0; t < nc; t++) {
    const int32_t w = C[t];
    int32_t a = 0, b = off[w], nd = 0;
    while (a < nc && b < off[w + 1]) {
      if (C[a] < cols[b]) a++;
      else if (C[a] > cols[b]) b++;
      else { D[nd++] = C[a]; a++; b++; }
    }
    total += ro_clique_level(off, cols, buf + maxd, maxd, D, nd, left - 1);
  }
  return total;
}

uint64_t ro_clique_k(int32_t n, const int32_t *off, const int32_t *cols, int32_t k) {
  if (k < 3) return 0;
  int32_t maxd = 1;
  for (int32_t u = 0; u < n; u++)
    if (off[u + 1] - off[u] > maxd) maxd = off[u + 1] - off[u];
  int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)maxd * (size_t)(k - 1));
  uint64_t total = 0;
  for (int32_t u = 0; u < n; u++) {
    for (int32_t e = off[u]; e < off[u + 1]; e++) {
      const int32_t v = cols[e];
      int32_t i = off[u], j = off[v], nw = 0;
      while (i < off[u + 1] && j < off[v + 1]) {
        if (cols[i] < cols[j]) i++;
        else if (cols[i] > cols[j]) j++;
        else { buf[nw++] = cols[i]; i++; j++; }
      }
      total += ro_clique_level(off, cols, buf + maxd, maxd, buf, nw, k - 2);
    }
  }
  free(buf);
  return total;
}

/* Pattern embeddings by definition, for the subgraph matching of SMOG
 * (SMOG/SMOG_hie/subgraph_match_hie.cu:58-406, the pattern encoding of
 * SMOG/SMOG_hie/script_hie.py:85-152): m_0 m_1 run over the stored edges;
 * for l >= 2 the candidates C_l are the keys of the reused level's set
 * (reuse[l] >= 0) or of the FIRST listed vertex's row, kept when every
 * listed vertex's row holds them (binary search); each m_l must pass the
 * level's check, checkRestriction (subgraph_match_hie.cu:23-42).  C_l is
 * stored whole (unfiltered), as a reused set is. */
typedef struct {
  const int32_t *off, *cols, *offsets, *backward, *restriction, *reuse;
  int32_t n, k, flags, maxd;
} ro_pat;

static int ro_row_has(const int32_t *off, const int32_t *cols, int32_t y, int32_t x) {
  int32_t lo = off[y], hi = off[y + 1];
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo) / 2;
    if (cols[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < off[y + 1] && cols[lo] == x;
}

static int ro_pat_ok(const ro_pat *p, int32_t l, int32_t x, const int32_t *map) {
  const int32_t r = p->restriction ? p->restriction[l] : -1;
  if ((p->flags & 2) && r < 0)
    for (int32_t i = 0; i < l; i++)
      if (map[i] == x) return 0;
  if ((p->flags & 1) && r >= 0 && x >= map[r]) return 0;
  return 1;
}

static uint64_t ro_pat_level(const ro_pat *p, int32_t l, int32_t *map, int32_t *buf,
                             int32_t *cnt) {
  const int32_t a = p->offsets[l - 1], z = p->offsets[l];
  const int32_t r = p->reuse ? p->reuse[l] : -1;
  const int32_t *base;
  int32_t nbase;
  if (r >= 0) {
    base = buf + (size_t)r * p->maxd;
    nbase = cnt[r];
  } else {
    int32_t first = -1;
    for (int32_t i = a; i < z && first < 0; i++)
      if (p->backward[i] >= 0) first = map[p->backward[i]];
    base = p->cols + p->off[first];
    nbase = p->off[first + 1] - p->off[first];
  }
  int32_t *C = buf + (size_t)l * p->maxd;
  int32_t nc = 0;
  for (int32_t t = 0; t < nbase; t++) {
    const int32_t x = base[t];
    int keep = 1;
    for (int32_t i = a; i < z && keep; i++)
      if (p->backward[i] >= 0) keep = ro_row_has(p->off, p->cols, map[p->backward[i]], x);
    if (keep) C[nc++] = x;
  }
  cnt[l] = nc;
  uint64_t total = 0;
  for (int32_t t = 0; t < nc; t++) {
    if (!ro_pat_ok(p, l, C[t], map)) continue;
    if (l == p->k - 1) {
      total++;
    } else {
      map[l] = C[t];
      total += ro_pat_level(p, l + 1, map, buf, cnt);
    }
  }
  return total;
}

static void ro_pat_body(void *ctx, int64_t lo, int64_t hi, uint64_t *acc) {
  const ro_pat *p = (const ro_pat *)ctx;
  int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)p->maxd * (size_t)p->k);
  int32_t map[64], cnt[64];
  for (int64_t u = lo; u < hi; u++) {
    for (int32_t e = p->off[u]; e < p->off[u + 1]; e++) {
      map[0] = (int32_t)u;
      map[1] = p->cols[e];
      if (!ro_pat_ok(p, 1, map[1], map)) continue;
      *acc += ro_pat_level(p, 2, map, buf, cnt);
    }
  }
  free(buf);
}

uint64_t ro_pattern_count(int32_t n, const int32_t *off, const int32_t *cols,
                          int32_t k, int32_t flags, const int32_t *offsets,
                          const int32_t *backward, const int32_t *restriction,
                          const int32_t *reuse, int32_t nthreads) {
  if (k < 3 || k > 64 || n <= 0) return 0;
  ro_pat p;
  p.off = off;
  p.cols = cols;
  p.offsets = offsets;
  p.backward = backward;
  p.restriction = restriction;
  p.reuse = reuse;
  p.n = n;
  p.k = k;
  p.flags = flags;
  p.maxd = 1;
  for (int32_t u = 0; u < n; u++)
    if (off[u + 1] - off[u] > p.maxd) p.maxd = off[u + 1] - off[u];
  return ro_parallel(n, 16, ro_pat_body, &p, nthreads);
}

/* ------------------------------------------------------------------------ */
/* synthetic inputs                                                          */
/* ------------------------------------------------------------------------ */

uint64_t ro_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void ro_rmat_thresholds(double a, double b, double c, int32_t *ta,
                        int32_t *tb, int32_t *tc) {
  *ta = (int32_t)(a * 65536.0 + 0.5);
  *tb = (int32_t)((a + b) * 65536.0 + 0.5);
  *tc = (int32_t)((a + b + c) * 65536.0 + 0.5);
}

void ro_rmat_edge(uint64_t seed, int64_t i, int32_t scale, int32_t ta,
                  int32_t tb, int32_t tc, int32_t *pu, int32_t *pv) {
  uint32_t u = 0, v = 0;
  uint64_t w = 0;
  for (int32_t l = 0; l < scale; l++) {
    if ((l & 3) == 0)
      w = ro_mix64(seed ^ ro_mix64((uint64_t)i * 8u + (uint64_t)(l >> 2)));
    int32_t r = (int32_t)((w >> (16 * (l & 3))) & 0xFFFF);
    uint32_t bu, bv;
    if (r < ta) {
      bu = 0;
      bv = 0;
    } else if (r < tb) {
      bu = 0;
      bv = 1;
    } else if (r < tc) {
      bu = 1;
      bv = 0;
    } else {
      bu = 1;
      bv = 1;
    }
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
  *pu = (int32_t)u;
  *pv = (int32_t)v;
}

uint32_t ro_relabel(uint64_t seed, int32_t scale, uint32_t x) {
  uint32_t mask = scale >= 32 ? 0xFFFFFFFFu : ((1u << scale) - 1u);
  int32_t sh = (scale + 1) / 2;
  for (int r = 0; r < 3; r++) {
    uint32_t M = (uint32_t)ro_mix64(seed ^ (0x5EC0DE00ull + 2 * r)) | 1u;
    uint32_t A = (uint32_t)ro_mix64(seed ^ (0x5EC0DE01ull + 2 * r));
    x = (x * M) & mask;
    x ^= x >> sh;
    x = (x + A) & mask;
  }
  return x;
}

static void radix_sort_u64(uint64_t *x, int64_t n) {
  uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
  int64_t cnt[65536];
  for (int pass = 0; pass < 4; pass++) {
    int sh = pass * 16;
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < n; i++) cnt[(x[i] >> sh) & 0xFFFF]++;
    int64_t acc = 0;
    for (int k = 0; k < 65536; k++) {
      int64_t c = cnt[k];
      cnt[k] = acc;
      acc += c;
    }
    for (int64_t i = 0; i < n; i++) tmp[cnt[(x[i] >> sh) & 0xFFFF]++] = x[i];
    memcpy(x, tmp, sizeof(uint64_t) * (size_t)n);
  }
  free(tmp);
}

ro_csr *ro_rmat_graph(int32_t scale, int32_t edge_factor, uint64_t seed,
                      double a, double b, double c, int32_t mode) {
  int32_t n = (int32_t)1 << scale;
  int64_t ne = (int64_t)edge_factor << scale;
  int32_t ta, tb, tc;
  ro_rmat_thresholds(a, b, c, &ta, &tb, &tc);
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(2 * ne + 1));
  int64_t k = 0;
  for (int64_t i = 0; i < ne; i++) {
    int32_t u, v;
    ro_rmat_edge(seed, i, scale, ta, tb, tc, &u, &v);
    if (!(mode & 2)) {
      u = (int32_t)ro_relabel(seed, scale, (uint32_t)u);
      v = (int32_t)ro_relabel(seed, scale, (uint32_t)v);
    }
    if (u == v) continue; /* self-loops removed */
    keys[k++] = ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
    keys[k++] = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
  }
  radix_sort_u64(keys, k);
  int64_t m = 0; /* duplicates removed */
  for (int64_t i = 0; i < k; i++)
    if (i == 0 || keys[i] != keys[i - 1]) keys[m++] = keys[i];
  int32_t *deg = (int32_t *)calloc((size_t)n, sizeof(int32_t));
  for (int64_t i = 0; i < m; i++) deg[keys[i] >> 32]++;
  ro_csr *g = (ro_csr *)malloc(sizeof(ro_csr));
  g->n = n;
  g->off = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
  int64_t w = 0;
  for (int64_t i = 0; i < m; i++) {
    int32_t u = (int32_t)(keys[i] >> 32), v = (int32_t)(keys[i] & 0xFFFFFFFFu);
    int keep = 1;
    if ((mode & 1) == 0) /* orient low degree -> high degree, ties by id */
      keep = deg[u] < deg[v] || (deg[u] == deg[v] && u < v);
    if (keep) {
      keys[w++] = keys[i];
      g->off[u + 1]++;
    }
  }
  for (int32_t u = 0; u < n; u++) g->off[u + 1] += g->off[u];
  g->m = w;
  g->cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(w > 0 ? w : 1));
  for (int64_t i = 0; i < w; i++)
    g->cols[i] = (int32_t)(keys[i] & 0xFFFFFFFFu);
  free(deg);
  free(keys);
  return g;
}

void ro_csr_free(ro_csr *g) {
  if (!g) return;
  free(g->off);
  free(g->cols);
  free(g);
}
