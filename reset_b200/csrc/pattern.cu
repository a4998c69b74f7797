// Pattern counting (subgraph matching) by multi-way hash-probe
// intersections: SMOG's DFSKernelForGeneral and DFSKernelForClique
// (SMOG/SMOG_hie/subgraph_match_hie.cu:58-406) over this library's tables,
// for any pattern in SMOG's encoding (reset_pattern in reset.h).
//
// One warp per start edge (dynamic 1-edge work items, as the clique
// kernels).  The edge fixes m_0 and m_1.  Level l >= 2 builds its
// candidate set C_l in one pass: the base is the reused level's set or the
// shortest row among the listed backward vertices; every base key is probed
// into the tables of the other listed rows (early exit per lane), and the
// hits are compacted into the warp's scratch row of level l (ballot/popc).
// A level with nothing to probe keeps a view of its base, without a copy.
// The last level is only counted; earlier levels are walked 32 candidates
// at a time, the next m_l being the first lane's key that passes the
// level's check.  Where no later level reuses C_l, keys failing l's check
// are dropped at compaction already.  The reference instead builds C_l by
// one pass per listed row, and walks candidates one by one.
//
// With strictly ascending rows (checked on the device in the same pass that
// finds the longest row), a restriction m_l < m_r cuts the base to its
// prefix below m_r before any probe, and a last level with nothing to probe
// is counted without a scan: the prefix length, or |C_l| less the earlier
// vertices that a binary search finds in it.  Such a last level is not
// entered at all: the level before it hands one candidate to each lane,
// which counts the last level for it.  A last level that intersects a fixed
// vertex's row with the row of the candidate just picked (N(m_a) ∩ N(x))
// is not entered either: such intersections of at most kLaneMax keys run
// one candidate per lane, longer ones by the whole warp.  A reusing
// k-clique chain without checks (SMOG's Q0, Q3, Q5, Q7) runs the k-clique
// kernel (clique.cu).
//
// Semantics differ from the reference in one case only: where two listed
// vertices of a level map to the same data vertex and that vertex has the
// shortest row, the reference skips both (its count then reads scratch left
// from an earlier edge); here N(x) ∩ N(x) = N(x).  No pattern of the
// reference's table reaches that case: in each, an edge, the distinctness
// check or a restriction separates the two vertices.
#include <algorithm>
#include <cstring>

#include "probe_common.cuh"

namespace rst {
namespace {

constexpr int kPatMax = RESET_PATTERN_MAX;
constexpr int kPtThreads = 256;
constexpr int kPtWarps = kPtThreads / 32;
// Scratch rows of all resident warps together stay below this; a graph
// whose largest row would need more runs fewer warps.
constexpr size_t kPtScratchBudget = size_t(1) << 30;

struct PatternDev {
  int32_t k, flags;
  int32_t restr[kPatMax];          // restriction[l], -1 = none
  int32_t reuse[kPatMax];          // reused level, -1 = none
  int32_t nb[kPatMax];             // listed backward vertices of level l
  int32_t back[kPatMax][kPatMax];  // ... their pattern indices (no -1)
  int32_t filt[kPatMax];           // 1: no later level reuses C_l
  int32_t chain;                   // a reusing clique chain without checks
  int32_t fuse;                    // the last level probes nothing
  int32_t pair;                    // the last level lists {pair_a, k-2} only
  int32_t pair_a;
};

// Intersections of the paired last level up to this length run one per
// lane; longer ones take the whole warp.
constexpr int kLaneMax = 32;

// checkRestriction (SMOG/SMOG_hie/subgraph_match_hie.cu:23-42) with the
// opposite sense: true when key x may be m_l.
__device__ __forceinline__ bool level_ok(const PatternDev& p, int l, int x, const int* map) {
  const int r = p.restr[l];
  if ((p.flags & RESET_PATTERN_DISTINCT) && r < 0)
    for (int i = 0; i < l; ++i)
      if (map[i] == x) return false;
  if ((p.flags & RESET_PATTERN_RESTRICT) && r >= 0 && x >= map[r]) return false;
  return true;
}

// First index of a[0 .. n) whose key is >= x (a ascending); plain loads,
// `a` may be the calling warp's scratch.
__device__ __forceinline__ int lower_bound_key(const int32_t* a, int n, int x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// One pass over a CSR: out[0] = the longest row (atomicMax), out[1] =
// adjacent key pairs in descending-or-equal order, out[2] = those pairs
// that straddle a row boundary.  Every row is strictly ascending exactly
// when out[1] == out[2].
__global__ void row_stats_kernel(const int32_t* __restrict__ off,
                                 const int32_t* __restrict__ cols, int32_t n, int64_t m,
                                 unsigned long long* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int mx = 0;
  unsigned long long desc_pairs = 0, edges = 0;
  for (int64_t i = t0; i < n; i += stride) {
    const int a = __ldg(off + i), z = __ldg(off + i + 1);
    mx = max(mx, z - a);
    if (z > a && z < m) edges += __ldg(cols + z - 1) >= __ldg(cols + z);
  }
  for (int64_t e = t0; e + 1 < m; e += stride)
    desc_pairs += __ldg(cols + e) >= __ldg(cols + e + 1);
  for (int o = 16; o; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    desc_pairs += __shfl_xor_sync(kFull, desc_pairs, o);
    edges += __shfl_xor_sync(kFull, edges, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)mx);
    if (desc_pairs) atomicAdd(out + 1, desc_pairs);
    if (edges) atomicAdd(out + 2, edges);
  }
}

template <bool HIER>
__global__ void __launch_bounds__(kPtThreads, 5)
    pattern_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ off,
                   const int32_t* __restrict__ cols, const int32_t* __restrict__ chunk_row,
                   int32_t n, int64_t m, const int32_t* __restrict__ table, int64_t bn, int b,
                   int lg_max, const PatternDev pat, int sorted,
                   int32_t* __restrict__ scratch, int32_t cap,
                   unsigned long long* __restrict__ count,
                   unsigned long long* __restrict__ cursor, int32_t* __restrict__ status) {
  __shared__ PatternDev sp;
  if (threadIdx.x == 0) sp = pat;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int k = sp.k;
  const int rows = k > 3 ? k - 3 : 1;
  int32_t* Sbase = scratch + gw * (int64_t)cap * rows;
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  unsigned long long hits = 0;
  int map[kPatMax], sz[kPatMax], it[kPatMax];
  const int32_t* cs[kPatMax];
  int4 pd[kPatMax];
  int u = 0;
  for (;;) {
    unsigned long long cc = 0;
    if (lane == 0) cc = atomicAdd(cursor, 1ull);
    const int64_t e = (int64_t)__shfl_sync(kFull, cc, 0);
    if (e >= me) break;
    if (lane == 0) {  // row of edge e: largest u with off[u] <= e
      const int64_t c = e >> 5;
      int lo = __ldg(chunk_row + c);
      int hi = c + 1 < n_chunks ? __ldg(chunk_row + c + 1) : n - 1;
      if ((unsigned)lo >= (unsigned)n) lo = 0;
      if (hi < lo || hi >= n) hi = n - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= e) lo = mid; else hi = mid - 1;
      }
      u = lo;
    }
    u = __shfl_sync(kFull, u, 0);
    const int v = __ldg(cols + e);
    if ((unsigned)v >= (unsigned)n) {
      if (lane == 0) atomicOr(status, kErrBadId);
      continue;
    }
    map[0] = u;
    map[1] = v;
    if (!level_ok(sp, 1, v, map)) continue;
    int lv = 2;  // warp-uniform depth
    bool build = true;
    while (lv >= 2) {
      if (build) {
        build = false;
        // the base of C_lv: the reused set, or the shortest listed row
        const int32_t* src = cols;
        int ns = 0, bv = -1;
        const int r = sp.reuse[lv];
        if (r >= 0) {
          src = cs[r];
          ns = sz[r];
        } else {
          ns = INT_MAX;
          for (int j = 0; j < sp.nb[lv]; ++j) {
            const int y = map[sp.back[lv][j]];
            const int4 dy = __ldg(desc + y);
            if (dy.y < ns) {
              ns = dy.y;
              bv = y;
              src = cols + dy.x;
            }
          }
        }
        // the other listed rows, each once, are probed
        int np = 0;
        for (int j = 0; j < sp.nb[lv]; ++j) {
          const int y = map[sp.back[lv][j]];
          if (y == bv) continue;
          bool seen = false;
          for (int q = 0; q < j; ++q) seen |= map[sp.back[lv][q]] == y;
          if (seen) continue;
          const int4 dy = __ldg(desc + y);
          if (dy.y == 0) ns = 0;
          pd[np++] = dy;
        }
        const bool last = lv == k - 1;
        const int rr = sp.restr[lv];
        // ascending rows: the keys a restriction m_lv < m_rr admits are a
        // prefix of the base (cut only where no later level reuses C_lv)
        if (sorted && (sp.flags & RESET_PATTERN_RESTRICT) && rr >= 0 && (last || sp.filt[lv]))
          ns = lower_bound_key(src, ns, map[rr]);
        if (last && np == 0 && sorted) {
          // C_lv is the base itself: |C_lv| less the earlier vertices in it
          int c = ns;
          if ((sp.flags & RESET_PATTERN_DISTINCT) && rr < 0)
            for (int i = 0; i < lv; ++i) {
              const int y = map[i];
              bool seen = false;
              for (int q = 0; q < i; ++q) seen |= map[q] == y;
              if (seen) continue;
              const int at = lower_bound_key(src, ns, y);
              if (at < ns && src[at] == y) --c;
            }
          if (lane == 0) hits += c;
          --lv;
          continue;
        }
        if (np == 0 && !last) {  // a view of the base
          cs[lv] = src;
          sz[lv] = ns;
          it[lv] = 0;
        } else {
          int32_t* dst = Sbase + (int64_t)(lv - 2) * cap;
          const bool chk = last || sp.filt[lv];
          int nw = 0;
          for (int j0 = 0; j0 < ns; j0 += 32) {
            const int j = j0 + lane;
            bool in = false;
            int x = 0;
            if (j < ns) {
              x = src[j];  // plain load: src may be this warp's scratch
              in = !chk || level_ok(sp, lv, x, map);
              for (int q = 0; in && q < np; ++q)
                in = probe_key<HIER>(x, table + desc_toff(pd[q]), desc_lg(pd[q]), lg_max, bn, b,
                                     status);
            }
            if (last) {
              hits += in;
            } else {
              const unsigned msk = __ballot_sync(kFull, in);
              if (in) {
                const int pos = nw + __popc(msk & lt);
                if (pos < cap) dst[pos] = x;
              }
              nw += __popc(msk);
            }
          }
          if (!last) {
            if (nw > cap) {  // cannot happen: no set outgrows the longest row
              if (lane == 0) atomicOr(status, kErrProbeLimit);
              nw = cap;
            }
            __syncwarp();
            cs[lv] = dst;
            sz[lv] = nw;
            it[lv] = 0;
          }
        }
        if (last) {
          --lv;
          continue;
        }
      }
      if (sp.pair && lv == k - 2) {
        // the last level is N(m_a) ∩ N(x) for the candidate x: short
        // intersections run one candidate per lane (each lane holds its own
        // m_lv = x in its copy of map), long ones afterwards by the warp
        const int L = k - 1, rr = sp.restr[L];
        const bool rcut = sorted && (sp.flags & RESET_PATTERN_RESTRICT) && rr >= 0;
        const int4 da = __ldg(desc + map[sp.pair_a]);
        for (int j0 = it[lv]; j0 < sz[lv]; j0 += 32) {
          const int j = j0 + lane;
          int x = j < sz[lv] ? cs[lv][j] : 0;
          bool act = j < sz[lv];
          if (act && (unsigned)x >= (unsigned)n) {
            atomicOr(status, kErrBadId);
            act = false;
          }
          act = act && level_ok(sp, lv, x, map);
          int len = 0;
          const int32_t* base = cols;
          const int32_t* tb = table;
          int tlg = 0;
          if (act) {
            const int4 dx = __ldg(desc + x);
            const int4 db = dx.y <= da.y ? dx : da, dt = dx.y <= da.y ? da : dx;
            base = cols + db.x;
            len = dt.y > 0 ? db.y : 0;
            tb = table + desc_toff(dt);
            tlg = desc_lg(dt);
            if (rcut) len = lower_bound_key(base, len, rr == lv ? x : map[rr]);
          }
          const bool big = len > kLaneMax;
          if (!big && len > 0) {
            map[lv] = x;
            unsigned long long c = 0;
            for (int t = 0; t < len; ++t) {
              const int z = base[t];
              c += level_ok(sp, L, z, map) && probe_key<HIER>(z, tb, tlg, lg_max, bn, b, status);
            }
            hits += c;
          }
          for (unsigned bm = __ballot_sync(kFull, big); bm; bm &= bm - 1) {
            const int f = __ffs(bm) - 1;
            const int xb = __shfl_sync(kFull, x, f);
            const int lb = __shfl_sync(kFull, len, f);
            const int32_t* bb = cols + __shfl_sync(kFull, (int)(base - cols), f);
            const int4 dx = __ldg(desc + xb);
            const int4 dt = dx.y <= da.y ? da : dx;
            map[lv] = xb;
            for (int t = lane; t < lb; t += 32) {
              const int z = bb[t];
              hits += level_ok(sp, L, z, map) &&
                      probe_key<HIER>(z, table + desc_toff(dt), desc_lg(dt), lg_max, bn, b, status);
            }
          }
        }
        --lv;
        continue;
      }
      if (sorted && sp.fuse && lv == k - 2) {
        // the last level probes nothing: every key x of C_lv that passes
        // lv's check is m_lv for one lane, which counts the last level's
        // keys for it at once (prefix below the restriction bound, less
        // the earlier vertices found in the base), without building it
        const int L = k - 1, rr = sp.restr[L], ru = sp.reuse[L];
        const bool rcut = (sp.flags & RESET_PATTERN_RESTRICT) && rr >= 0;
        const bool dist = (sp.flags & RESET_PATTERN_DISTINCT) && rr < 0;
        for (int j = it[lv] + lane; j < sz[lv]; j += 32) {
          const int x = cs[lv][j];
          if ((unsigned)x >= (unsigned)n) {
            atomicOr(status, kErrBadId);
            continue;
          }
          if (!level_ok(sp, lv, x, map)) continue;
          const int32_t* base;
          int nbase;
          if (ru >= 0) {
            base = cs[ru];
            nbase = sz[ru];
          } else {
            const int lj = sp.back[L][0];
            const int4 dy = __ldg(desc + (lj == lv ? x : map[lj]));
            base = cols + dy.x;
            nbase = dy.y;
          }
          if (rcut) nbase = lower_bound_key(base, nbase, rr == lv ? x : map[rr]);
          int c = nbase;
          if (dist)
            for (int i = 0; i <= lv; ++i) {
              const int y = i == lv ? x : map[i];
              bool seen = false;
              for (int q = 0; q < i; ++q) seen |= map[q] == y;
              if (seen) continue;
              const int at = lower_bound_key(base, nbase, y);
              if (at < nbase && base[at] == y) --c;
            }
          hits += c;
        }
        --lv;
        continue;
      }
      // the next key of C_lv that passes the level's check becomes m_lv
      int x = -1;
      while (it[lv] < sz[lv]) {
        const int j = it[lv] + lane;
        const int y = j < sz[lv] ? cs[lv][j] : 0;
        const bool bad = j < sz[lv] && (unsigned)y >= (unsigned)n;
        if (bad) atomicOr(status, kErrBadId);
        const bool ok = j < sz[lv] && !bad && level_ok(sp, lv, y, map);
        const unsigned msk = __ballot_sync(kFull, ok);
        if (msk) {
          const int f = __ffs(msk) - 1;
          x = __shfl_sync(kFull, y, f);
          it[lv] += f + 1;
          break;
        }
        it[lv] += 32;
      }
      if (x < 0) {
        --lv;
        continue;
      }
      map[lv] = x;
      ++lv;
      build = true;
    }
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

// Checks a pattern and lays it out for the kernel.
reset_status compile_pattern(const reset_pattern* p, PatternDev* d) {
  if (!p) return arg_fail("NULL pattern");
  const int k = p->k;
  if (k < 3 || k > kPatMax) return arg_fail("pattern k must be in 3..RESET_PATTERN_MAX");
  if (p->flags & ~(RESET_PATTERN_RESTRICT | RESET_PATTERN_DISTINCT))
    return arg_fail("unknown pattern flags");
  if (!p->offsets || !p->backward) return arg_fail("NULL pattern offsets or backward");
  if (p->offsets[0] != 0 || p->offsets[1] != 1 || p->backward[0] != 0)
    return arg_fail("pattern level 1 must list exactly vertex 0");
  std::memset(d, 0, sizeof(*d));
  d->k = k;
  d->flags = p->flags;
  for (int l = 0; l < k; ++l) {
    d->restr[l] = p->restriction ? p->restriction[l] : -1;
    d->reuse[l] = p->reuse ? p->reuse[l] : -1;
    d->filt[l] = 1;
  }
  if (d->restr[0] != -1) return arg_fail("restriction[0] must be -1");
  for (int l = 1; l < k; ++l)
    if (d->restr[l] < -1 || d->restr[l] >= l)
      return arg_fail("restriction[l] must be -1 or an earlier vertex");
  for (int l = 0; l < k; ++l) {
    const int r = d->reuse[l];
    if (r == -1) continue;
    if (l < 3 || r < 2 || r >= l) return arg_fail("reuse[l] must be -1 or a level in [2, l)");
    d->filt[r] = 0;
  }
  for (int l = 2; l < k; ++l) {
    const int a = p->offsets[l - 1], z = p->offsets[l];
    if (z < a || z - a > kPatMax) return arg_fail("pattern offsets must rise by at most RESET_PATTERN_MAX");
    int minus = 0, nb = 0;
    for (int i = a; i < z; ++i) {
      const int j = p->backward[i];
      if (j == -1) {
        ++minus;
        continue;
      }
      if (j < 0 || j >= l) return arg_fail("backward entries must be -1 or earlier vertices");
      d->back[l][nb++] = j;
    }
    if (minus != (d->reuse[l] >= 0 ? 1 : 0))
      return arg_fail("a reusing level lists exactly one -1, other levels none");
    if (nb == 0 && d->reuse[l] < 0)
      return arg_fail("every level needs a listed vertex or a reused set");
    d->nb[l] = nb;
  }
  // The reusing k-clique chain (SMOG's Q0, Q3, Q5, Q7): level 2 lists
  // {0, 1}, every later level l reuses l-1 and lists l-1; with no active
  // check its count is the k-clique search's.
  bool checks = (d->flags & RESET_PATTERN_DISTINCT) != 0;
  for (int l = 1; l < k; ++l) checks |= (d->flags & RESET_PATTERN_RESTRICT) && d->restr[l] >= 0;
  bool chain = !checks && d->nb[2] == 2 && d->reuse[2] < 0 &&
               ((d->back[2][0] == 0 && d->back[2][1] == 1) || (d->back[2][0] == 1 && d->back[2][1] == 0));
  for (int l = 3; l < k && chain; ++l)
    chain = d->reuse[l] == l - 1 && d->nb[l] == 1 && d->back[l][0] == l - 1;
  d->chain = chain ? 1 : 0;
  d->fuse = k >= 4 && ((d->reuse[k - 1] >= 0 && d->nb[k - 1] == 0) ||
                       (d->reuse[k - 1] < 0 && d->nb[k - 1] == 1));
  d->pair = 0;
  if (k >= 4 && d->reuse[k - 1] < 0 && d->nb[k - 1] == 2) {
    const int a = d->back[k - 1][0], c = d->back[k - 1][1];
    if ((a == k - 2) != (c == k - 2)) {
      d->pair = 1;
      d->pair_a = a == k - 2 ? c : a;
    }
  }
  return RESET_OK;
}

// SMOG's query patterns (SMOG/SMOG_hie/script_hie.py:85-152) and the graph
// each is counted on (SMOG/SMOG_hie/common_hie.cu:72-85).
struct NamedPattern {
  const char* name;
  int32_t k, flags, oriented;
  int32_t offsets[kPatMax], backward[2 * kPatMax], restriction[kPatMax], reuse[kPatMax];
  bool has_restriction, has_reuse;
};

constexpr int32_t kRD = RESET_PATTERN_RESTRICT | RESET_PATTERN_DISTINCT;
const NamedPattern kNamed[] = {
    {"Q0", 3, 0, 1, {0, 1, 3}, {0, 0, 1}, {}, {}, false, false},
    {"Q1", 4, RESET_PATTERN_RESTRICT, 0, {0, 1, 2, 4}, {0, 0, 1, 2}, {-1, 0, 1, 0}, {},
     true, false},
    {"Q2", 4, RESET_PATTERN_RESTRICT, 0, {0, 1, 3, 5}, {0, 0, 1, 1, 2}, {-1, -1, 1, 0}, {},
     true, false},
    {"Q3", 4, 0, 1, {0, 1, 3, 5}, {0, 0, 1, -1, 2}, {}, {-1, -1, -1, 2}, false, true},
    {"Q4", 5, kRD, 0, {0, 1, 3, 5, 6}, {0, 0, 1, -1, 2, -1}, {-1, 0, -1, 2, -1},
     {-1, -1, -1, 2, 2}, true, true},
    {"Q5", 5, 0, 1, {0, 1, 3, 5, 7}, {0, 0, 1, -1, 2, -1, 3}, {}, {-1, -1, -1, 2, 3}, false,
     true},
    {"Q6", 5, kRD, 0, {0, 1, 3, 4, 6}, {0, 0, 1, -1, 2, 3}, {-1, 0, -1, 2, -1},
     {-1, -1, -1, 2, -1}, true, true},
    {"Q7", 6, 0, 1, {0, 1, 3, 5, 7, 9}, {0, 0, 1, -1, 2, -1, 3, -1, 4}, {},
     {-1, -1, -1, 2, 3, 4}, false, true},
    {"Q8", 5, RESET_PATTERN_RESTRICT, 0, {0, 1, 3, 5, 6}, {0, 0, 1, -1, 2, -1},
     {-1, 0, -1, -1, 3}, {-1, -1, -1, 2, 3}, true, true},
};

}  // namespace
}  // namespace rst

using namespace rst;

extern "C" reset_status reset_pattern_named(const char* name, reset_pattern* out,
                                            int32_t* oriented) {
  if (!name || !out) return arg_fail("NULL name or pattern");
  for (const NamedPattern& q : kNamed) {
    if (std::strcmp(q.name, name) != 0) continue;
    out->k = q.k;
    out->flags = q.flags;
    out->offsets = q.offsets;
    out->backward = q.backward;
    out->restriction = q.has_restriction ? q.restriction : nullptr;
    out->reuse = q.has_reuse ? q.reuse : nullptr;
    if (oriented) *oriented = q.oriented;
    return RESET_OK;
  }
  return arg_fail("unknown pattern name (SMOG's table has Q0..Q8)");
}

extern "C" reset_status reset_pattern_count(const reset_table* t, const int32_t* d_off,
                                            const int32_t* d_cols, int64_t m,
                                            const reset_pattern* p, uint64_t* d_count,
                                            reset_stream_t stream) {
  if (!t || !d_count) return arg_fail("NULL table or count");
  PatternDev pat;
  {
    const reset_status s = compile_pattern(p, &pat);
    if (s != RESET_OK) return s;
  }
  if (m < 0 || m > INT32_MAX) return arg_fail("m out of range");
  if (m > 0 && (!d_off || !d_cols)) return arg_fail("NULL offsets or cols");
  if (d_off != t->build_off || m != t->m)
    return arg_fail("d_off/m must be the CSR the table was built on");
  if (pat.chain) return reset_clique_count(t, d_off, d_cols, m, pat.k, d_count, stream);
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m == 0 || t->n == 0) return RESET_OK;
  unsigned long long stats[3] = {0, 0, 0};
  {
    unsigned long long* d_st = nullptr;
    RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_st), sizeof(stats), st));
    cudaError_t e = cudaMemsetAsync(d_st, 0, sizeof(stats), st);
    if (e == cudaSuccess) {
      note_launch();
      row_stats_kernel<<<sm_count() * 4, 256, 0, st>>>(d_off, d_cols, t->n, m, d_st);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(stats, d_st, sizeof(stats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(d_st, st);
    if (e != cudaSuccess) return cuda_fail(e, "row stats", __FILE__, __LINE__);
  }
  const int32_t cap = stats[0] > 0 ? (int32_t)stats[0] : 1;
  const int sorted = stats[1] == stats[2] ? 1 : 0;
  const int64_t rows = pat.k > 3 ? pat.k - 3 : 1;
  const void* kf = t->hier ? (const void*)pattern_kernel<true> : (const void*)pattern_kernel<false>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, kPtThreads, 0);
  if (per_sm < 1) per_sm = 1;
  const size_t per_block = sizeof(int32_t) * (size_t)cap * (size_t)rows * kPtWarps;
  const int64_t fit = std::max<int64_t>(1, (int64_t)(kPtScratchBudget / per_block));
  const int64_t grid = std::min<int64_t>(std::min<int64_t>((int64_t)sm_count() * per_sm, fit),
                                         (m + kPtWarps - 1) / kPtWarps);
  int32_t* d_scr = nullptr;
  unsigned long long* d_cur = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_scr), per_block * (size_t)grid, st));
  cudaError_t e = scratch_malloc(reinterpret_cast<void**>(&d_cur), sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_cur, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    note_launch();
    if (t->hier)
      pattern_kernel<true><<<(int)grid, kPtThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num,
          t->bucket, t->lg_max, pat, sorted, d_scr, cap, reinterpret_cast<unsigned long long*>(d_count),
          d_cur, t->d_status);
    else
      pattern_kernel<false><<<(int)grid, kPtThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num,
          t->bucket, t->lg_max, pat, sorted, d_scr, cap, reinterpret_cast<unsigned long long*>(d_count),
          d_cur, t->d_status);
    e = cudaGetLastError();
  }
  cudaFreeAsync(d_scr, st);
  if (d_cur) cudaFreeAsync(d_cur, st);
  if (e != cudaSuccess) return cuda_fail(e, "pattern_kernel", __FILE__, __LINE__);
  return RESET_OK;
}
