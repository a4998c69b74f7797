// Device helpers shared by the probe kernels.
#pragma once

#include <climits>

#include "common.cuh"

namespace rst {

// Row of edge e (warp-collective).  u0 is the row of the chunk's first edge;
// row(e) = u0 + #{j : off[u0+1+j] <= e}, searched 32 rows at a time.
__device__ __forceinline__ int row_of_edge(const int32_t* __restrict__ off,
                                           int n, int u0, int e) {
  const int lane = threadIdx.x & 31;
  int row = -1;
  for (int ub = u0;; ub += 32) {
    const int idx = ub + 1 + lane;
    const int q = idx <= n ? __ldg(off + idx) : INT_MAX;
    int c = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      int qq = __shfl_sync(kFull, q, c + step - 1);
      if (qq <= e) c += step;
    }
    const int q31 = __shfl_sync(kFull, q, 31);
    if (c == 31 && q31 <= e) c = 32;
    if (row < 0 && c < 32) row = ub + c;
    if (__all_sync(kFull, row >= 0)) break;
  }
  return row;
}

// search_in_hashtable (triangle-count/TC.cu:11-31): walk the slots of the
// home bucket, then the next bucket (mod len); equal slot = hit, -1 = miss.
// Bounded by the table size (a full table raises kErrProbeLimit).
template <bool HIER>
__device__ __forceinline__ bool probe_key(int x, const int32_t* __restrict__ tb,
                                          int lg, int lg_max, int64_t bn,
                                          int b, int32_t* status) {
  const int l = 1 << lg;
  int h = home_bucket<HIER>(x, lg, lg_max);
  int k = 0;
  const int64_t cap = (int64_t)l * b;
  for (int64_t t = 0; t < cap; ++t) {
    const int s = __ldg(tb + h + (int64_t)k * bn);
    if (s == x) return true;
    if (s == -1) return false;
    if (++k == b) {
      k = 0;
      h = (h + 1) & (l - 1);
    }
  }
  atomicOr(status, kErrProbeLimit);
  return false;
}

// Continues a probe from slot k of bucket h (slots before it held other
// keys).  Same rule and bound as probe_key.
template <bool HIER>
__device__ __forceinline__ bool probe_rest(int x, const int32_t* __restrict__ tb,
                                           int lg, int h, int k, int64_t bn,
                                           int b, int32_t* status) {
  const int l = 1 << lg;
  if (k == b) {
    k = 0;
    h = (h + 1) & (l - 1);
  }
  // walk with a running slot pointer (one multiply up front)
  const int32_t* __restrict__ p = tb + h + (int64_t)k * bn;
  const int64_t cap = (int64_t)l * b;
  for (int64_t t = 1; t < cap; ++t) {
    const int s = __ldg(p);
    if (s == x) return true;
    if (s == -1) return false;
    if (++k == b) {
      k = 0;
      h = (h + 1) & (l - 1);
      p = tb + h;
    } else {
      p += bn;
    }
  }
  atomicOr(status, kErrProbeLimit);
  return false;
}

// Queue walk: continues a probe from slot k of bucket h with a running slot
// pointer and a 32-bit step count; walks longer than 64 slots (a crowded
// region) finish in probe_rest.  Same answer as probe_rest.
template <bool HIER>
__device__ __forceinline__ bool probe_walk(int x, const int32_t* __restrict__ tb,
                                           int lg, int h, int k, int64_t bn, int b,
                                           int32_t* status) {
  const int lmask = (1 << lg) - 1;
  if (k == b) {
    k = 0;
    h = (h + 1) & lmask;
  }
  const int32_t* __restrict__ p = tb + h + (int64_t)k * bn;
#pragma unroll 1
  for (int t = 0; t < 64; ++t) {
    const int s = __ldg(p);
    if (s == x) return true;
    if (s == -1) return false;
    if (++k == b) {
      k = 0;
      h = (h + 1) & lmask;
      p = tb + h;
    } else {
      p += bn;
    }
  }
  return probe_rest<HIER>(x, tb, lg, h, k, bn, b, status);
}

// Warp-inclusive scan; returns the exclusive prefix and sets *total.
__device__ __forceinline__ int warp_excl_scan(int s, int* total) {
  const int lane = threadIdx.x & 31;
  int incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  *total = __shfl_sync(kFull, incl, 31);
  return incl - s;
}

// Largest lane k with P_k <= f (P nondecreasing across lanes, P_0 = 0).
__device__ __forceinline__ int owner_lane(int P, int f) {
  int k = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    int pk = __shfl_sync(kFull, P, k + step);
    if (pk <= f) k += step;
  }
  return k;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return v;
}

// Resolves a probe whose first two slots (k = 0, 1 of the home bucket) are
// already loaded; walks further only when both held other keys.
template <bool HIER>
__device__ __forceinline__ bool probe_resolve2(int x, int s0, int s1,
                                               const int32_t* __restrict__ tb,
                                               int lg, int h, int64_t bn, int b,
                                               int32_t* status) {
  if (s0 == x) return true;
  if (s0 == -1) return false;
  if (b == 1) return probe_rest<HIER>(x, tb, lg, h, 1, bn, b, status);
  if (s1 == x) return true;
  if (s1 == -1) return false;
  return probe_rest<HIER>(x, tb, lg, h, 2, bn, b, status);
}

// One pair probed by the whole warp: keys[0 .. s) into the table tb, lane i
// taking keys i, i+32, ... in batches of kWarpRounds rounds.  Software
// pipelined: the next batch's keys are loaded while this batch's slot-0/1
// loads are in flight.  Probes whose two first slots hold other keys are
// compacted into the warp's shared-memory queue (qx/qh, 32*kWarpRounds
// entries) and walked together after the batch, so the divergent tail runs
// once per batch.  Rounds past the end of the pair are skipped (warp-uniform).
// Returns this lane's hits.
constexpr int kWarpRoundsMax = 4;

template <bool HIER, int kWarpRounds>
__device__ __forceinline__ int warp_probe_pair(const int32_t* __restrict__ keys,
                                               int s,
                                               const int32_t* __restrict__ tb,
                                               int lg, int lg_max, int64_t bn,
                                               int b, int32_t* status,
                                               int* qx, int* qh) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t bn1 = b > 1 ? bn : 0;
  int hits = 0;
  int xn[kWarpRounds];
#pragma unroll
  for (int r = 0; r < kWarpRounds; ++r) {
    const int j = r * 32 + lane;
    xn[r] = j < s ? __ldg(keys + j) : -1;
  }
  for (int j0 = 0; j0 < s; j0 += 32 * kWarpRounds) {
    int x[kWarpRounds], h[kWarpRounds], s0[kWarpRounds], s1[kWarpRounds];
#pragma unroll
    for (int r = 0; r < kWarpRounds; ++r) {
      x[r] = xn[r];
      h[r] = home_bucket<HIER>(x[r], lg, lg_max);
      s0[r] = s1[r] = -1;
      if (j0 + r * 32 < s) {  // warp-uniform
        if (j0 + r * 32 + lane < s) {
          s0[r] = __ldg(tb + h[r]);
          s1[r] = __ldg(tb + h[r] + bn1);
        }
      }
    }
    const int jn = j0 + 32 * kWarpRounds;
#pragma unroll
    for (int r = 0; r < kWarpRounds; ++r) {
      const int j = jn + r * 32 + lane;
      xn[r] = j < s ? __ldg(keys + j) : -1;
    }
    int nq = 0;
#pragma unroll
    for (int r = 0; r < kWarpRounds; ++r) {
      if (j0 + r * 32 >= s) continue;  // warp-uniform
      const bool act = j0 + r * 32 + lane < s;
      bool pend = false;
      if (act) {
        if (s0[r] == x[r]) {
          ++hits;
        } else if (s0[r] != -1) {
          if (b == 1) {
            pend = true;
          } else if (s1[r] == x[r]) {
            ++hits;
          } else if (s1[r] != -1) {
            pend = true;
          }
        }
      }
      const unsigned pm = __ballot_sync(kFull, pend);
      if (pend) {
        const int pos = nq + __popc(pm & lt);
        qx[pos] = x[r];
        qh[pos] = h[r];
      }
      nq += __popc(pm);
    }
    if (nq) {
      __syncwarp();
      const int k0 = b == 1 ? 1 : 2;
      for (int i = lane; i < nq; i += 32)
        hits += probe_rest<HIER>(qx[i], tb, lg, qh[i], k0, bn, b, status);
      __syncwarp();
    }
  }
  return hits;
}

// Lean whole-warp pair loop: R rounds of 32 keys per batch; per round a key
// load, the home bucket, loads of slots 0 and 1 (independent), and a
// branch-free resolve; probes that both slots leave open go to the warp's
// shared-memory queue (qx/qh, 32*R entries), walked together after the
// batch.  No prefetch across batches: latency is hidden by the other
// resident warps.  Returns this lane's hits.
//
// EARLY (decisions only): after every batch the warp totals its hits and
// stops once they reach need_hits or once its misses exceed max_miss; the
// partial total then decides a threshold rule exactly as the full one would.
template <bool HIER, int R, bool EARLY = false>
__device__ __forceinline__ int warp_probe_pair_lean(const int32_t* __restrict__ keys,
                                                    int s,
                                                    const int32_t* __restrict__ tb,
                                                    int lg, int lg_max, int64_t bn,
                                                    int b, int32_t* status,
                                                    int* qx, int* qh,
                                                    int need_hits = 0, int max_miss = 0) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int32_t* __restrict__ tb1 = tb + (b > 1 ? bn : 0);
  const unsigned hmask = HIER ? ((1u << lg_max) - 1u) : ((1u << lg) - 1u);
  const int hsh = HIER ? (lg_max - lg) : 0;
  const int k0 = b == 1 ? 1 : 2;  // where queued probes continue
  int hits = 0;
  for (int base = 0; base < s; base += 32 * R) {
    const int nr = min(R, (s - base + 31) >> 5);  // rounds with keys (warp-uniform)
    int x[R], h[R], s0[R], s1[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = base + r * 32 + lane;
      x[r] = -2;
      if (r < nr && j < s) x[r] = __ldg(keys + j);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      h[r] = (int)(((unsigned)x[r] & hmask) >> hsh);
      s0[r] = -1;
      s1[r] = -1;
      if (r < nr && x[r] >= 0) {
        s0[r] = __ldg(tb + h[r]);
        s1[r] = __ldg(tb1 + h[r]);
      }
    }
    int nq = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (r >= nr) break;
      const bool e0 = s0[r] == -1, m0 = s0[r] == x[r];
      const bool e1 = s1[r] == -1, m1 = s1[r] == x[r];
      hits += (int)(m0 | (!e0 & m1));
      const bool pend = (x[r] >= 0) & !m0 & !e0 & !m1 & !e1;
      const unsigned pm = __ballot_sync(kFull, pend);
      if (pend) {
        const int pos = nq + __popc(pm & lt);
        qx[pos] = x[r];
        qh[pos] = h[r];
      }
      nq += __popc(pm);
    }
    if (nq) {
      __syncwarp();
      for (int i = lane; i < nq; i += 32)
        hits += probe_walk<HIER>(qx[i], tb, lg, qh[i], k0, bn, b, status);
      __syncwarp();
    }
    if (EARLY) {
      const int tot = __reduce_add_sync(kFull, hits);
      const int done = min(base + 32 * R, s);
      if (tot >= need_hits || done - tot > max_miss) return lane == 0 ? tot : 0;
    }
  }
  return hits;
}

// Flattened probing of 32 (probe side, table side) pairs held one per lane.
// Pair j probes keys[a_j .. a_j + s_j) into the table at toff_j.  Round r
// gives lane i the probe with flat index 32r+i (consecutive lanes read
// consecutive keys of a pair, and with hash-ordered keys probe nearby
// buckets).  kRounds rounds are issued together -- first their key loads,
// then the loads of slots 0 and 1 of each home bucket (two independent
// loads per probe: with load factor 0.2 and 5-slot buckets almost every
// probe is settled by these two), and only then the rare longer walks.
// For every hit, on_hit(k) is called on the lane that probed, with k the
// lane index of the owning pair; returns the number of hits of this lane.
constexpr int kRounds = 4;

template <bool HIER, class OnHit>
__device__ __forceinline__ int flat_probe(const int32_t* __restrict__ keys,
                                          int64_t n_keys,
                                          const int32_t* __restrict__ table,
                                          int s, int a_start, int64_t toff,
                                          int lg, int lg_max, int64_t bn,
                                          int b, int32_t* status,
                                          OnHit on_hit) {
  (void)n_keys;
  const int lane = threadIdx.x & 31;
  int S, hits = 0;
  const int P = warp_excl_scan(s, &S);
  const int64_t bn1 = b > 1 ? bn : 0;
  for (int base = 0; base < S; base += 32 * kRounds) {
    int x[kRounds], h[kRounds], klg[kRounds], own[kRounds], s0[kRounds], s1[kRounds];
    const int32_t* tb[kRounds];
    bool act[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      const int f = base + r * 32 + lane;
      act[r] = f < S;
      x[r] = 0;
      klg[r] = 3;
      tb[r] = table;
      own[r] = 0;
      if (base + r * 32 >= S) continue;  // warp-uniform: round past the end
      const int k = owner_lane(P, f);
      const int kp = __shfl_sync(kFull, P, k);
      const int ka = __shfl_sync(kFull, a_start, k);
      klg[r] = __shfl_sync(kFull, lg, k);
      tb[r] = table + __shfl_sync(kFull, toff, k);
      own[r] = k;
      x[r] = act[r] ? __ldg(keys + ka + (f - kp)) : 0;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      h[r] = home_bucket<HIER>(x[r], klg[r], lg_max);
      s0[r] = act[r] ? __ldg(tb[r] + h[r]) : -1;
      s1[r] = act[r] ? __ldg(tb[r] + h[r] + bn1) : -1;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      if (!act[r]) continue;
      if (probe_resolve2<HIER>(x[r], s0[r], s1[r], tb[r], klg[r], h[r], bn, b, status)) {
        ++hits;
        on_hit(own[r]);
      }
    }
  }
  return hits;
}

}  // namespace rst
