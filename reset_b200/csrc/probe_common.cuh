// Device helpers shared by the probe kernels.
#pragma once

#include "common.cuh"

namespace rst {

enum : int32_t { kErrBadId = 4 };

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

// Flattened probing of 32 (probe side, table side) pairs held one per lane.
// For every hit, on_hit(k) is called on the lane that probed, with k the
// lane index of the owning pair; returns the number of hits of this lane.
template <bool HIER, class OnHit>
__device__ __forceinline__ int flat_probe(const int32_t* __restrict__ keys,
                                           const int32_t* __restrict__ table,
                                           int s, int a_start, int64_t toff,
                                           int lg, int lg_max, int64_t bn,
                                           int b, int32_t* status,
                                           OnHit on_hit) {
  const int lane = threadIdx.x & 31;
  int S, hits = 0;
  const int P = warp_excl_scan(s, &S);
  for (int base = 0; base < S; base += 32) {
    const int f = base + lane;
    const int k = owner_lane(P, f);
    const int kp = __shfl_sync(kFull, P, k);
    const int ka = __shfl_sync(kFull, a_start, k);
    const int klg = __shfl_sync(kFull, lg, k);
    const int64_t kt = __shfl_sync(kFull, toff, k);
    if (f < S) {
      const int x = __ldg(keys + ka + (f - kp));
      if (probe_key<HIER>(x, table + kt, klg, lg_max, bn, b, status)) {
        ++hits;
        on_hit(k);
      }
    }
  }
  return hits;
}

}  // namespace rst
