// Hash-probe intersection kernels: triangle counting, set-similarity search,
// the raw two-set intersection, and conjunctive retrieval.
//
// Reference kernels: dynamic_triangle_count (triangle-count/TC.cu:128-190),
// set_similarity_search_kernel (set-similarity-search/sss.cu:93-154),
// intersection_kernel (set_size/intersection.cu:154-181), ir_kernel
// (information-retrieval/ir.cu:94-176).  All share the probe rule of
// search_in_hashtable (TC.cu:11-31): walk the slots of the home bucket, then
// the next bucket; a hit is an equal slot, a miss an empty (-1) slot.
//
// Scheduling (B200): the reference gives every pair a whole warp, so a warp
// probing a 3-element set idles 29 lanes.  Here a warp takes 32 pairs (one
// per lane), loads each pair's two packed 16-byte set descriptors, and
// flattens the probes of all 32 pairs: round r gives lane i the probe with
// flat index 32r+i, found by a 5-step shuffle binary search over the pairs'
// prefix sums.  Tiny intersections thus run at thread granularity, medium
// ones spread over the warp, and hub x hub pairs over as many rounds as
// they need; the grid is persistent and walks 32-pair chunks grid-stride.
#include <cub/cub.cuh>

#include <climits>

#include "common.cuh"
#include "probe_common.cuh"

namespace rst {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIrSlice = 512;  // candidates per IR work item

// ----------------------------------------------------------------- TC ----

template <bool HIER, int ROUNDS, bool LEAN>
__global__ void __launch_bounds__(kThreads, 4)
    tc_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ off,
              const int32_t* __restrict__ cols,
              const int32_t* __restrict__ chunk_row, int32_t n, int64_t m,
              const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
              unsigned long long* __restrict__ count,
              unsigned long long* __restrict__ cursor, int warp_pair_min,
              int32_t* __restrict__ status) {
  __shared__ int s_qx[kWarps][32 * ROUNDS], s_qh[kWarps][32 * ROUNDS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // edges past off[n] have no row: never read them (nor their chunk rows)
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  unsigned long long hits = 0;
  // dynamic schedule: a warp takes the next 32-edge chunk when it is done
  for (;;) {
    unsigned long long cc = 0;
    if (lane == 0) cc = atomicAdd(cursor, 1ull);
    const int64_t c = (int64_t)__shfl_sync(kFull, cc, 0);
    if (c >= n_chunks) break;
    const int64_t e64 = c * 32 + lane;
    const bool valid = e64 < me;
    const int e = (int)(valid ? e64 : me - 1);
    int u0 = __ldg(chunk_row + c);
    if ((unsigned)u0 >= (unsigned)n) u0 = 0;
    int u = row_of_edge(off, n, u0, e);
    int v = __ldg(cols + e);
    bool ok = valid;
    if ((unsigned)u >= (unsigned)n || (unsigned)v >= (unsigned)n) {
      if (valid) atomicOr(status, kErrBadId);
      ok = false;
      u = v = 0;
    }
    const int4 du = __ldg(desc + u);
    const int4 dv = __ldg(desc + v);
    // TC.cu:148-157: the larger set's table is probed (ties: u probes v).
    const bool sw = du.y > dv.y;
    const int4 A = sw ? dv : du;
    const int4 B = sw ? du : dv;
    const int s = ok ? A.y : 0;
    // pairs with a warp's worth of keys get the whole warp, one at a time;
    // the rest are flattened across the lanes
    const bool big = s >= warp_pair_min;
    unsigned bigm = __ballot_sync(kFull, big);
    const int64_t bt = desc_toff(B);
    const int blg = desc_lg(B);
    while (bigm) {
      const int k = __ffs(bigm) - 1;
      bigm &= bigm - 1;
      const int ks = __shfl_sync(kFull, s, k);
      const int ka = __shfl_sync(kFull, A.x, k);
      const int klg = __shfl_sync(kFull, blg, k);
      const int64_t kt = __shfl_sync(kFull, bt, k);
      if (LEAN)
        hits += warp_probe_pair_lean<HIER, ROUNDS>(cols + ka, ks, table + kt, klg, lg_max,
                                                   bn, b, status, s_qx[warp], s_qh[warp]);
      else
        hits += warp_probe_pair<HIER, ROUNDS>(cols + ka, ks, table + kt, klg, lg_max,
                                              bn, b, status, s_qx[warp], s_qh[warp]);
    }
    hits += flat_probe<HIER>(cols, me, table, big ? 0 : s, A.x, bt, blg, lg_max,
                             bn, b, status, [](int) {});
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

// ---------------------------------------------------------------- SSS ----

template <bool HIER, bool FLOAT_RULE, int ROUNDS, bool LEAN, bool EARLY = false>
__global__ void __launch_bounds__(kThreads, 4)
    sss_kernel(const int4* __restrict__ desc, int32_t n,
               const int32_t* __restrict__ elems, int64_t n_elems,
               const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
               int64_t np, const int64_t* __restrict__ np_dev,
               unsigned long long* __restrict__ cursor,
               const int32_t* __restrict__ table, int64_t bn, int b,
               int lg_max, int num, int den, float thr, int warp_pair_min,
               uint8_t* __restrict__ flags, int32_t* __restrict__ inter,
               int32_t* __restrict__ status) {
  __shared__ int s_hits[kWarps][32];
  __shared__ int s_qx[kWarps][32 * ROUNDS], s_qh[kWarps][32 * ROUNDS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (np_dev) np = *np_dev;  // pair count set on the device (captured graphs)
  const int64_t n_chunks = (np + 31) >> 5;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t it = 0;; ++it) {
    int64_t c;
    if (cursor) {  // dynamic schedule: next chunk of 32 pairs
      unsigned long long cc = 0;
      if (lane == 0) cc = atomicAdd(cursor, 1ull);
      c = (int64_t)__shfl_sync(kFull, cc, 0);
    } else {
      c = gw + it * nw;
    }
    if (c >= n_chunks) break;
    const int64_t p = c * 32 + lane;
    const bool valid = p < np;
    int a = valid ? __ldg(pa + p) : 0;
    int q = valid ? __ldg(pb + p) : 0;
    bool ok = valid;
    if ((unsigned)a >= (unsigned)n || (unsigned)q >= (unsigned)n) {
      if (valid) atomicOr(status, kErrBadId);
      ok = false;
      a = q = 0;
    }
    const int4 da = __ldg(desc + a);
    const int4 dq = __ldg(desc + q);
    const bool sw = da.y > dq.y;  // sss.cu:108-115
    const int4 A = sw ? dq : da;
    const int4 B = sw ? da : dq;
    const int s = ok ? A.y : 0;
    s_hits[warp][lane] = 0;
    __syncwarp();
    // pairs with a warp's worth of keys: the whole warp, one pair at a time
    const bool big = s >= warp_pair_min;
    unsigned bigm = __ballot_sync(kFull, big);
    const int64_t bt = desc_toff(B);
    const int blg = desc_lg(B);
    while (bigm) {
      const int k = __ffs(bigm) - 1;
      bigm &= bigm - 1;
      const int ks = __shfl_sync(kFull, s, k);
      const int ka = __shfl_sync(kFull, A.x, k);
      const int klg = __shfl_sync(kFull, blg, k);
      const int64_t kt = __shfl_sync(kFull, bt, k);
      int h;
      if (EARLY) {
        // decisions only: need = smallest I with den*I >= num*(|A|+|B|-I)
        const int kd = __shfl_sync(kFull, da.y + dq.y, k);
        const int64_t need64 = ((int64_t)num * kd + (num + den) - 1) / (num + den);
        const int need = (int)need64;
        if (need > ks) {
          h = 0;  // unreachable: not similar, no probes
        } else {
          h = warp_probe_pair_lean<HIER, ROUNDS, true>(elems + ka, ks, table + kt, klg,
                                                       lg_max, bn, b, status, s_qx[warp],
                                                       s_qh[warp], need, ks - need);
        }
      } else if (LEAN) {
        h = warp_probe_pair_lean<HIER, ROUNDS>(elems + ka, ks, table + kt, klg, lg_max, bn,
                                               b, status, s_qx[warp], s_qh[warp]);
      } else {
        h = warp_probe_pair<HIER, ROUNDS>(elems + ka, ks, table + kt, klg, lg_max, bn, b,
                                          status, s_qx[warp], s_qh[warp]);
      }
      h = __reduce_add_sync(kFull, h);
      if (lane == 0) s_hits[warp][k] += h;
      __syncwarp();
    }
    flat_probe<HIER>(elems, n_elems, table, big ? 0 : s, A.x, bt, blg, lg_max, bn,
                     b, status, [&](int k) { atomicAdd(&s_hits[warp][k], 1); });
    __syncwarp();
    const int I = s_hits[warp][lane];
    __syncwarp();
    if (ok) {
      const int U = da.y + dq.y - I;
      bool f;
      if (FLOAT_RULE) {
        f = ((float)I / (float)U) >= thr;  // sss.cu:139-140
      } else {
        f = U > 0 && (int64_t)den * I >= (int64_t)num * U;
      }
      flags[p] = (uint8_t)f;
      if (inter) inter[p] = I;
    } else if (valid) {
      flags[p] = 0;
      if (inter) inter[p] = 0;
    }
  }
}

// ----------------------------------------------------------- raw pair ----

__global__ void __launch_bounds__(kThreads)
    pair_probe_kernel(const int32_t* __restrict__ a, int64_t na,
                      const int32_t* __restrict__ table, int lg, int64_t bn,
                      int b, unsigned long long* __restrict__ count,
                      int32_t* __restrict__ status) {
  unsigned long long hits = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na;
       i += (int64_t)gridDim.x * blockDim.x) {
    // set_size/intersection.cu:169: d_hash(key, len) = key & (len-1)
    hits += probe_key<false>(__ldg(a + i), table, lg, lg, bn, b, status);
  }
  hits = warp_sum_u64(hits);
  if ((threadIdx.x & 31) == 0 && hits) atomicAdd(count, hits);
}

// ----------------------------------------------------------------- IR ----

__global__ void ir_plan_kernel(const int4* __restrict__ desc, int32_t n,
                               const int32_t* __restrict__ query,
                               const int32_t* __restrict__ qoff, int32_t nq,
                               int64_t* __restrict__ sl_off,
                               int32_t* __restrict__ status) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int qs = qoff[q], ql = qoff[q + 1] - qs;
    int64_t ns = 0;
    if (ql > 0) {
      const int t0 = query[qs];
      if ((unsigned)t0 < (unsigned)n) {
        const int df = desc[t0].y;
        ns = (df + kIrSlice - 1) / kIrSlice;
      } else {
        atomicOr(status, kErrBadId);
      }
    }
    sl_off[q] = ns;
  }
}

__global__ void ir_total_kernel(const int64_t* __restrict__ ns_excl,
                                int64_t* __restrict__ sl_off, int32_t nq,
                                int64_t* __restrict__ total) {
  // sl_off holds the exclusive scan of the slice counts for q < nq; the
  // count of the last query is recomputed by the caller into ns_excl[0].
  int64_t t = nq > 0 ? sl_off[nq - 1] + ns_excl[0] : 0;
  sl_off[nq] = t;
  *total = t;
}

// One warp per slice of kIrSlice candidates of the first term's list:
// every candidate is checked against all further terms (early exit per
// lane), survivors are compacted with ballot/popc to the front of the
// slice's own region stage[slice * kIrSlice ...], in first-term order, and
// their number goes to sl_cnt[slice].
template <bool HIER>
__global__ void __launch_bounds__(kThreads)
    ir_slice_kernel(const int4* __restrict__ desc, int32_t n,
                    const int32_t* __restrict__ docs,
                    const int32_t* __restrict__ query,
                    const int32_t* __restrict__ qoff, int32_t nq,
                    const int64_t* __restrict__ sl_off,
                    int32_t* __restrict__ stage, int32_t* __restrict__ sl_cnt,
                    const int32_t* __restrict__ table, int64_t bn, int b,
                    int lg_max, int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t total = sl_off[nq];
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sidx = gw; sidx < total; sidx += nw) {
    // query owning this slice: largest q with sl_off[q] <= sidx
    int lo = 0, hi = nq - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (sl_off[mid] <= sidx) lo = mid; else hi = mid - 1;
    }
    const int q = lo;
    const int qs = qoff[q], ql = qoff[q + 1] - qs;
    const int4 d0 = desc[query[qs]];
    const int64_t j0 = (sidx - sl_off[q]) * kIrSlice;
    const int64_t j1 = min((int64_t)d0.y, j0 + kIrSlice);
    int32_t* out = stage + sidx * kIrSlice;
    int w = 0;
    for (int64_t jb = j0; jb < j1; jb += 32) {
      const int64_t j = jb + lane;
      const bool active = j < j1;
      const int x = active ? __ldg(docs + d0.x + j) : 0;
      bool ok = active;
      for (int i = 1; i < ql; ++i) {  // ir.cu:131-161, all terms per candidate
        const int t = __ldg(query + qs + i);
        if ((unsigned)t >= (unsigned)n) {
          if (ok) atomicOr(status, kErrBadId);
          ok = false;
          continue;
        }
        if (!__any_sync(kFull, ok)) break;
        const int4 dt = __ldg(desc + t);
        if (ok)
          ok = probe_key<HIER>(x, table + desc_toff(dt), desc_lg(dt), lg_max,
                               bn, b, status);
      }
      const unsigned msk = __ballot_sync(kFull, ok);
      if (ok) out[w + __popc(msk & lt)] = x;
      w += __popc(msk);
    }
    if (lane == 0) sl_cnt[sidx] = w;
  }
}

// Exclusive scan of per-slice survivor counts in one block (chunks of
// blockDim with a running carry): pos[s] = survivors before slice s,
// pos[ns] = all survivors.
__global__ void slice_scan_kernel(const int32_t* __restrict__ cnt, int64_t ns,
                                  int64_t* __restrict__ pos) {
  __shared__ int64_t s_part[32];
  __shared__ int64_t s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < ns; base += blockDim.x) {
    const int64_t i = base + tid;
    const int64_t v = i < ns ? cnt[i] : 0;
    int64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_part[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      int64_t w = lane < nw ? s_part[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += t;
      }
      if (lane < nw) s_part[lane] = w;
    }
    __syncthreads();
    const int64_t before = s_carry + (warp > 0 ? s_part[warp - 1] : 0);
    if (i < ns) pos[i] = before + incl - v;
    __syncthreads();
    if (tid == blockDim.x - 1) s_carry = before + incl;
    __syncthreads();
  }
  if (tid == 0) pos[ns] = s_carry;
}

// One warp per slice: copies its survivors out of the stage, out of place,
// so all slices move in parallel.  Query q's survivors land at
//   res + res_off[q] + (pos[s] - pos[sl_off[q]])   (res_off given), or
//   res + pos[s]                                    (packed, res_off NULL).
__global__ void __launch_bounds__(kThreads)
    ir_gather_kernel(const int64_t* __restrict__ sl_off, int32_t nq,
                     const int32_t* __restrict__ sl_cnt,
                     const int64_t* __restrict__ pos,
                     const int32_t* __restrict__ stage,
                     const int64_t* __restrict__ res_off,
                     int32_t* __restrict__ res) {
  const int lane = threadIdx.x & 31;
  const int64_t total = sl_off[nq];
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t s = gw; s < total; s += nw) {
    const int c = sl_cnt[s];
    if (c == 0) continue;
    int64_t dst = pos[s];
    if (res_off) {
      int lo = 0, hi = nq - 1;  // query owning slice s
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sl_off[mid] <= s) lo = mid; else hi = mid - 1;
      }
      dst = res_off[lo] + (pos[s] - pos[sl_off[lo]]);
    }
    const int32_t* src = stage + s * kIrSlice;
    for (int j = lane; j < c; j += 32) res[dst + j] = src[j];
  }
}

// Per query: its count, and (packed mode) where its survivors start.
__global__ void ir_counts_kernel(const int64_t* __restrict__ sl_off, int32_t nq,
                                 const int64_t* __restrict__ pos,
                                 int32_t* __restrict__ cnt,
                                 int64_t* __restrict__ packed_off) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = pos[sl_off[q]], b = pos[sl_off[q + 1]];
    cnt[q] = (int32_t)(b - a);
    if (packed_off) {
      packed_off[q] = a;
      if (q == nq - 1) packed_off[nq] = b;
    }
  }
}

// Launches the slice, scan, gather and count kernels for a planned batch.
template <bool HIER>
reset_status ir_run(const reset_table* t, const int4* desc, const int32_t* docs,
                    const int32_t* query, const int32_t* qoff, int32_t nq,
                    const int64_t* sl_off, int64_t total_slices,
                    const int64_t* res_off, int32_t* res, int32_t* stage,
                    int32_t* sl_cnt, int64_t* pos, int32_t* cnt,
                    int64_t* packed_off, cudaStream_t st, bool yield);

int persistent_grid(const void* kernel) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0);
  if (per_sm < 1) per_sm = 1;
  return sm_count() * per_sm;
}

int64_t clamp_grid(int64_t want, int cap) {
  if (want < 1) want = 1;
  return want < cap ? want : cap;
}

template <bool HIER>
reset_status ir_run(const reset_table* t, const int4* desc, const int32_t* docs,
                    const int32_t* query, const int32_t* qoff, int32_t nq,
                    const int64_t* sl_off, int64_t total_slices,
                    const int64_t* res_off, int32_t* res, int32_t* stage,
                    int32_t* sl_cnt, int64_t* pos, int32_t* cnt,
                    int64_t* packed_off, cudaStream_t st, bool yield) {
  // yield: one warp per slice and no persistent grid, so the blocks retire
  // as they finish and the block scheduler can interleave other streams'
  // (higher-priority) work; otherwise a persistent grid walks the slices
  const int64_t per_slice = std::min<int64_t>((total_slices + kWarps - 1) / kWarps, INT32_MAX);
  if (total_slices > 0) {
    const int64_t g = yield ? per_slice
                            : clamp_grid(per_slice,
                                         persistent_grid((const void*)ir_slice_kernel<HIER>));
    note_launch();
    ir_slice_kernel<HIER><<<(int)g, kThreads, 0, st>>>(
        desc, t->n, docs, query, qoff, nq, sl_off, stage, sl_cnt, t->d_table,
        t->bucket_num, t->bucket, t->lg_max, t->d_status);
    RST_CUDA(cudaGetLastError());
  }
  note_launch();
  slice_scan_kernel<<<1, 1024, 0, st>>>(sl_cnt, total_slices, pos);
  RST_CUDA(cudaGetLastError());
  if (total_slices > 0) {
    const int64_t g = yield ? per_slice
                            : clamp_grid(per_slice, persistent_grid((const void*)ir_gather_kernel));
    note_launch();
    ir_gather_kernel<<<(int)g, kThreads, 0, st>>>(sl_off, nq, sl_cnt, pos, stage, res_off,
                                                   res);
    RST_CUDA(cudaGetLastError());
  }
  note_launch();
  ir_counts_kernel<<<(int)clamp_grid((nq + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      sl_off, nq, pos, cnt, packed_off);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

// Resolves the descriptor array for a probe call: the table's own when the
// caller passes the offsets the table was built on, else a fresh one.
struct DescScope {
  const int4* desc = nullptr;
  int4* owned = nullptr;
  cudaStream_t st = nullptr;
  ~DescScope() {
    if (owned) cudaFreeAsync(owned, st);
  }
};

reset_status resolve_desc(const reset_table* t, const int32_t* d_off,
                          cudaStream_t st, DescScope* ds) {
  ds->st = st;
  if (!d_off || d_off == t->build_off) {
    ds->desc = t->d_desc;
    return RESET_OK;
  }
  RST_CHECK(make_desc(t, d_off, &ds->owned, st));
  ds->desc = ds->owned;
  return RESET_OK;
}

}  // namespace

// Persistent pair kernel for the batched form: pair count read on the device
// (np_dev), dynamic 32-pair chunks (cursor, zeroed by the caller), exact
// rule.  No allocation and no synchronisation, so it can be captured.
reset_status sss_launch_persistent(const reset_table* t, const int32_t* elems,
                                   const int32_t* pa, const int32_t* pb,
                                   const int64_t* np_dev,
                                   unsigned long long* cursor, int64_t capacity,
                                   int32_t num, int32_t den, uint8_t* flags,
                                   int32_t* inter, bool decisions_only,
                                   cudaStream_t st) {
  const reset_tuning tun = tuning();
  const int wpm = tun.warp_pair_min;
#define SSS_P(H, R, LN, E)                                                     \
  do {                                                                         \
    const int64_t g = clamp_grid(((capacity + 31) / 32 + kWarps - 1) / kWarps, \
                                 persistent_grid((const void*)sss_kernel<H, false, R, LN, E>)); \
    note_launch();                                                             \
    sss_kernel<H, false, R, LN, E><<<(int)g, kThreads, 0, st>>>(               \
        t->d_desc, t->n, elems, t->m, pa, pb, capacity, np_dev, cursor,        \
        t->d_table, t->bucket_num, t->bucket, t->lg_max, num, den, 0.f, wpm,   \
        flags, E ? nullptr : inter, t->d_status);                              \
  } while (0)
  if (decisions_only) {
    if (t->hier) SSS_P(true, 8, true, true); else SSS_P(false, 8, true, true);
  } else if (tun.probe_variant == 1) {
    if (t->hier) SSS_P(true, 8, true, false); else SSS_P(false, 8, true, false);
  } else {
    if (t->hier) SSS_P(true, 4, false, false); else SSS_P(false, 4, false, false);
  }
#undef SSS_P
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

int ir_slice_size() { return kIrSlice; }

// Conjunctive retrieval for a batch whose slice plan is on the device:
// sl_off[q] = sum over earlier queries of ceil(df(first term) / kIrSlice),
// sl_off[nq] = total_slices.  Scratch: stage (total_slices * kIrSlice ints),
// sl_cnt (total_slices ints), pos (total_slices + 1 int64).  Results go to
// res at res_off[q] (as reset_ir) or, with res_off NULL, packed query after
// query with packed_off[q] (nq + 1 int64) giving where each starts.  Uses
// the table's own descriptors.  No allocation, no synchronisation.
reset_status ir_launch_planned(const reset_table* t, const int32_t* docs,
                               const int32_t* query, const int32_t* qoff,
                               int32_t nq, const int64_t* sl_off,
                               int64_t total_slices, const int64_t* res_off,
                               int32_t* res, int32_t* stage, int32_t* sl_cnt,
                               int64_t* pos, int32_t* cnt, int64_t* packed_off,
                               cudaStream_t st, bool yield) {
  if (nq <= 0) return RESET_OK;
  if (t->hier)
    return ir_run<true>(t, t->d_desc, docs, query, qoff, nq, sl_off, total_slices, res_off,
                        res, stage, sl_cnt, pos, cnt, packed_off, st, yield);
  return ir_run<false>(t, t->d_desc, docs, query, qoff, nq, sl_off, total_slices, res_off,
                       res, stage, sl_cnt, pos, cnt, packed_off, st, yield);
}

}  // namespace rst

using namespace rst;

extern "C" {

reset_status reset_tc_count_ex(const reset_table* t, const int32_t* d_off,
                               const int32_t* d_cols, int64_t m, int32_t method,
                               uint64_t* d_count, reset_stream_t stream) {
  if (!t || !d_count) return arg_fail("NULL table or count");
  if (m < 0 || m > INT32_MAX) return arg_fail("m out of range");
  if (m > 0 && (!d_cols || !d_off)) return arg_fail("NULL offsets or cols");
  if (method < 0 || method > 3) return arg_fail("method must be 0, 1, 2 or 3");
  const bool cols16 = (reinterpret_cast<uintptr_t>(d_cols) & 15) == 0;
  if (method == 3 && !cols16)
    return arg_fail("method 3 needs a 16-byte aligned column array");
  if (method == 0) method = cols16 && m <= INT32_MAX - 16 ? 3 : 1;
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m == 0 || t->n == 0) return RESET_OK;
  DescScope ds;
  RST_CHECK(resolve_desc(t, d_off, st, &ds));
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(d_count);
  if (method == 2) return tc_staged(t, ds.desc, d_cols, m, cnt, st);
  const int32_t* rows = t->d_chunk_row;
  int32_t* owned_rows = nullptr;
  if (d_off != t->build_off || m != t->m) {
    RST_CHECK(make_chunk_rows(d_off, t->n, m, &owned_rows, st));
    rows = owned_rows;
  }
  if (method == 3) {
    reset_status s = tc_owner(t, ds.desc, d_off, d_cols, m, d_off, d_cols, rows, m, cnt, st);
    if (owned_rows) cudaFreeAsync(owned_rows, st);
    return s;
  }
  unsigned long long* cursor = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&cursor), sizeof(*cursor), st));
  cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(*cursor), st);
  const reset_tuning tun = tuning();
  const int wpm = tun.warp_pair_min;
#define TC_LAUNCH(H, R, LN)                                                    \
  do {                                                                         \
    const int64_t g = clamp_grid(((m + 31) / 32 + kWarps - 1) / kWarps,        \
                                 persistent_grid((const void*)tc_kernel<H, R, LN>)); \
    note_launch();                                                             \
    tc_kernel<H, R, LN><<<(int)g, kThreads, 0, st>>>(                          \
        ds.desc, d_off, d_cols, rows, t->n, m, t->d_table, t->bucket_num,      \
        t->bucket, t->lg_max, cnt, cursor, wpm, t->d_status);                  \
  } while (0)
  if (e == cudaSuccess) {
    const bool lean = tun.probe_variant == 1;
    if (t->hier) {
      if (lean) {
        if (tun.probe_rounds == 2) TC_LAUNCH(true, 2, true);
        else if (tun.probe_rounds == 8) TC_LAUNCH(true, 8, true);
        else TC_LAUNCH(true, 4, true);
      } else {
        if (tun.probe_rounds == 2) TC_LAUNCH(true, 2, false); else TC_LAUNCH(true, 4, false);
      }
    } else {
      if (lean) {
        if (tun.probe_rounds == 2) TC_LAUNCH(false, 2, true);
        else if (tun.probe_rounds == 8) TC_LAUNCH(false, 8, true);
        else TC_LAUNCH(false, 4, true);
      } else {
        if (tun.probe_rounds == 2) TC_LAUNCH(false, 2, false); else TC_LAUNCH(false, 4, false);
      }
    }
    e = cudaGetLastError();
  }
#undef TC_LAUNCH
  cudaFreeAsync(cursor, st);
  if (owned_rows) cudaFreeAsync(owned_rows, st);
  if (e != cudaSuccess) return cuda_fail(e, "tc_kernel launch", __FILE__, __LINE__);
  return RESET_OK;
}

reset_status reset_tc_count(const reset_table* t, const int32_t* d_off,
                            const int32_t* d_cols, int64_t m,
                            uint64_t* d_count, reset_stream_t stream) {
  return reset_tc_count_ex(t, d_off, d_cols, m, 0, d_count, stream);
}

static reset_status sss_common(const reset_table* t, const int32_t* d_off,
                               const int32_t* d_elems, const int32_t* d_pa,
                               const int32_t* d_pb, int64_t np, bool float_rule,
                               int32_t num, int32_t den, float thr,
                               uint8_t* d_flags, int32_t* d_inter,
                               reset_stream_t stream) {
  if (!t) return arg_fail("NULL table");
  if (np < 0) return arg_fail("negative pair count");
  if (np == 0) return RESET_OK;
  if (!d_elems || !d_pa || !d_pb || !d_flags) return arg_fail("NULL pointer");
  if (!float_rule && (den <= 0 || num < 0)) return arg_fail("threshold num/den");
  cudaStream_t st = as_stream(stream);
  DescScope ds;
  RST_CHECK(resolve_desc(t, d_off, st, &ds));
  const reset_tuning tun = tuning();
  const bool el16 = (reinterpret_cast<uintptr_t>(d_elems) & 15) == 0;
  if (tun.pair_method == 2 && !el16)
    return arg_fail("pair_method 2 needs a 16-byte aligned element array");
  // default: the pair-flattened kernel (measured faster or equal on B200 for
  // graph pairs and self-join candidates, and it stops deciding pairs early)
  if (tun.pair_method == 2 && el16 && np <= INT32_MAX && t->m <= INT32_MAX - 4)
    return sss_owner(t, ds.desc, d_elems, t->m, d_pa, d_pb, np, float_rule, num, den, thr,
                     d_flags, d_inter, st);
#define SSS_LAUNCH(H, F, R, LN, ...)                                         \
  do {                                                                       \
    const int64_t g = clamp_grid(((np + 31) / 32 + kWarps - 1) / kWarps,     \
                                 persistent_grid((const void*)sss_kernel<H, F, R, LN, ##__VA_ARGS__>)); \
    note_launch(); sss_kernel<H, F, R, LN, ##__VA_ARGS__><<<(int)g, kThreads, 0, st>>>( \
        ds.desc, t->n, d_elems, t->m, d_pa, d_pb, np, nullptr, nullptr,      \
        t->d_table, t->bucket_num, t->bucket, t->lg_max, num, den, thr,       \
        tun.warp_pair_min, d_flags, d_inter, t->d_status);                    \
  } while (0)
#define SSS_V(H, F)                                                          \
  do {                                                                       \
    if (tun.probe_variant == 1) SSS_LAUNCH(H, F, 8, true);                   \
    else SSS_LAUNCH(H, F, 4, false);                                         \
  } while (0)
  if (!float_rule && !d_inter) {
    // decisions only: pairs stop as soon as the rule is settled
    if (t->hier) SSS_LAUNCH(true, false, 8, true, true);
    else SSS_LAUNCH(false, false, 8, true, true);
  } else if (t->hier) {
    if (float_rule) SSS_V(true, true); else SSS_V(true, false);
  } else {
    if (float_rule) SSS_V(false, true); else SSS_V(false, false);
  }
#undef SSS_V
#undef SSS_LAUNCH
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

reset_status reset_sss(const reset_table* t, const int32_t* d_off,
                       const int32_t* d_elems, const int32_t* d_pair_a,
                       const int32_t* d_pair_b, int64_t npairs, int32_t num,
                       int32_t den, uint8_t* d_flags, int32_t* d_inter,
                       reset_stream_t stream) {
  return sss_common(t, d_off, d_elems, d_pair_a, d_pair_b, npairs, false, num,
                    den, 0.f, d_flags, d_inter, stream);
}

reset_status reset_sss_float(const reset_table* t, const int32_t* d_off,
                             const int32_t* d_elems, const int32_t* d_pair_a,
                             const int32_t* d_pair_b, int64_t npairs,
                             float thr, uint8_t* d_flags, int32_t* d_inter,
                             reset_stream_t stream) {
  return sss_common(t, d_off, d_elems, d_pair_a, d_pair_b, npairs, true, 0, 1,
                    thr, d_flags, d_inter, stream);
}

reset_status reset_intersect_count(const int32_t* d_a, int64_t na,
                                   const int32_t* d_b, int64_t nb,
                                   const reset_params* params,
                                   int64_t* d_count, reset_stream_t stream) {
  if (!d_count) return arg_fail("NULL count");
  if (na < 0 || nb < 0 || nb > INT32_MAX) return arg_fail("sizes out of range");
  if ((na > 0 && !d_a) || (nb > 0 && !d_b)) return arg_fail("NULL set");
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int64_t), st));
  if (na == 0 || nb == 0) return RESET_OK;
  int32_t* d_offb = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_offb), 2 * sizeof(int32_t), st));
  const int32_t h_offb[2] = {0, (int32_t)nb};
  RST_CUDA(cudaMemcpyAsync(d_offb, h_offb, sizeof(h_offb), cudaMemcpyHostToDevice, st));
  reset_table* t = nullptr;
  reset_status s = reset_table_build(d_offb, d_b, 1, nb, params, 0, nullptr, &t, stream);
  if (s != RESET_OK) {
    cudaFreeAsync(d_offb, st);
    return s;
  }
  const int lg = t->lg_max;
  const int64_t g = clamp_grid((na + kThreads - 1) / kThreads,
                               persistent_grid((const void*)pair_probe_kernel));
  note_launch(); pair_probe_kernel<<<(int)g, kThreads, 0, st>>>(
      d_a, na, t->d_table, lg, t->bucket_num, t->bucket,
      reinterpret_cast<unsigned long long*>(d_count), t->d_status);
  cudaError_t e = cudaGetLastError();
  reset_status cs = reset_table_check(t, stream);  // synchronises `stream`
  cudaFree(d_offb);
  reset_table_free(t);
  if (e != cudaSuccess) return cuda_fail(e, "pair_probe_kernel", __FILE__, __LINE__);
  return cs;
}

reset_status reset_ir(const reset_table* t, const int32_t* d_toff,
                      const int32_t* d_docs, const int32_t* d_query,
                      const int32_t* d_qoff, int32_t nq,
                      const int64_t* d_res_off, int32_t* d_res,
                      int32_t* d_cnt, reset_stream_t stream) {
  if (!t) return arg_fail("NULL table");
  if (nq < 0) return arg_fail("negative query count");
  if (nq == 0) return RESET_OK;
  if (!d_docs || !d_query || !d_qoff || !d_res_off || !d_res || !d_cnt)
    return arg_fail("NULL pointer");
  cudaStream_t st = as_stream(stream);
  DescScope ds;
  RST_CHECK(resolve_desc(t, d_toff, st, &ds));
  int64_t* d_sl = nullptr;
  int64_t* d_tot = nullptr;
  int32_t* d_slc = nullptr;
  int64_t* d_pos = nullptr;
  int32_t* d_stage = nullptr;
  void* d_tmp = nullptr;
  reset_status rs = RESET_OK;
  auto cleanup = [&]() {
    if (d_pos) cudaFreeAsync(d_pos, st);
    if (d_stage) cudaFreeAsync(d_stage, st);
    if (d_sl) cudaFreeAsync(d_sl, st);
    if (d_tot) cudaFreeAsync(d_tot, st);
    if (d_slc) cudaFreeAsync(d_slc, st);
    if (d_tmp) cudaFreeAsync(d_tmp, st);
  };
#define IR_CUDA(call)                                                       \
  do {                                                                      \
    cudaError_t _e = (call);                                                \
    if (_e != cudaSuccess) {                                                \
      rs = cuda_fail(_e, #call, __FILE__, __LINE__);                        \
      cleanup();                                                            \
      return rs;                                                            \
    }                                                                       \
  } while (0)
  IR_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_sl), sizeof(int64_t) * (nq + 1), st));
  IR_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_tot), sizeof(int64_t) * 2, st));
  note_launch(); ir_plan_kernel<<<(int)clamp_grid((nq + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      ds.desc, t->n, d_query, d_qoff, nq, d_sl, t->d_status);
  IR_CUDA(cudaGetLastError());
  // keep the last count, then scan in place
  IR_CUDA(cudaMemcpyAsync(d_tot + 1, d_sl + (nq - 1), sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
  size_t tb = 0;
  IR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_sl, d_sl, nq, st));
  IR_CUDA(scratch_malloc(&d_tmp, tb, st));
  IR_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tb, d_sl, d_sl, nq, st));
  note_launch(); ir_total_kernel<<<1, 1, 0, st>>>(d_tot + 1, d_sl, nq, d_tot);
  IR_CUDA(cudaGetLastError());
  int64_t total = 0;
  IR_CUDA(cudaMemcpyAsync(&total, d_tot, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  IR_CUDA(cudaStreamSynchronize(st));
  IR_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_slc), sizeof(int32_t) * (total > 0 ? total : 1), st));
  IR_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_pos), sizeof(int64_t) * (total + 1), st));
  IR_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_stage),
                          sizeof(int32_t) * (size_t)(total > 0 ? total : 1) * kIrSlice, st));
  rs = t->hier ? ir_run<true>(t, ds.desc, d_docs, d_query, d_qoff, nq, d_sl, total, d_res_off,
                              d_res, d_stage, d_slc, d_pos, d_cnt, nullptr, st, false)
               : ir_run<false>(t, ds.desc, d_docs, d_query, d_qoff, nq, d_sl, total, d_res_off,
                               d_res, d_stage, d_slc, d_pos, d_cnt, nullptr, st, false);
  if (rs != RESET_OK) {
    cleanup();
    return rs;
  }
#undef IR_CUDA
  cleanup();
  return RESET_OK;
}

}  // extern "C"
