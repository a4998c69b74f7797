// Owner-grouped set-similarity decisions: the pairs are grouped by the set
// whose table they probe, and each such table is read from HBM once, into
// shared memory.
//
// Same decisions as set_similarity_search_kernel
// (set-similarity-search/sss.cu:93-154): I = |A ∩ B| by looking up the keys
// of the smaller set in the larger set's table (ties: the first set's keys
// in the second set's table, sss.cu:108-115) with the reference's layout,
// hash and probe rule; U = |A| + |B| - I; similar when den*I >= num*U
// (exact) or, with the float rule, when (float)I / (float)U >= thr
// (sss.cu:139-141).
//
// The grouping and bins are those of the owner-grouped triangle count
// (tc_owner.cu): pair_count / CUB scan / pair_scatter put the (row start,
// row length) of every pair's probing set and the pair's index into its
// owner's group; the owners are binned into CTA units, warp owners and
// direct owners; one persistent kernel stages every CTA or warp owner's
// table with 1-D bulk copies and streams its probers' rows through it with
// 16-byte loads, counting hits per pair in shared memory.  The pair count
// may be read on the device (np_dev), so the whole sequence can be captured
// in a CUDA graph with scratch sized for a capacity.
#include <cub/cub.cuh>

#include <algorithm>

#include "common.cuh"
#include "probe_common.cuh"
#include "staged.cuh"

namespace rst {
namespace {

struct PairOwner {
  int owner, prober_start, prober_len;
  bool ok;
};

// Owner of pair p: the second set unless the first is larger (sss.cu:108-115).
__device__ __forceinline__ PairOwner pair_owner(const int4* __restrict__ desc, int n,
                                                const int32_t* __restrict__ pa,
                                                const int32_t* __restrict__ pb, int64_t p,
                                                int64_t np, int32_t* status,
                                                uint8_t* __restrict__ flags,
                                                int32_t* __restrict__ inter, bool report) {
  PairOwner r{-1, 0, 0, false};
  if (p >= np) return r;
  const int a = __ldg(pa + p), q = __ldg(pb + p);
  if ((unsigned)a >= (unsigned)n || (unsigned)q >= (unsigned)n) {
    if (report) {  // not grouped: decided here (not similar, no common keys)
      atomicOr(status, kErrBadId);
      flags[p] = 0;
      if (inter) inter[p] = 0;
    }
    return r;
  }
  const int4 da = __ldg(desc + a), dq = __ldg(desc + q);
  const bool sw = da.y > dq.y;
  const int4 A = sw ? dq : da;
  r.owner = sw ? a : q;
  r.prober_start = A.x;
  r.prober_len = A.y;
  r.ok = true;
  return r;
}

__global__ void __launch_bounds__(kOT)
    pair_count_kernel(const int4* __restrict__ desc, int32_t n, const int32_t* __restrict__ pa,
                      const int32_t* __restrict__ pb, int64_t np,
                      const int64_t* __restrict__ np_dev, int32_t* __restrict__ cnt,
                      uint8_t* __restrict__ flags, int32_t* __restrict__ inter,
                      int32_t* __restrict__ status) {
  if (np_dev) np = *np_dev;
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < np; base += stride) {
    const PairOwner po =
        pair_owner(desc, n, pa, pb, base + threadIdx.x, np, status, flags, inter, true);
    const unsigned grp = __match_any_sync(kFull, po.ok ? po.owner : -1);
    if (po.ok && lane == __ffs(grp) - 1) atomicAdd(cnt + po.owner, __popc(grp));
  }
}

__global__ void __launch_bounds__(kOT)
    pair_scatter_kernel(const int4* __restrict__ desc, int32_t n,
                        const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
                        int64_t np, const int64_t* __restrict__ np_dev,
                        const int32_t* __restrict__ goff, int32_t* __restrict__ left,
                        int2* __restrict__ ent, int32_t* __restrict__ pidx,
                        int32_t* __restrict__ status) {
  if (np_dev) np = *np_dev;
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < np; base += stride) {
    const int64_t p = base + threadIdx.x;
    const PairOwner po = pair_owner(desc, n, pa, pb, p, np, status, nullptr, nullptr, false);
    const unsigned grp = __match_any_sync(kFull, po.ok ? po.owner : -1);
    const int leader = __ffs(grp) - 1;
    int top = 0;
    if (po.ok && lane == leader) top = atomicSub(left + po.owner, __popc(grp));
    top = __shfl_sync(kFull, top, leader);
    if (po.ok) {
      const int pos = __ldg(goff + po.owner) + top - __popc(grp) + __popc(grp & lanemask_lt());
      ent[pos] = make_int2(po.prober_start, po.prober_len);
      pidx[pos] = (int32_t)p;
    }
  }
}

__global__ void __launch_bounds__(kOT)
    pair_classify_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                         const int2* __restrict__ ent, int32_t n, int b,
                         int2* __restrict__ units, int32_t* __restrict__ wlist,
                         int32_t* __restrict__ dlist, int2* __restrict__ dunits,
                         int32_t* __restrict__ ctr) {
  classify_owners(desc, goff, ent, n, b, units, wlist, dlist, dunits, ctr);
}

template <bool FLOAT_RULE>
__device__ __forceinline__ void decide(int64_t p, int I, int sa, int sb, int num, int den,
                                       float thr, uint8_t* __restrict__ flags,
                                       int32_t* __restrict__ inter) {
  const int64_t U = (int64_t)sa + sb - I;
  bool f;
  if (FLOAT_RULE) {
    f = ((float)I / (float)U) >= thr;  // sss.cu:139-140
  } else {
    f = U > 0 && (int64_t)den * I >= (int64_t)num * U;
  }
  flags[p] = (uint8_t)f;
  if (inter) inter[p] = I;
}

template <bool HIER, bool FLOAT_RULE, int R>
__global__ void __launch_bounds__(kOT, 2)
    sss_owner_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                     const int2* __restrict__ ent, const int32_t* __restrict__ pidx,
                     const int32_t* __restrict__ elems, int64_t m,
                     const int2* __restrict__ units, const int32_t* __restrict__ wlist,
                     const int32_t* __restrict__ dlist, const int2* __restrict__ dunits,
                     int32_t* __restrict__ ctr,
                     const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
                     int num, int den, float thr, uint8_t* __restrict__ flags,
                     int32_t* __restrict__ inter, int32_t* __restrict__ status) {
  extern __shared__ __align__(128) int sm[];
  __shared__ __align__(8) uint64_t s_bar[kOW + 1];
  __shared__ int s_item, s_next;
  __shared__ int s_qx[kOW][kQueue], s_qh[kOW][kQueue];
  __shared__ int s_cnt[kOW][32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid <= kOW) mbar_init(&s_bar[tid]);
  fence_mbar_init();
  __syncthreads();
  uint32_t par_cta = 0, par_warp = 0;
  const int n_units = ctr[0], n_warp = ctr[1], n_direct = ctr[2], n_dunits = ctr[6];
  int* C = s_cnt[warp];

  // one batch of up to 32 probers of owner w (length dw), table staged at S
  auto batch = [&](int g, int c, const int* S, int lg, int dw) {
    C[lane] = 0;
    __syncwarp();
    staged_keys<HIER, R, true>(ent + g, c, elems, m, S, lg, lg_max, b, status, s_qx[warp],
                               s_qh[warp], C);
    __syncwarp();
    if (lane < c)
      decide<FLOAT_RULE>(__ldg(pidx + g + lane), C[lane], __ldg(&ent[g + lane].y), dw, num,
                         den, thr, flags, inter);
    __syncwarp();
  };

  // ---- CTA units
  for (;;) {
    if (tid == 0) {
      s_item = atomicAdd(ctr + 3, 1);
      s_next = 0;
    }
    __syncthreads();
    const int ui = s_item;
    if (ui >= n_units) break;
    const int2 unit = __ldg(units + ui);
    const int4 dw = __ldg(desc + unit.x);
    const int lg = desc_lg(dw);
    if (tid == 0) stage_table(sm, table, desc_toff(dw), lg, bn, b, &s_bar[kOW]);
    const bool ok =
        __syncthreads_and(stage_wait(&s_bar[kOW], par_cta, sm, lg, b, tid == 0));
    par_cta ^= 1u;
    if (!ok) {
      if (tid == 0) atomicOr(status, kErrStageTimeout);
      mbar_wait(&s_bar[kOW], par_cta ^ 1u);
      return;
    }
    const int g0 = __ldg(goff + unit.x) + unit.y * kCtaSeg;
    const int g1 = min(__ldg(goff + unit.x + 1), g0 + kCtaSeg);
    for (;;) {
      int g = 0;
      if (lane == 0) g = g0 + atomicAdd(&s_next, kGrab);
      g = __shfl_sync(kFull, g, 0);
      if (g >= g1) break;
      batch(g, min(kGrab, g1 - g), sm, lg, dw.y);
    }
    __syncthreads();
  }

  // ---- direct units: up to kDirSeg pairs of one owner whose table stays in
  // HBM, 32 pairs at a time, their probes flattened across the lanes
  for (;;) {
    int ui = 0;
    if (lane == 0) ui = atomicAdd(ctr + 7, 1);
    ui = __shfl_sync(kFull, ui, 0);
    if (ui >= n_dunits) break;
    const int2 unit = __ldg(dunits + ui);
    const int4 dw = __ldg(desc + unit.x);
    const int g0 = __ldg(goff + unit.x) + unit.y * kDirSeg;
    const int g1 = min(__ldg(goff + unit.x + 1), g0 + kDirSeg);
    for (int g = g0; g < g1; g += 32) {
      const int gi = g + lane;
      const int2 e = gi < g1 ? __ldg(ent + gi) : make_int2(0, 0);
      C[lane] = 0;
      __syncwarp();
      flat_probe<HIER>(elems, m, table, e.y, e.x, desc_toff(dw), desc_lg(dw), lg_max, bn, b,
                       status, [&](int kk) { atomicAdd(C + kk, 1); });
      __syncwarp();
      if (gi < g1)
        decide<FLOAT_RULE>(__ldg(pidx + gi), C[lane], e.y, dw.y, num, den, thr, flags, inter);
      __syncwarp();
    }
  }

  // ---- warp owners
  int* W = sm + warp * kWarpTab;
  for (;;) {
    int wi = 0;
    if (lane == 0) wi = atomicAdd(ctr + 4, 1);
    wi = __shfl_sync(kFull, wi, 0);
    if (wi >= n_warp) break;
    const int w = __ldg(wlist + wi);
    const int4 dw = __ldg(desc + w);
    const int lg = desc_lg(dw);
    __syncwarp();
    if (lane == 0) stage_table(W, table, desc_toff(dw), lg, bn, b, &s_bar[warp]);
    const bool ok = __all_sync(kFull, stage_wait(&s_bar[warp], par_warp, W, lg, b, lane == 0));
    __syncwarp();
    par_warp ^= 1u;
    if (!ok) {
      if (lane == 0) atomicOr(status, kErrStageTimeout);
      mbar_wait(&s_bar[warp], par_warp ^ 1u);
      return;
    }
    const int g0 = __ldg(goff + w), g1 = __ldg(goff + w + 1);
    for (int g = g0; g < g1; g += 32) batch(g, min(32, g1 - g), W, lg, dw.y);
  }

  // ---- direct owners: 32 owners per warp, (owner, pair) flattened
  for (;;) {
    int ci = 0;
    if (lane == 0) ci = atomicAdd(ctr + 5, 1);
    ci = __shfl_sync(kFull, ci, 0);
    if ((int64_t)ci * 32 >= n_direct) break;
    const int64_t i = (int64_t)ci * 32 + lane;
    int g0 = 0, P = 0, lg = 3, dlen = 0;
    int64_t toff = 0;
    if (i < n_direct) {
      const int w = __ldg(dlist + i);
      const int4 dw = __ldg(desc + w);
      g0 = __ldg(goff + w);
      P = __ldg(goff + w + 1) - g0;
      lg = desc_lg(dw);
      toff = desc_toff(dw);
      dlen = dw.y;
    }
    int TP;
    const int Q = warp_excl_scan(P, &TP);
    for (int base = 0; base < TP; base += 32) {
      const int f = base + lane;
      const int k = owner_lane(Q, f);
      const int kq = __shfl_sync(kFull, Q, k);
      const int kg = __shfl_sync(kFull, g0, k);
      const int klg = __shfl_sync(kFull, lg, k);
      const int kdl = __shfl_sync(kFull, dlen, k);
      const int64_t kt = __shfl_sync(kFull, toff, k);
      const int gi = kg + (f - kq);
      const int2 e = f < TP ? __ldg(ent + gi) : make_int2(0, 0);
      C[lane] = 0;
      __syncwarp();
      flat_probe<HIER>(elems, m, table, e.y, e.x, kt, klg, lg_max, bn, b, status,
                       [&](int kk) { atomicAdd(C + kk, 1); });
      __syncwarp();
      if (f < TP) decide<FLOAT_RULE>(__ldg(pidx + gi), C[lane], e.y, kdl, num, den, thr,
                                     flags, inter);
      __syncwarp();
    }
  }
}

int blocks(int64_t items, int cap) {
  const int64_t b = (items + kOT - 1) / kOT;
  return (int)(b < 1 ? 1 : (b < cap ? b : cap));
}

}  // namespace

// Scratch for n sets and up to cap pairs, one stream-ordered allocation.
reset_status pair_owner_alloc(int32_t n, int64_t cap, PairOwnerScratch* s, cudaStream_t st) {
  *s = PairOwnerScratch{};
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, s->cub_bytes, (int32_t*)nullptr,
                                         (int32_t*)nullptr, (int)((int64_t)n + 1), st));
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const int64_t c = cap > 0 ? cap : 1;
  const size_t sz_n1 = al(sizeof(int32_t) * ((size_t)n + 1));
  const size_t sz_ent = al(sizeof(int2) * c), sz_pidx = al(sizeof(int32_t) * c);
  const size_t sz_units = al(sizeof(int2) * ((size_t)n + c / kCtaSeg + 1));
  const size_t sz_dunits = al(sizeof(int2) * ((size_t)n + c / kDirSeg + 1));
  const size_t sz_list = al(sizeof(int32_t) * ((size_t)n + 1)), sz_ctr = al(sizeof(int32_t) * 8);
  const size_t total = 2 * sz_n1 + sz_ent + sz_pidx + sz_units + sz_dunits + 2 * sz_list +
                       sz_ctr + al(s->cub_bytes);
  char* p = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&p), total, st));
  s->base = p;
  s->cnt = reinterpret_cast<int32_t*>(p); p += sz_n1;
  s->goff = reinterpret_cast<int32_t*>(p); p += sz_n1;
  s->ent = reinterpret_cast<int2*>(p); p += sz_ent;
  s->pidx = reinterpret_cast<int32_t*>(p); p += sz_pidx;
  s->units = reinterpret_cast<int2*>(p); p += sz_units;
  s->wlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  s->dlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  s->dunits = reinterpret_cast<int2*>(p); p += sz_dunits;
  s->ctr = reinterpret_cast<int32_t*>(p); p += sz_ctr;
  s->cub_tmp = p;
  return RESET_OK;
}

void pair_owner_free(PairOwnerScratch* s, cudaStream_t st) {
  if (s->base) cudaFreeAsync(s->base, st);
  *s = PairOwnerScratch{};
}

// Decisions (and sizes, if inter) for the pairs (pa[p], pb[p]), p < np (or
// < *np_dev when np_dev is set; cap bounds it) of sets described by desc
// (elems 16-byte aligned), with scratch from pair_owner_alloc(n, cap).  No
// allocation and no host synchronisation: capturable.
reset_status pair_owner_launch(const reset_table* t, const int4* desc, const int32_t* elems,
                               int64_t m, const int32_t* pa, const int32_t* pb, int64_t cap,
                               const int64_t* np_dev, bool float_rule, int32_t num, int32_t den,
                               float thr, uint8_t* flags, int32_t* inter,
                               const PairOwnerScratch& s, cudaStream_t st) {
  const int32_t n = t->n;
  if (m > INT32_MAX - 4) return arg_fail("owner-grouped pairs take at most 2^31 - 5 elements");
  const int sms = sm_count();
  RST_CUDA(cudaMemsetAsync(s.cnt, 0, sizeof(int32_t) * ((size_t)n + 1), st));
  RST_CUDA(cudaMemsetAsync(s.ctr, 0, sizeof(int32_t) * 8, st));
  const int gp = blocks(cap, sms * 8);
  note_launch();
  pair_count_kernel<<<gp, kOT, 0, st>>>(desc, n, pa, pb, cap, np_dev, s.cnt, flags, inter,
                                        t->d_status);
  RST_CUDA(cudaGetLastError());
  size_t cb = s.cub_bytes;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(s.cub_tmp, cb, s.cnt, s.goff, (int)((int64_t)n + 1), st));
  note_launch();
  pair_scatter_kernel<<<gp, kOT, 0, st>>>(desc, n, pa, pb, cap, np_dev, s.goff, s.cnt, s.ent,
                                          s.pidx, t->d_status);
  RST_CUDA(cudaGetLastError());
  note_launch();
  pair_classify_kernel<<<blocks(n, sms * 8), kOT, 0, st>>>(desc, s.goff, s.ent, n, t->bucket,
                                                           s.units, s.wlist, s.dlist, s.dunits,
                                                           s.ctr);
  RST_CUDA(cudaGetLastError());
  const size_t smem = sizeof(int) * kCtaTab;
#define SO_KERNEL(H, F) sss_owner_kernel<H, F, 4>
  const void* k = t->hier ? (float_rule ? (const void*)SO_KERNEL(true, true)
                                        : (const void*)SO_KERNEL(true, false))
                          : (float_rule ? (const void*)SO_KERNEL(false, true)
                                        : (const void*)SO_KERNEL(false, false));
  RST_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  RST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kOT, smem));
  const int grid = sms * (per_sm > 0 ? per_sm : 1);
  note_launch();
#define SO_LAUNCH(H, F)                                                                   \
  SO_KERNEL(H, F)<<<grid, kOT, smem, st>>>(desc, s.goff, s.ent, s.pidx, elems, m, s.units, \
                                           s.wlist, s.dlist, s.dunits, s.ctr, t->d_table, \
                                           t->bucket_num, t->bucket, t->lg_max, num, den,  \
                                           thr, flags, inter, t->d_status)
  if (t->hier) {
    if (float_rule) SO_LAUNCH(true, true); else SO_LAUNCH(true, false);
  } else {
    if (float_rule) SO_LAUNCH(false, true); else SO_LAUNCH(false, false);
  }
#undef SO_LAUNCH
#undef SO_KERNEL
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

// One call: scratch for np pairs, launch, stream-ordered free.
reset_status sss_owner(const reset_table* t, const int4* desc, const int32_t* elems, int64_t m,
                       const int32_t* pa, const int32_t* pb, int64_t np, bool float_rule,
                       int32_t num, int32_t den, float thr, uint8_t* flags, int32_t* inter,
                       cudaStream_t st) {
  if (np <= 0 || t->n == 0) return RESET_OK;
  PairOwnerScratch s;
  RST_CHECK(pair_owner_alloc(t->n, np, &s, st));
  reset_status r = pair_owner_launch(t, desc, elems, m, pa, pb, np, nullptr, float_rule, num,
                                     den, thr, flags, inter, s, st);
  pair_owner_free(&s, st);
  return r;
}

}  // namespace rst
