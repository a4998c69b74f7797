// Owner-grouped triangle counting: every probed table is read from HBM once,
// into shared memory, and the keys of all sets that probe it stream through.
//
// Same count as dynamic_triangle_count (triangle-count/TC.cu:128-190): for
// every oriented edge (u, v) the keys of the smaller row are looked up in the
// larger row's table (ties: u's keys in v's table, TC.cu:148-157) with the
// reference's bucket layout, hash and probe rule (search_in_hashtable,
// TC.cu:11-31), so rows with repeated entries give the reference's number.
//
// What changes is the order of the work.  Probing edge by edge costs every
// key a random 4-byte table read in HBM, which moves a whole 32-byte sector,
// from tables far larger than L2.  Here the edges are first grouped by the
// set whose table they probe -- its "owner", the larger row -- so
//   * each owner's table is staged once in shared memory: one 1-D bulk copy
//     (cp.async.bulk, the TMA engine) per slot plane, since plane k of set w
//     is len[w] contiguous ints at table + off[w] + k*bucket_num;
//   * the keys of its probers (whole CSR rows) stream through it with
//     128-bit loads; every lookup then reads shared memory only.
// HBM traffic per probe drops from ~4 B of key + a 32 B sector to ~4 B.
//
// Passes (all stream-ordered, no host synchronisation):
//   own_count_kernel    owner of every edge; probers per owner
//   CUB exclusive scan  group offsets
//   own_scatter_kernel  (row start, row length) of every edge's prober,
//                       grouped by owner
//   own_classify_kernel one of three bins per owner:
//     CTA    large groups (or tables above a warp's share of shared memory):
//            the whole CTA stages the table, its warps split the probers,
//            groups of more than kCtaSeg probers are cut into several units;
//     warp   a warp stages the table in its own region and walks the probers;
//     direct small groups, where staging costs more than it saves, and
//            tables too large for shared memory: probes go to the HBM table,
//            flattened across the lanes (thread granularity).
//   tc_owner_kernel     one persistent launch: CTA units, then warp owners,
//                       then direct owners, each from its own work counter.
#include <cub/cub.cuh>

#include <algorithm>

#include "common.cuh"
#include "probe_common.cuh"
#include "staged.cuh"

namespace rst {
namespace {

// ------------------------------------------------------------- passes ----

// Owner of edge (u, v) of the edge CSR: v unless u's key row is longer
// (TC.cu:148-157); the prober is the other end.  Rows (lengths and starts)
// come from the key CSR koff, which for plain triangle counting is the edge
// CSR itself and for an element shard its filtered rows.  ok = false for
// lanes past the end or bad ids.
struct EdgeOwner {
  int owner, prober_start, prober_len;
  bool ok;
};

__device__ __forceinline__ EdgeOwner edge_owner(const int32_t* __restrict__ eoff,
                                                const int32_t* __restrict__ ecols,
                                                const int32_t* __restrict__ chunk_row,
                                                const int32_t* __restrict__ koff, int n,
                                                int64_t me, int64_t c, int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t e64 = c * 32 + lane;
  const bool valid = e64 < me;
  const int e = (int)(valid ? e64 : me - 1);
  int u0 = __ldg(chunk_row + c);
  if ((unsigned)u0 >= (unsigned)n) u0 = 0;
  const int u = row_of_edge(eoff, n, u0, e);
  const int v = __ldg(ecols + e);
  EdgeOwner r{-1, 0, 0, false};
  if (!valid) return r;
  if ((unsigned)u >= (unsigned)n || (unsigned)v >= (unsigned)n) {
    atomicOr(status, kErrBadId);
    return r;
  }
  const int us = __ldg(koff + u), du = __ldg(koff + u + 1) - us;
  const int vs = __ldg(koff + v), dv = __ldg(koff + v + 1) - vs;
  const bool own_u = du > dv;
  r.owner = own_u ? u : v;
  r.prober_start = own_u ? vs : us;
  r.prober_len = own_u ? dv : du;
  r.ok = true;
  return r;
}

__global__ void __launch_bounds__(kOT)
    own_count_kernel(const int32_t* __restrict__ eoff, const int32_t* __restrict__ ecols,
                     const int32_t* __restrict__ chunk_row, const int32_t* __restrict__ koff,
                     int32_t n, int64_t m, int32_t* __restrict__ cnt,
                     int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t me = min(m, (int64_t)__ldg(eoff + n));
  const int64_t n_chunks = (me + 31) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_chunks;
       c += nw) {
    const EdgeOwner eo = edge_owner(eoff, ecols, chunk_row, koff, n, me, c, status);
    const unsigned grp = __match_any_sync(kFull, eo.ok ? eo.owner : -1);
    if (eo.ok && lane == __ffs(grp) - 1) atomicAdd(cnt + eo.owner, __popc(grp));
  }
}

__global__ void __launch_bounds__(kOT)
    own_scatter_kernel(const int32_t* __restrict__ eoff, const int32_t* __restrict__ ecols,
                       const int32_t* __restrict__ chunk_row, const int32_t* __restrict__ koff,
                       int32_t n, int64_t m, const int32_t* __restrict__ goff,
                       int32_t* __restrict__ left, int2* __restrict__ ent,
                       int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t me = min(m, (int64_t)__ldg(eoff + n));
  const int64_t n_chunks = (me + 31) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_chunks;
       c += nw) {
    const EdgeOwner eo = edge_owner(eoff, ecols, chunk_row, koff, n, me, c, status);
    const unsigned grp = __match_any_sync(kFull, eo.ok ? eo.owner : -1);
    const int leader = __ffs(grp) - 1;
    int top = 0;
    // `left` counts down from the group size: positions [left-k, left)
    if (eo.ok && lane == leader) top = atomicSub(left + eo.owner, __popc(grp));
    top = __shfl_sync(kFull, top, leader);
    if (eo.ok) {
      const int pos = top - __popc(grp) + __popc(grp & lanemask_lt());
      ent[__ldg(goff + eo.owner) + pos] = make_int2(eo.prober_start, eo.prober_len);
    }
  }
}

// Bin of every owner with a non-empty group (see the file comment).
// ctr[0] CTA units, ctr[1] warp owners, ctr[2] small direct owners,
// ctr[6] direct units.
__global__ void __launch_bounds__(kOT)
    own_classify_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                        const int2* __restrict__ ent, int32_t n, int b,
                        int2* __restrict__ units, int32_t* __restrict__ wlist,
                        int32_t* __restrict__ dlist, int2* __restrict__ dunits,
                        int32_t* __restrict__ ctr) {
  classify_owners(desc, goff, ent, n, b, units, wlist, dlist, dunits, ctr);
}

// Rounds of 32 key chunks a warp keeps in flight, and whether the next
// rounds' keys are loaded before the current ones are probed.
constexpr int kOwnerRounds = 2;
constexpr bool kOwnerPrefetch = false;
// Keys a lane loads per round (4 or 8).  8 (two 16-byte loads) pays the row
// search and chunk bookkeeping once per 8 keys: scale 24, b 1, 131 -> 120 ms.
constexpr int kOwnerChunk = 8;

// OWN: every owner's hits are also added to owner_hits[owner] (per-graph
// counts of a batch of disjoint graphs are sums over their vertex ranges).
template <bool HIER, int R, bool OWN = false>
__global__ void __launch_bounds__(kOT, 2)
    tc_owner_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                    const int2* __restrict__ ent, const int32_t* __restrict__ cols, int64_t m,
                    const int2* __restrict__ units, const int32_t* __restrict__ wlist,
                    const int32_t* __restrict__ dlist, const int2* __restrict__ dunits,
                    int32_t* __restrict__ ctr,
                    const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
                    unsigned long long* __restrict__ count,
                    unsigned long long* __restrict__ owner_hits, int32_t* __restrict__ status) {
  extern __shared__ __align__(128) int sm[];
  __shared__ __align__(8) uint64_t s_bar[kOW + 1];
  __shared__ int s_item, s_next;
  // pending-probe queues (keys only) of four rounds, kept over all the
  // batches a warp takes from one staged table and walked once three rounds'
  // worth is queued (or the table changes), so walks run with full warps
  constexpr int QCAP = 4 * kQueue;
  constexpr bool PF = kOwnerPrefetch;
  __shared__ int s_q[kOW][QCAP];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid <= kOW) mbar_init(&s_bar[tid]);
  fence_mbar_init();
  __syncthreads();
  unsigned long long hits = 0;
  uint32_t par_cta = 0, par_warp = 0;
  const int n_units = ctr[0], n_warp = ctr[1], n_direct = ctr[2], n_dunits = ctr[6];
  // this warp's hits since h0 credited to owner w (warp-collective)
  auto credit = [&](int w, unsigned long long h0) {
    if (OWN) {
      const unsigned long long d = warp_sum_u64(hits - h0);
      if (lane == 0 && d) atomicAdd(owner_hits + w, d);
    }
  };

  // ---- CTA units: the whole CTA stages one table, warps share its probers
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
    if (!ok) {  // a copy that never landed: report, let it drain, stop
      if (tid == 0) atomicOr(status, kErrStageTimeout);
      mbar_wait(&s_bar[kOW], par_cta ^ 1u);
      return;
    }
    const int g0 = __ldg(goff + unit.x) + unit.y * kCtaSeg;
    const int g1 = min(__ldg(goff + unit.x + 1), g0 + kCtaSeg);
    const unsigned long long h0 = hits;
    int nq = 0;
    for (;;) {
      int g = 0;
      if (lane == 0) g = g0 + atomicAdd(&s_next, kGrab);
      g = __shfl_sync(kFull, g, 0);
      if (g >= g1) break;
      hits += staged_keys<HIER, R, false, kGrab, QCAP, true, PF, kOwnerChunk>(
          ent + g, min(kGrab, g1 - g), cols, m, sm, lg, lg_max, b, status, s_q[warp], nullptr,
          nullptr, &nq);
    }
    if (nq) hits += walk_keys<HIER>(s_q[warp], nq, sm, lg, lg_max, b, status);
    credit(unit.x, h0);
    __syncthreads();
  }

  // ---- direct units: up to kDirSeg probers of one owner whose table stays
  // in HBM, 32 probers at a time, their probes flattened across the lanes
  for (;;) {
    int ui = 0;
    if (lane == 0) ui = atomicAdd(ctr + 7, 1);
    ui = __shfl_sync(kFull, ui, 0);
    if (ui >= n_dunits) break;
    const int2 unit = __ldg(dunits + ui);
    const int4 dw = __ldg(desc + unit.x);
    const int g0 = __ldg(goff + unit.x) + unit.y * kDirSeg;
    const int g1 = min(__ldg(goff + unit.x + 1), g0 + kDirSeg);
    const unsigned long long h0 = hits;
    for (int g = g0; g < g1; g += 32) {
      const int2 e = g + lane < g1 ? __ldg(ent + g + lane) : make_int2(0, 0);
      hits += flat_probe<HIER>(cols, m, table, e.y, e.x, desc_toff(dw), desc_lg(dw), lg_max,
                               bn, b, status, [](int) {});
    }
    credit(unit.x, h0);
  }

  // ---- warp owners: each warp stages a table in its own region
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
    const unsigned long long h0 = hits;
    int nq = 0;
    for (int g = g0; g < g1; g += 32)
      hits += staged_keys<HIER, R, false, 32, QCAP, true, PF, kOwnerChunk>(
          ent + g, min(32, g1 - g), cols, m, W, lg, lg_max, b, status, s_q[warp], nullptr,
          nullptr, &nq);
    if (nq) hits += walk_keys<HIER>(s_q[warp], nq, W, lg, lg_max, b, status);
    credit(w, h0);
  }

  // ---- direct owners: 32 owners per warp, their (owner, prober) pairs
  // flattened across the lanes, probes into the HBM tables flattened again
  for (;;) {
    int ci = 0;
    if (lane == 0) ci = atomicAdd(ctr + 5, 1);
    ci = __shfl_sync(kFull, ci, 0);
    const int64_t i = (int64_t)ci * 32 + lane;
    if ((int64_t)ci * 32 >= n_direct) break;
    int g0 = 0, P = 0, lg = 3, w = 0;
    int64_t toff = 0;
    if (i < n_direct) {
      w = __ldg(dlist + i);
      const int4 dw = __ldg(desc + w);
      g0 = __ldg(goff + w);
      P = __ldg(goff + w + 1) - g0;
      lg = desc_lg(dw);
      toff = desc_toff(dw);
    }
    int TP;
    const int Q = warp_excl_scan(P, &TP);
    // OWN: the queue (idle in this phase) holds, per pair lane, its owner
    // lane and, per owner lane, its hits
    int* pair_owner = s_q[warp];
    int* own_hits = s_q[warp] + 32;
    if (OWN) own_hits[lane] = 0;
    for (int base = 0; base < TP; base += 32) {
      const int f = base + lane;
      const int k = owner_lane(Q, f);
      const int kq = __shfl_sync(kFull, Q, k);
      const int kg = __shfl_sync(kFull, g0, k);
      const int klg = __shfl_sync(kFull, lg, k);
      const int64_t kt = __shfl_sync(kFull, toff, k);
      const int2 e = f < TP ? __ldg(ent + kg + (f - kq)) : make_int2(0, 0);
      if (OWN) {
        pair_owner[lane] = k;
        __syncwarp();
      }
      hits += flat_probe<HIER>(cols, m, table, e.y, e.x, kt, klg, lg_max, bn, b, status,
                               [&](int kk) {
                                 if (OWN) atomicAdd(own_hits + pair_owner[kk], 1);
                               });
      if (OWN) __syncwarp();
    }
    if (OWN && i < n_direct && own_hits[lane])
      atomicAdd(owner_hits + w, (unsigned long long)own_hits[lane]);
    if (OWN) __syncwarp();
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

int grid_stride_blocks(int64_t items_per_block_unit, int cap) {
  if (items_per_block_unit < 1) items_per_block_unit = 1;
  return (int)std::min<int64_t>(items_per_block_unit, cap);
}

}  // namespace

// Owner-grouped sum over the edges (u, v) of the edge CSR (eoff, ecols, me;
// echunk_rows its 32-edge chunk rows) of |K(u) ∩ K(v)|, K = the key CSR
// (koff, kcols, mk; kdesc its descriptors) that table t was built on.  For
// triangle counting both CSRs are the graph.  *count must already be zeroed.
reset_status tc_owner(const reset_table* t, const int4* kdesc, const int32_t* koff,
                      const int32_t* kcols, int64_t mk, const int32_t* eoff,
                      const int32_t* ecols, const int32_t* echunk_rows, int64_t me,
                      unsigned long long* count, cudaStream_t st,
                      unsigned long long* owner_hits) {
  const int64_t n = t->n;
  const int64_t m = me;
  if (n == 0 || me == 0 || mk == 0) return RESET_OK;
  if (mk > INT32_MAX - 16)
    return arg_fail("the owner-grouped count takes at most 2^31 - 17 keys");
  // scratch, one allocation: cnt/left, goff, ent, units, wlist, dlist, dunits,
  // ctr, CUB
  size_t cub_bytes = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int32_t*)nullptr,
                                         (int32_t*)nullptr, (int)(n + 1), st));
  const int64_t max_units = n + m / kCtaSeg + 1, max_dunits = n + m / kDirSeg + 1;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t sz_cnt = al(sizeof(int32_t) * (n + 1)), sz_goff = sz_cnt;
  const size_t sz_ent = al(sizeof(int2) * m), sz_units = al(sizeof(int2) * max_units);
  const size_t sz_list = al(sizeof(int32_t) * n), sz_ctr = al(sizeof(int32_t) * 8);
  const size_t sz_dunits = al(sizeof(int2) * max_dunits);
  const size_t total = sz_cnt + sz_goff + sz_ent + sz_units + 2 * sz_list + sz_dunits +
                       sz_ctr + al(cub_bytes);
  char* base = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&base), total, st));
  char* p = base;
  int32_t* cnt = reinterpret_cast<int32_t*>(p); p += sz_cnt;
  int32_t* goff = reinterpret_cast<int32_t*>(p); p += sz_goff;
  int2* ent = reinterpret_cast<int2*>(p); p += sz_ent;
  int2* units = reinterpret_cast<int2*>(p); p += sz_units;
  int32_t* wlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  int32_t* dlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  int2* dunits = reinterpret_cast<int2*>(p); p += sz_dunits;
  int32_t* ctr = reinterpret_cast<int32_t*>(p); p += sz_ctr;
  void* cub_tmp = p;

  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 8, st);
  const int sms = sm_count();
  const int64_t chunks = (m + 31) / 32;
  const int g_edges = grid_stride_blocks((chunks + kOW - 1) / kOW, sms * 8);
  if (e == cudaSuccess) {
    note_launch();
    own_count_kernel<<<g_edges, kOT, 0, st>>>(eoff, ecols, echunk_rows, koff, t->n, me, cnt,
                                              t->d_status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, cnt, goff, (int)(n + 1), st);
  if (e == cudaSuccess) {
    note_launch();
    own_scatter_kernel<<<g_edges, kOT, 0, st>>>(eoff, ecols, echunk_rows, koff, t->n, me, goff,
                                                cnt, ent, t->d_status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    note_launch();
    own_classify_kernel<<<grid_stride_blocks((n + kOT - 1) / kOT, sms * 8), kOT, 0, st>>>(
        kdesc, goff, ent, t->n, t->bucket, units, wlist, dlist, dunits, ctr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const size_t smem = sizeof(int) * kCtaTab;
    const bool own = owner_hits != nullptr;
#define OWN_K(H, O) tc_owner_kernel<H, kOwnerRounds, O>
    const void* k = t->hier ? (own ? (const void*)OWN_K(true, true) : (const void*)OWN_K(true, false))
                            : (own ? (const void*)OWN_K(false, true)
                                   : (const void*)OWN_K(false, false));
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kOT, smem);
    if (e == cudaSuccess) {
      const int grid = sms * (per_sm > 0 ? per_sm : 1);
      note_launch();
#define OWN_LAUNCH(H, O)                                                                   \
  OWN_K(H, O)<<<grid, kOT, smem, st>>>(kdesc, goff, ent, kcols, mk, units, wlist, dlist,    \
                                       dunits, ctr, t->d_table, t->bucket_num, t->bucket,  \
                                       t->lg_max, count, owner_hits, t->d_status)
      if (t->hier) {
        if (own) OWN_LAUNCH(true, true); else OWN_LAUNCH(true, false);
      } else {
        if (own) OWN_LAUNCH(false, true); else OWN_LAUNCH(false, false);
      }
#undef OWN_LAUNCH
#undef OWN_K
      e = cudaGetLastError();
    }
  }
  cudaFreeAsync(base, st);
  if (e != cudaSuccess) return cuda_fail(e, "owner-grouped TC", __FILE__, __LINE__);
  return RESET_OK;
}

}  // namespace rst

using namespace rst;

extern "C" reset_status reset_tc_count_batch(const reset_table* t, const int32_t* d_off,
                                             const int32_t* d_cols, int64_t m,
                                             const int32_t* d_graph_off, int32_t n_graphs,
                                             uint64_t* d_counts, reset_stream_t stream) {
  if (!t || !d_counts || !d_graph_off) return arg_fail("NULL table, graph offsets or counts");
  if (n_graphs < 1) return arg_fail("n_graphs must be >= 1");
  if (m < 0 || m > INT32_MAX - 16) return arg_fail("m out of range");
  if (m > 0 && (!d_cols || !d_off)) return arg_fail("NULL offsets or cols");
  if ((reinterpret_cast<uintptr_t>(d_cols) & 15) != 0)
    return arg_fail("reset_tc_count_batch needs a 16-byte aligned column array");
  if (d_off != t->build_off || m != t->m)
    return arg_fail("d_off/m must be the CSR the table was built on");
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(uint64_t) * (size_t)n_graphs, st));
  if (m == 0 || t->n == 0) return RESET_OK;
  size_t cub_bytes = 0;
  RST_CUDA(cub::DeviceSegmentedReduce::Sum(nullptr, cub_bytes, (unsigned long long*)nullptr,
                                           (unsigned long long*)nullptr, n_graphs, d_graph_off,
                                           d_graph_off + 1, st));
  const size_t own_bytes = (sizeof(unsigned long long) * ((size_t)t->n + 1) + 255) & ~(size_t)255;
  char* buf = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&buf), own_bytes + 256 + cub_bytes, st));
  auto* owner_hits = reinterpret_cast<unsigned long long*>(buf);
  auto* total = reinterpret_cast<unsigned long long*>(buf + own_bytes);
  cudaError_t e = cudaMemsetAsync(buf, 0, own_bytes + 256, st);
  reset_status s = RESET_OK;
  if (e == cudaSuccess)
    s = tc_owner(t, t->d_desc, d_off, d_cols, m, d_off, d_cols, t->d_chunk_row, m, total, st,
                 owner_hits);
  if (e == cudaSuccess && s == RESET_OK)
    e = cub::DeviceSegmentedReduce::Sum(buf + own_bytes + 256, cub_bytes, owner_hits,
                                        reinterpret_cast<unsigned long long*>(d_counts), n_graphs,
                                        d_graph_off, d_graph_off + 1, st);
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_fail(e, "reset_tc_count_batch", __FILE__, __LINE__);
  return s;
}
