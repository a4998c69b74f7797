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

namespace rst {
namespace {

constexpr int kOT = 256;             // threads per CTA
constexpr int kOW = kOT / 32;        // warps per CTA
constexpr int kCtaTab = 24576;       // ints of shared memory per CTA (96 KB)
constexpr int kWarpTab = kCtaTab / kOW;  // a warp's region (3072 ints)
constexpr int kCtaSeg = 512;         // probers per CTA work unit
constexpr int kBigGroup = 256;       // groups above this are CTA work
constexpr int kCtaWork = 32768;      // probes that make a smaller group CTA work
constexpr int kWaitLimit = 1 << 22;  // polls of a bulk-copy barrier before giving up

// ------------------------------------------------------- bulk copies ------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory before
// later bulk copies into it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity`; false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Issues the bulk copies of set w's table (b planes of 1 << lg ints) into S.
__device__ __forceinline__ void stage_table(int* S, const int32_t* __restrict__ table,
                                            int64_t toff, int lg, int64_t bn, int b,
                                            uint64_t* bar) {
  const int L = 1 << lg;
  const uint32_t plane = (uint32_t)L * 4u;
  fence_proxy_async_smem();
  mbar_expect_tx(bar, plane * (uint32_t)b);
  for (int k = 0; k < b; ++k) bulk_g2s(S + (int64_t)k * L, table + toff + k * bn, plane, bar);
}

// -------------------------------------------------- shared-memory probe --

// Continues search_in_hashtable (TC.cu:11-31) in a staged table (plane k at
// S + k*L) after slot 0 of bucket h held another key.  Same bound as
// probe_key (the whole table).
__device__ __forceinline__ unsigned smem_walk(int x, const int* S, int L, int h, int b,
                                              int32_t* status) {
  int k = 1;
  const int cap = L * b;
  for (int t = 1; t < cap; ++t) {
    if (k == b) {
      k = 0;
      h = (h + 1) & (L - 1);
    }
    const int s = S[k * L + h];
    if (s == x) return 1;
    if (s == -1) return 0;
    ++k;
  }
  atomicOr(status, kErrProbeLimit);
  return 0;
}

// The keys of up to 32 probers (lane i: ent[i] = {row start, row length}
// in cols) looked up in one staged table.  The rows' 16-byte chunks are
// flattened across the lanes (round r: lane i loads chunk 32r+i of the
// concatenation, owner found by a shuffle binary search) and R rounds are in
// flight at once.  Returns this lane's hits.
template <bool HIER, int R>
__device__ __forceinline__ unsigned staged_keys(const int2* __restrict__ ent, int cnt,
                                                const int32_t* __restrict__ cols, int64_t m,
                                                const int* S, int lg, int lg_max, int b,
                                                int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int2 e = lane < cnt ? __ldg(ent + lane) : make_int2(0, 0);
  const int64_t end = (int64_t)e.x + e.y;
  const int nc = e.y > 0 ? (int)(((end + 3) >> 2) - (e.x >> 2)) : 0;
  int total;
  const int P = warp_excl_scan(nc, &total);
  const int L = 1 << lg;
  const unsigned hmask = HIER ? ((1u << lg_max) - 1u) : (unsigned)(L - 1);
  const int hsh = HIER ? (lg_max - lg) : 0;
  const int4* __restrict__ cols4 = reinterpret_cast<const int4*>(cols);
  const int64_t full4 = m >> 2;  // chunks that lie wholly inside cols
  unsigned hits = 0;
  for (int base = 0; base < total; base += 32 * R) {
    int x[R][4];
    unsigned vm[R];  // bit j: element j of this lane's chunk belongs to the row
#pragma unroll
    for (int r = 0; r < R; ++r) {
      vm[r] = 0;
      x[r][0] = x[r][1] = x[r][2] = x[r][3] = 0;
      if (base + r * 32 < total) {  // warp-uniform
        const int f = base + r * 32 + lane;
        const int k = owner_lane(P, f);
        const int kp = __shfl_sync(kFull, P, k);
        const int kb = __shfl_sync(kFull, e.x, k);
        const int kd = __shfl_sync(kFull, e.y, k);
        if (f < total) {
          const int64_t c = (int64_t)(kb >> 2) + (f - kp);
          const int64_t i0 = c * 4;
          const int lo = (int)max((int64_t)kb - i0, (int64_t)0);
          const int hi = (int)min((int64_t)kb + kd - i0, (int64_t)4);
          vm[r] = ((1u << hi) - 1u) & ~((1u << lo) - 1u);
          if (c < full4) {
            const int4 q = __ldg(cols4 + c);
            x[r][0] = q.x;
            x[r][1] = q.y;
            x[r][2] = q.z;
            x[r][3] = q.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if ((vm[r] >> j) & 1u) x[r][j] = __ldg(cols + i0 + j);
          }
        }
      }
    }
    int h[R][4], s0[R][4];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        h[r][j] = (int)(((unsigned)x[r][j] & hmask) >> hsh);
        s0[r][j] = ((vm[r] >> j) & 1u) ? S[h[r][j]] : -1;
      }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!((vm[r] >> j) & 1u)) continue;
        if (s0[r][j] == x[r][j]) {
          ++hits;
        } else if (s0[r][j] != -1) {
          hits += smem_walk(x[r][j], S, L, h[r][j], b, status);
        }
      }
  }
  return hits;
}

// ------------------------------------------------------------- passes ----

// Owner of edge (u, v): v unless u's row is longer (TC.cu:148-157); the
// prober is the other end.  ok = false for lanes past the end or bad ids.
struct EdgeOwner {
  int owner, prober_start, prober_len;
  bool ok;
};

__device__ __forceinline__ EdgeOwner edge_owner(const int32_t* __restrict__ off,
                                                const int32_t* __restrict__ cols,
                                                const int32_t* __restrict__ chunk_row, int n,
                                                int64_t me, int64_t c, int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t e64 = c * 32 + lane;
  const bool valid = e64 < me;
  const int e = (int)(valid ? e64 : me - 1);
  int u0 = __ldg(chunk_row + c);
  if ((unsigned)u0 >= (unsigned)n) u0 = 0;
  const int u = row_of_edge(off, n, u0, e);
  const int v = __ldg(cols + e);
  EdgeOwner r{-1, 0, 0, false};
  if (!valid) return r;
  if ((unsigned)u >= (unsigned)n || (unsigned)v >= (unsigned)n) {
    atomicOr(status, kErrBadId);
    return r;
  }
  const int us = __ldg(off + u), du = __ldg(off + u + 1) - us;
  const int vs = __ldg(off + v), dv = __ldg(off + v + 1) - vs;
  const bool own_u = du > dv;
  r.owner = own_u ? u : v;
  r.prober_start = own_u ? vs : us;
  r.prober_len = own_u ? dv : du;
  r.ok = true;
  return r;
}

__global__ void __launch_bounds__(kOT)
    own_count_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ cols,
                     const int32_t* __restrict__ chunk_row, int32_t n, int64_t m,
                     int32_t* __restrict__ cnt, int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_chunks;
       c += nw) {
    const EdgeOwner eo = edge_owner(off, cols, chunk_row, n, me, c, status);
    const unsigned grp = __match_any_sync(kFull, eo.ok ? eo.owner : -1);
    if (eo.ok && lane == __ffs(grp) - 1) atomicAdd(cnt + eo.owner, __popc(grp));
  }
}

__global__ void __launch_bounds__(kOT)
    own_scatter_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ cols,
                       const int32_t* __restrict__ chunk_row, int32_t n, int64_t m,
                       const int32_t* __restrict__ goff, int32_t* __restrict__ left,
                       int2* __restrict__ ent, int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n_chunks;
       c += nw) {
    const EdgeOwner eo = edge_owner(off, cols, chunk_row, n, me, c, status);
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
// ctr[0] CTA units, ctr[1] warp owners, ctr[2] direct owners.
__global__ void __launch_bounds__(kOT)
    own_classify_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                        const int2* __restrict__ ent, int32_t n, int b,
                        int2* __restrict__ units, int32_t* __restrict__ wlist,
                        int32_t* __restrict__ dlist, int32_t* __restrict__ ctr) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
    const int64_t w = base + threadIdx.x;
    int bin = -1, nunits = 0;
    if (w < n) {
      const int g0 = __ldg(goff + w), P = __ldg(goff + w + 1) - g0;
      if (P > 0) {
        const int64_t T = (int64_t)b << desc_lg(__ldg(desc + w));  // table ints
        bool big = P > kBigGroup;
        int64_t work = 0;
        if (!big) {
          for (int i = 0; i < P; ++i) work += __ldg(&ent[g0 + i].y);
          big = work >= kCtaWork;
        }
        // staging pays when the table has at most ~4 ints per probe
        const bool stage = T <= kCtaTab && (P > kBigGroup || T <= 4 * work);
        if (!stage) {
          bin = 2;
        } else if (big || T > kWarpTab) {
          bin = 0;
          nunits = (P + kCtaSeg - 1) / kCtaSeg;
        } else {
          bin = 1;
        }
      }
    }
    // warp-aggregated appends
    {
      int tot;
      const int pre = warp_excl_scan(bin == 0 ? nunits : 0, &tot);
      int b0 = 0;
      if (lane == 0 && tot) b0 = atomicAdd(ctr + 0, tot);
      b0 = __shfl_sync(kFull, b0, 0);
      for (int s = 0; s < nunits; ++s) units[b0 + pre + s] = make_int2((int)w, s);
    }
#pragma unroll
    for (int which = 1; which <= 2; ++which) {
      const unsigned bm = __ballot_sync(kFull, bin == which);
      int b0 = 0;
      if (lane == 0 && bm) b0 = atomicAdd(ctr + which, __popc(bm));
      b0 = __shfl_sync(kFull, b0, 0);
      if (bin == which) (which == 1 ? wlist : dlist)[b0 + __popc(bm & lanemask_lt())] = (int)w;
    }
  }
}

template <bool HIER, int R>
__global__ void __launch_bounds__(kOT, 2)
    tc_owner_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ goff,
                    const int2* __restrict__ ent, const int32_t* __restrict__ cols, int64_t m,
                    const int2* __restrict__ units, const int32_t* __restrict__ wlist,
                    const int32_t* __restrict__ dlist, int32_t* __restrict__ ctr,
                    const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
                    unsigned long long* __restrict__ count, int32_t* __restrict__ status) {
  extern __shared__ __align__(128) int sm[];
  __shared__ __align__(8) uint64_t s_bar[kOW + 1];
  __shared__ int s_item, s_next;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid <= kOW) mbar_init(&s_bar[tid]);
  fence_mbar_init();
  __syncthreads();
  unsigned long long hits = 0;
  uint32_t par_cta = 0, par_warp = 0;
  const int n_units = ctr[0], n_warp = ctr[1], n_direct = ctr[2];

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
    const bool ok = __syncthreads_and(mbar_wait(&s_bar[kOW], par_cta));
    par_cta ^= 1u;
    if (!ok) {  // a copy that never landed: report, let it drain, stop
      if (tid == 0) atomicOr(status, kErrStageTimeout);
      mbar_wait(&s_bar[kOW], par_cta ^ 1u);
      return;
    }
    const int g0 = __ldg(goff + unit.x) + unit.y * kCtaSeg;
    const int g1 = min(__ldg(goff + unit.x + 1), g0 + kCtaSeg);
    for (;;) {
      int g = 0;
      if (lane == 0) g = g0 + atomicAdd(&s_next, 32);
      g = __shfl_sync(kFull, g, 0);
      if (g >= g1) break;
      hits += staged_keys<HIER, R>(ent + g, min(32, g1 - g), cols, m, sm, lg, lg_max, b, status);
    }
    __syncthreads();
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
    const bool ok = __all_sync(kFull, mbar_wait(&s_bar[warp], par_warp));
    par_warp ^= 1u;
    if (!ok) {
      if (lane == 0) atomicOr(status, kErrStageTimeout);
      mbar_wait(&s_bar[warp], par_warp ^ 1u);
      return;
    }
    const int g0 = __ldg(goff + w), g1 = __ldg(goff + w + 1);
    for (int g = g0; g < g1; g += 32)
      hits += staged_keys<HIER, R>(ent + g, min(32, g1 - g), cols, m, W, lg, lg_max, b, status);
  }

  // ---- direct owners: 32 owners per warp, their (owner, prober) pairs
  // flattened across the lanes, probes into the HBM tables flattened again
  for (;;) {
    int ci = 0;
    if (lane == 0) ci = atomicAdd(ctr + 5, 1);
    ci = __shfl_sync(kFull, ci, 0);
    const int64_t i = (int64_t)ci * 32 + lane;
    if ((int64_t)ci * 32 >= n_direct) break;
    int g0 = 0, P = 0, lg = 3;
    int64_t toff = 0;
    if (i < n_direct) {
      const int w = __ldg(dlist + i);
      const int4 dw = __ldg(desc + w);
      g0 = __ldg(goff + w);
      P = __ldg(goff + w + 1) - g0;
      lg = desc_lg(dw);
      toff = desc_toff(dw);
    }
    int TP;
    const int Q = warp_excl_scan(P, &TP);
    for (int base = 0; base < TP; base += 32) {
      const int f = base + lane;
      const int k = owner_lane(Q, f);
      const int kq = __shfl_sync(kFull, Q, k);
      const int kg = __shfl_sync(kFull, g0, k);
      const int klg = __shfl_sync(kFull, lg, k);
      const int64_t kt = __shfl_sync(kFull, toff, k);
      const int2 e = f < TP ? __ldg(ent + kg + (f - kq)) : make_int2(0, 0);
      hits += flat_probe<HIER>(cols, m, table, e.y, e.x, kt, klg, lg_max, bn, b, status,
                               [](int) {});
    }
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

int grid_stride_blocks(int64_t items_per_block_unit, int cap) {
  if (items_per_block_unit < 1) items_per_block_unit = 1;
  return (int)std::min<int64_t>(items_per_block_unit, cap);
}

}  // namespace

// Owner-grouped count of the CSR (d_off, d_cols, m) against table t; desc
// and chunk_rows belong to d_off.  *count must already be zeroed.
reset_status tc_owner(const reset_table* t, const int4* desc, const int32_t* d_off,
                      const int32_t* d_cols, const int32_t* chunk_rows, int64_t m,
                      unsigned long long* count, cudaStream_t st) {
  const int64_t n = t->n;
  if (n == 0 || m == 0) return RESET_OK;
  // scratch, one allocation: cnt/left, goff, ent, units, wlist, dlist, ctr, CUB
  size_t cub_bytes = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int32_t*)nullptr,
                                         (int32_t*)nullptr, (int)(n + 1), st));
  const int64_t max_units = n + m / kCtaSeg + 1;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t sz_cnt = al(sizeof(int32_t) * (n + 1)), sz_goff = sz_cnt;
  const size_t sz_ent = al(sizeof(int2) * m), sz_units = al(sizeof(int2) * max_units);
  const size_t sz_list = al(sizeof(int32_t) * n), sz_ctr = al(sizeof(int32_t) * 8);
  const size_t total = sz_cnt + sz_goff + sz_ent + sz_units + 2 * sz_list + sz_ctr +
                       al(cub_bytes);
  char* base = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&base), total, st));
  char* p = base;
  int32_t* cnt = reinterpret_cast<int32_t*>(p); p += sz_cnt;
  int32_t* goff = reinterpret_cast<int32_t*>(p); p += sz_goff;
  int2* ent = reinterpret_cast<int2*>(p); p += sz_ent;
  int2* units = reinterpret_cast<int2*>(p); p += sz_units;
  int32_t* wlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  int32_t* dlist = reinterpret_cast<int32_t*>(p); p += sz_list;
  int32_t* ctr = reinterpret_cast<int32_t*>(p); p += sz_ctr;
  void* cub_tmp = p;

  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 8, st);
  const int sms = sm_count();
  const int64_t chunks = (m + 31) / 32;
  const int g_edges = grid_stride_blocks((chunks + kOW - 1) / kOW, sms * 8);
  if (e == cudaSuccess) {
    note_launch();
    own_count_kernel<<<g_edges, kOT, 0, st>>>(d_off, d_cols, chunk_rows, t->n, m, cnt,
                                              t->d_status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, cnt, goff, (int)(n + 1), st);
  if (e == cudaSuccess) {
    note_launch();
    own_scatter_kernel<<<g_edges, kOT, 0, st>>>(d_off, d_cols, chunk_rows, t->n, m, goff, cnt,
                                                ent, t->d_status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    note_launch();
    own_classify_kernel<<<grid_stride_blocks((n + kOT - 1) / kOT, sms * 8), kOT, 0, st>>>(
        desc, goff, ent, t->n, t->bucket, units, wlist, dlist, ctr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const size_t smem = sizeof(int) * kCtaTab;
    const void* k = t->hier ? (const void*)tc_owner_kernel<true, 4>
                            : (const void*)tc_owner_kernel<false, 4>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kOT, smem);
    if (e == cudaSuccess) {
      const int grid = sms * (per_sm > 0 ? per_sm : 1);
      note_launch();
      if (t->hier)
        tc_owner_kernel<true, 4><<<grid, kOT, smem, st>>>(
            desc, goff, ent, d_cols, m, units, wlist, dlist, ctr, t->d_table, t->bucket_num,
            t->bucket, t->lg_max, count, t->d_status);
      else
        tc_owner_kernel<false, 4><<<grid, kOT, smem, st>>>(
            desc, goff, ent, d_cols, m, units, wlist, dlist, ctr, t->d_table, t->bucket_num,
            t->bucket, t->lg_max, count, t->d_status);
      e = cudaGetLastError();
    }
  }
  cudaFreeAsync(base, st);
  if (e != cudaSuccess) return cuda_fail(e, "owner-grouped TC", __FILE__, __LINE__);
  return RESET_OK;
}

}  // namespace rst
