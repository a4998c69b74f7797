// 4-clique counting on an oriented graph by multi-way hash-probe
// intersections: the depth-4 case of the clique DFS of SMOG
// (SMOG/SMOG_hie/subgraph_match_hie.cu:58-247, DFSKernelForClique), written
// over this library's tables.
//
// With edges oriented low -> high (degree, then id), every 4-clique
// {a < b < c < d} is found exactly once: from edge (a, b), the common
// out-neighbours W = N+(a) ∩ N+(b) contain c and d, and d ∈ W ∩ N+(c).
// So
//   count = sum over edges (u, v) of sum over w in W(u, v) of |W ∩ N+(w)|.
// One warp per edge (dynamic 1-edge work items): level 3 probes the smaller
// of N+(u), N+(v) into the other's table and compacts the hits W into the
// warp's scratch row (ballot/popc, first-set order); level 4 probes all of W
// into the table of each w in W.
#include <algorithm>

#include "probe_common.cuh"

namespace rst {
namespace {

constexpr int kCqThreads = 256;
constexpr int kCqWarps = kCqThreads / 32;

template <bool HIER>
__global__ void __launch_bounds__(kCqThreads)
    clique4_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ off,
                   const int32_t* __restrict__ cols,
                   const int32_t* __restrict__ chunk_row, int32_t n, int64_t m,
                   const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
                   int32_t* __restrict__ scratch, int32_t cap,
                   unsigned long long* __restrict__ count,
                   unsigned long long* __restrict__ cursor,
                   int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int32_t* W = scratch + gw * (int64_t)cap;
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  unsigned long long hits = 0;
  int u = 0;
  for (;;) {
    unsigned long long cc = 0;
    if (lane == 0) cc = atomicAdd(cursor, 1ull);
    const int64_t e = (int64_t)__shfl_sync(kFull, cc, 0);
    if (e >= me) break;
    // row of edge e: largest u with off[u] <= e, searched between the rows
    // of the 32-edge chunks around e (lane 0)
    if (lane == 0) {
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
    const int4 du = __ldg(desc + u), dv = __ldg(desc + v);
    const bool sw = du.y > dv.y;
    const int4 A = sw ? dv : du, Bd = sw ? du : dv;
    const int32_t* tb = table + desc_toff(Bd);
    const int blg = desc_lg(Bd);
    // level 3: W = A ∩ B, compacted into the warp's scratch row
    int nw = 0;
    for (int j0 = 0; j0 < A.y; j0 += 32) {
      const int j = j0 + lane;
      bool in = false;
      int x = 0;
      if (j < A.y) {
        x = __ldg(cols + A.x + j);
        in = probe_key<HIER>(x, tb, blg, lg_max, bn, b, status);
      }
      const unsigned msk = __ballot_sync(kFull, in);
      if (in) {
        const int pos = nw + __popc(msk & lt);
        if (pos < cap) W[pos] = x;
      }
      nw += __popc(msk);
    }
    if (nw > cap) {  // cannot happen when cap >= the largest out-degree
      if (lane == 0) atomicOr(status, kErrProbeLimit);
      continue;
    }
    __syncwarp();
    // level 4: for every w in W, |W ∩ N+(w)|
    for (int t = 0; t < nw; ++t) {
      const int w = W[t];
      const int4 dw = __ldg(desc + w);
      if (dw.y == 0) continue;
      const int32_t* tw = table + desc_toff(dw);
      const int wlg = desc_lg(dw);
      for (int j = lane; j < nw; j += 32)
        hits += probe_key<HIER>(W[j], tw, wlg, lg_max, bn, b, status);
    }
    __syncwarp();
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

// k-cliques, 3 <= k <= kMaxClique: SMOG's clique search
// (SMOG/SMOG_hie/subgraph_match_hie.cu:58-247) as a warp-level depth-first
// search over hash-probe intersections.  An edge (u, v) fixes two vertices;
// the candidates of the third are C0 = N+(u) ∩ N+(v); after picking w from
// C_j, the candidates of the next vertex are C_{j+1} = C_j ∩ N+(w) (the
// keys of C_j probed into w's table, hits compacted into the warp's scratch
// row of level j+1).  The last level is only counted: sum over w in C_j of
// |C_j ∩ N+(w)|.  Orientation orders every clique's vertices, so each is
// counted once.  Scratch: k-3 rows of `cap` ints per warp (levels 0..k-4).
constexpr int kMaxClique = 16;

template <bool HIER>
__global__ void __launch_bounds__(kCqThreads)
    clique_k_kernel(const int4* __restrict__ desc, const int32_t* __restrict__ off,
                    const int32_t* __restrict__ cols, const int32_t* __restrict__ chunk_row,
                    int32_t n, int64_t m, const int32_t* __restrict__ table, int64_t bn, int b,
                    int lg_max, int k, int32_t* __restrict__ scratch, int32_t cap,
                    unsigned long long* __restrict__ count,
                    unsigned long long* __restrict__ cursor, int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int levels = k > 3 ? k - 3 : 1;
  int32_t* Cbase = scratch + gw * (int64_t)cap * levels;
  const int64_t me = min(m, (int64_t)__ldg(off + n));
  const int64_t n_chunks = (me + 31) >> 5;
  unsigned long long hits = 0;
  int sz[kMaxClique], it[kMaxClique];
  int u = 0;
  for (;;) {
    unsigned long long cc = 0;
    if (lane == 0) cc = atomicAdd(cursor, 1ull);
    const int64_t e = (int64_t)__shfl_sync(kFull, cc, 0);
    if (e >= me) break;
    if (lane == 0) {  // row of edge e (as clique4_kernel)
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
    const int4 du = __ldg(desc + u), dv = __ldg(desc + v);
    const bool sw = du.y > dv.y;
    const int4 A = sw ? dv : du, Bd = sw ? du : dv;
    const int32_t* tb = table + desc_toff(Bd);
    const int blg = desc_lg(Bd);
    // level 0: C0 = N+(u) ∩ N+(v)
    int32_t* C0 = Cbase;
    int nw = 0;
    for (int j0 = 0; j0 < A.y; j0 += 32) {
      const int j = j0 + lane;
      bool in = false;
      int x = 0;
      if (j < A.y) {
        x = __ldg(cols + A.x + j);
        in = probe_key<HIER>(x, tb, blg, lg_max, bn, b, status);
      }
      const unsigned msk = __ballot_sync(kFull, in);
      if (in && k > 3) {
        const int pos = nw + __popc(msk & lt);
        if (pos < cap) C0[pos] = x;
      }
      nw += __popc(msk);
    }
    if (k == 3) {  // triangles through (u, v)
      if (lane == 0) hits += nw;
      continue;
    }
    if (nw > cap) {  // cannot happen when cap >= the largest out-degree
      if (lane == 0) atomicOr(status, kErrProbeLimit);
      continue;
    }
    __syncwarp();
    sz[0] = nw;
    it[0] = 0;
    int lv = 0;  // warp-uniform depth
    while (lv >= 0) {
      int32_t* C = Cbase + (int64_t)lv * cap;
      if (lv == k - 4) {  // last level: count, do not store
        for (int t = 0; t < sz[lv]; ++t) {
          const int4 dw = __ldg(desc + C[t]);
          if (dw.y == 0) continue;
          const int32_t* tw = table + desc_toff(dw);
          const int wlg = desc_lg(dw);
          for (int j = lane; j < sz[lv]; j += 32)
            hits += probe_key<HIER>(C[j], tw, wlg, lg_max, bn, b, status);
        }
        --lv;
        continue;
      }
      if (it[lv] >= sz[lv]) {
        --lv;
        continue;
      }
      const int4 dw = __ldg(desc + C[it[lv]]);
      ++it[lv];
      int32_t* D = C + cap;
      int nd = 0;
      if (dw.y > 0) {
        const int32_t* tw = table + desc_toff(dw);
        const int wlg = desc_lg(dw);
        for (int j0 = 0; j0 < sz[lv]; j0 += 32) {
          const int j = j0 + lane;
          bool in = false;
          int x = 0;
          if (j < sz[lv]) {
            x = C[j];
            in = probe_key<HIER>(x, tw, wlg, lg_max, bn, b, status);
          }
          const unsigned msk = __ballot_sync(kFull, in);
          if (in) D[nd + __popc(msk & lt)] = x;
          nd += __popc(msk);
        }
      }
      __syncwarp();
      if (nd == 0) continue;  // no clique grows from this pick
      ++lv;
      sz[lv] = nd;
      it[lv] = 0;
    }
    __syncwarp();
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

__global__ void max_degree_kernel(const int32_t* __restrict__ off, int32_t n,
                                  int32_t* __restrict__ out) {
  int mx = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    mx = max(mx, off[i + 1] - off[i]);
  for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// Largest row length of a CSR (d_off, n rows) into *out; synchronises `st`.
reset_status max_row_length(const int32_t* d_off, int32_t n, cudaStream_t st, int32_t* out) {
  *out = 0;
  int32_t* d_mx = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_mx), sizeof(int32_t), st));
  cudaError_t e = cudaMemsetAsync(d_mx, 0, sizeof(int32_t), st);
  if (e == cudaSuccess) {
    note_launch();
    max_degree_kernel<<<sm_count() * 4, 256, 0, st>>>(d_off, n, d_mx);
    e = cudaGetLastError();
  }
  int32_t mx = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&mx, d_mx, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(d_mx, st);
  if (e != cudaSuccess) return cuda_fail(e, "max degree", __FILE__, __LINE__);
  *out = mx;
  return RESET_OK;
}

}  // namespace
}  // namespace rst

using namespace rst;

extern "C" reset_status reset_clique4_count(const reset_table* t, const int32_t* d_off,
                                            const int32_t* d_cols, int64_t m,
                                            uint64_t* d_count, reset_stream_t stream) {
  if (!t || !d_count) return arg_fail("NULL table or count");
  if (m < 0 || m > INT32_MAX) return arg_fail("m out of range");
  if (m > 0 && (!d_off || !d_cols)) return arg_fail("NULL offsets or cols");
  if (d_off != t->build_off || m != t->m)
    return arg_fail("d_off/m must be the CSR the table was built on");
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m == 0 || t->n == 0) return RESET_OK;
  int32_t mx = 0;
  {
    const reset_status s = max_row_length(d_off, t->n, st, &mx);
    if (s != RESET_OK) return s;
  }
  const int32_t cap = mx > 0 ? mx : 1;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, t->hier ? (const void*)clique4_kernel<true> : (const void*)clique4_kernel<false>,
      kCqThreads, 0);
  if (per_sm < 1) per_sm = 1;
  const int64_t grid = std::min<int64_t>((int64_t)sm_count() * per_sm, (m + kCqWarps - 1) / kCqWarps);
  const int64_t warps = grid * kCqWarps;
  int32_t* d_scr = nullptr;
  unsigned long long* d_cur = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_scr), sizeof(int32_t) * warps * cap, st));
  cudaError_t e = scratch_malloc(reinterpret_cast<void**>(&d_cur), sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_cur, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    note_launch();
    if (t->hier)
      clique4_kernel<true><<<(int)grid, kCqThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num, t->bucket, t->lg_max,
          d_scr, cap, reinterpret_cast<unsigned long long*>(d_count), d_cur, t->d_status);
    else
      clique4_kernel<false><<<(int)grid, kCqThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num, t->bucket, t->lg_max,
          d_scr, cap, reinterpret_cast<unsigned long long*>(d_count), d_cur, t->d_status);
    e = cudaGetLastError();
  }
  cudaFreeAsync(d_scr, st);
  if (d_cur) cudaFreeAsync(d_cur, st);
  if (e != cudaSuccess) return cuda_fail(e, "clique4_kernel", __FILE__, __LINE__);
  return RESET_OK;
}

extern "C" reset_status reset_clique_count(const reset_table* t, const int32_t* d_off,
                                           const int32_t* d_cols, int64_t m, int32_t k,
                                           uint64_t* d_count, reset_stream_t stream) {
  if (!t || !d_count) return arg_fail("NULL table or count");
  if (k < 3 || k > kMaxClique) return arg_fail("k must be in 3..16");
  if (m < 0 || m > INT32_MAX) return arg_fail("m out of range");
  if (m > 0 && (!d_off || !d_cols)) return arg_fail("NULL offsets or cols");
  if (d_off != t->build_off || m != t->m)
    return arg_fail("d_off/m must be the CSR the table was built on");
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m == 0 || t->n == 0) return RESET_OK;
  int32_t mx = 0;
  {
    const reset_status s = max_row_length(d_off, t->n, st, &mx);
    if (s != RESET_OK) return s;
  }
  const int32_t cap = mx > 0 ? mx : 1;
  const void* kf = t->hier ? (const void*)clique_k_kernel<true> : (const void*)clique_k_kernel<false>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, kCqThreads, 0);
  if (per_sm < 1) per_sm = 1;
  const int64_t grid = std::min<int64_t>((int64_t)sm_count() * per_sm, (m + kCqWarps - 1) / kCqWarps);
  const int64_t warps = grid * kCqWarps;
  const int64_t levels = k > 3 ? k - 3 : 1;
  int32_t* d_scr = nullptr;
  unsigned long long* d_cur = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&d_scr),
                          sizeof(int32_t) * (size_t)warps * (size_t)cap * (size_t)levels, st));
  cudaError_t e = scratch_malloc(reinterpret_cast<void**>(&d_cur), sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_cur, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    note_launch();
    if (t->hier)
      clique_k_kernel<true><<<(int)grid, kCqThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num,
          t->bucket, t->lg_max, k, d_scr, cap, reinterpret_cast<unsigned long long*>(d_count),
          d_cur, t->d_status);
    else
      clique_k_kernel<false><<<(int)grid, kCqThreads, 0, st>>>(
          t->d_desc, d_off, d_cols, t->d_chunk_row, t->n, m, t->d_table, t->bucket_num,
          t->bucket, t->lg_max, k, d_scr, cap, reinterpret_cast<unsigned long long*>(d_count),
          d_cur, t->d_status);
    e = cudaGetLastError();
  }
  cudaFreeAsync(d_scr, st);
  if (d_cur) cudaFreeAsync(d_cur, st);
  if (e != cudaSuccess) return cuda_fail(e, "clique_k_kernel", __FILE__, __LINE__);
  return RESET_OK;
}
