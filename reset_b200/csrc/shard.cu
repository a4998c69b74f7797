// Element-modulo sharding (multi-GPU/tc-multi-GPU/main.cu:113-137,
// multi-GPU/sss-multi-GPU/main.cu:120-160): shard g of G keeps, in every
// row, the elements x with x % G == g.  Every intersection splits exactly
// over the shards, |A ∩ B| = sum_g |A_g ∩ B_g| (for rows without repeated
// entries), so G devices -- or G passes on one device, as the reference
// runs them -- each build the tables of one shard and probe every pair of
// the full pair list; partial triangle counts add up, partial pair
// intersections add up and are decided afterwards with the full set sizes.
//
//   reset_csr_shard      the shard's rows (flag, CUB scan, scatter)
//   reset_tc_count_shard sum over the edges of the full CSR of
//                        |K_g(u) ∩ K_g(v)| (owner-grouped count, tc_owner.cu)
//   reset_sss_decide     the integer Jaccard decision from summed partials
#include <cub/cub.cuh>

#include "common.cuh"

namespace rst {
namespace {

constexpr int kT = 256;

__global__ void shard_flag_kernel(const int32_t* __restrict__ cols, int64_t m, int32_t G,
                                  int32_t g, int32_t* __restrict__ keep) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x)
    keep[e] = (__ldg(cols + e) % G) == g;  // C remainder: negative ids never match
}

__global__ void shard_scatter_kernel(const int32_t* __restrict__ cols, int64_t m,
                                     const int32_t* __restrict__ keep,
                                     const int32_t* __restrict__ pos,
                                     int32_t* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x)
    if (keep[e]) out[pos[e]] = __ldg(cols + e);
}

__global__ void shard_offsets_kernel(const int32_t* __restrict__ off, int32_t n,
                                     const int32_t* __restrict__ pos,
                                     int32_t* __restrict__ off_out, int64_t* __restrict__ m_out) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u <= n;
       u += (int64_t)gridDim.x * blockDim.x) {
    off_out[u] = pos[__ldg(off + u)];
    if (u == n && m_out) *m_out = pos[__ldg(off + n)];
  }
}

__global__ void sss_decide_kernel(const int32_t* __restrict__ off, int32_t n,
                                  const int32_t* __restrict__ pa,
                                  const int32_t* __restrict__ pb, int64_t np,
                                  const int32_t* __restrict__ inter, int32_t num, int32_t den,
                                  uint8_t* __restrict__ flags, int32_t* __restrict__ status) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int a = __ldg(pa + p), q = __ldg(pb + p);
    if ((unsigned)a >= (unsigned)n || (unsigned)q >= (unsigned)n) {
      if (status) atomicOr(status, kErrBadId);
      flags[p] = 0;
      continue;
    }
    const int64_t I = __ldg(inter + p);
    const int64_t U = (int64_t)(__ldg(off + a + 1) - __ldg(off + a)) +
                      (__ldg(off + q + 1) - __ldg(off + q)) - I;
    flags[p] = (uint8_t)(U > 0 && (int64_t)den * I >= (int64_t)num * U);
  }
}

int blocks_for(int64_t items) {
  const int64_t b = (items + kT - 1) / kT;
  const int cap = sm_count() * 8;
  return (int)(b < 1 ? 1 : (b < cap ? b : cap));
}

}  // namespace
}  // namespace rst

using namespace rst;

extern "C" {

reset_status reset_csr_shard(const int32_t* d_off, const int32_t* d_cols, int32_t n, int64_t m,
                             int32_t shards, int32_t shard, int32_t* d_off_out,
                             int32_t* d_cols_out, int64_t* d_m_out, reset_stream_t stream) {
  if (n < 0 || m < 0 || m > INT32_MAX - 1) return arg_fail("n or m out of range");
  if (shards < 1 || shard < 0 || shard >= shards) return arg_fail("shard must be in [0, shards)");
  if (!d_off || !d_off_out || (m > 0 && (!d_cols || !d_cols_out)))
    return arg_fail("NULL offsets or columns");
  cudaStream_t st = as_stream(stream);
  size_t cub_bytes = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int32_t*)nullptr,
                                         (int32_t*)nullptr, (int)(m + 1), st));
  const size_t a = ((size_t)(m + 1) * 4 + 255) & ~(size_t)255;
  char* buf = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&buf), 2 * a + cub_bytes, st));
  int32_t* keep = reinterpret_cast<int32_t*>(buf);
  int32_t* pos = reinterpret_cast<int32_t*>(buf + a);
  cudaError_t e = cudaMemsetAsync(keep + m, 0, sizeof(int32_t), st);
  if (e == cudaSuccess && m > 0) {
    note_launch();
    shard_flag_kernel<<<blocks_for(m), kT, 0, st>>>(d_cols, m, shards, shard, keep);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(buf + 2 * a, cub_bytes, keep, pos, (int)(m + 1), st);
  if (e == cudaSuccess && m > 0) {
    note_launch();
    shard_scatter_kernel<<<blocks_for(m), kT, 0, st>>>(d_cols, m, keep, pos, d_cols_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    note_launch();
    shard_offsets_kernel<<<blocks_for((int64_t)n + 1), kT, 0, st>>>(d_off, n, pos, d_off_out,
                                                                   d_m_out);
    e = cudaGetLastError();
  }
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_fail(e, "reset_csr_shard", __FILE__, __LINE__);
  return RESET_OK;
}

reset_status reset_tc_count_shard(const reset_table* t, const int32_t* d_key_off,
                                  const int32_t* d_key_cols, int64_t m_keys,
                                  const int32_t* d_edge_off, const int32_t* d_edge_cols,
                                  int64_t m_edges, uint64_t* d_count, reset_stream_t stream) {
  if (!t || !d_count) return arg_fail("NULL table or count");
  if (m_keys < 0 || m_keys > INT32_MAX || m_edges < 0 || m_edges > INT32_MAX)
    return arg_fail("m out of range");
  if (!d_key_off || !d_edge_off || (m_keys > 0 && !d_key_cols) ||
      (m_edges > 0 && !d_edge_cols))
    return arg_fail("NULL offsets or columns");
  if ((reinterpret_cast<uintptr_t>(d_key_cols) & 15) != 0)
    return arg_fail("the key column array must be 16-byte aligned");
  cudaStream_t st = as_stream(stream);
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m_keys == 0 || m_edges == 0 || t->n == 0) return RESET_OK;
  const int4* kdesc = t->d_desc;
  int4* owned_desc = nullptr;
  if (d_key_off != t->build_off) {
    RST_CHECK(make_desc(t, d_key_off, &owned_desc, st));
    kdesc = owned_desc;
  }
  int32_t* rows = nullptr;
  reset_status s = make_chunk_rows(d_edge_off, t->n, m_edges, &rows, st);
  if (s == RESET_OK)
    s = tc_owner(t, kdesc, d_key_off, d_key_cols, m_keys, d_edge_off, d_edge_cols, rows, m_edges,
                 reinterpret_cast<unsigned long long*>(d_count), st);
  if (rows) cudaFreeAsync(rows, st);
  if (owned_desc) cudaFreeAsync(owned_desc, st);
  return s;
}

reset_status reset_sss_decide(const int32_t* d_off, int32_t n, const int32_t* d_pair_a,
                              const int32_t* d_pair_b, int64_t npairs, const int32_t* d_inter,
                              int32_t num, int32_t den, uint8_t* d_flags,
                              int32_t* d_status_bits, reset_stream_t stream) {
  if (npairs < 0) return arg_fail("negative pair count");
  if (npairs == 0) return RESET_OK;
  if (!d_off || !d_pair_a || !d_pair_b || !d_inter || !d_flags) return arg_fail("NULL pointer");
  if (den <= 0 || num < 0) return arg_fail("threshold num/den");
  cudaStream_t st = as_stream(stream);
  note_launch();
  sss_decide_kernel<<<blocks_for(npairs), kT, 0, st>>>(d_off, n, d_pair_a, d_pair_b, npairs,
                                                      d_inter, num, den, d_flags, d_status_bits);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

}  // extern "C"
