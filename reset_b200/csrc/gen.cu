// Seeded R-MAT graph generator on the device: the synthetic stand-in for the
// reference's graph datasets (graph500 sc18-20, SNAP graphs), which are not
// available here.
//
// Edge i draws 2^scale x 2^scale quadrants level by level from 16-bit fields
// of w_g = mix64(seed ^ mix64(8*i + g)) (four levels per 64-bit word, mix64
// the splitmix64 finaliser), quadrant a/b/c/d by integer thresholds on
// [0, 65536).  Vertex labels then go through a seeded bijection, as Graph500
// permutes the labels of its Kronecker graphs: raw R-MAT ids keep the
// quadrant bias in every bit (hubs at small ids), which would concentrate
// keys in a few buckets of any table that hashes by id bits.  The graph is
// then cleaned the way the reference's
// preprocessing does it (preprocess/preprocessor.py:158-210): symmetrised,
// self-loops and duplicates removed; for triangle counting each edge is kept
// once, oriented from the lower (degree, id) end to the higher one.  Rows
// come out sorted ascending.
#include <cub/cub.cuh>

#include "common.cuh"

namespace rst {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Seeded bijection of [0, 2^scale): vertex relabeling (Graph500 permutes
// the labels of its Kronecker graphs the same way).  Three rounds of
// multiply by an odd constant, xor-shift by ceil(scale/2), add a constant.
struct Relabel {
  uint32_t M[3], A[3], mask;
  int sh;
};

Relabel make_relabel(uint64_t seed, int scale);

__device__ __forceinline__ uint32_t relabel(const Relabel& r, uint32_t x) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    x = (x * r.M[i]) & r.mask;
    x ^= x >> r.sh;
    x = (x + r.A[i]) & r.mask;
  }
  return x;
}

__global__ void rmat_kernel(uint64_t seed, int scale, int64_t ne, int ta,
                            int tb, int tc, int do_relabel, Relabel rl,
                            uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t u = 0, v = 0;
    uint64_t w = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 3) == 0) w = mix64(seed ^ mix64((uint64_t)i * 8u + (uint64_t)(l >> 2)));
      const int r = (int)((w >> (16 * (l & 3))) & 0xFFFF);
      const uint32_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (do_relabel) {
      u = relabel(rl, u);
      v = relabel(rl, v);
    }
    if (u == v) {
      keys[2 * i] = keys[2 * i + 1] = ~0ull;
    } else {
      keys[2 * i] = ((uint64_t)u << 32) | v;
      keys[2 * i + 1] = ((uint64_t)v << 32) | u;
    }
  }
}

__global__ void degree_kernel(const uint64_t* __restrict__ keys, int64_t nk,
                              int32_t* __restrict__ deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&deg[keys[i] >> 32], 1);
}

__global__ void orient_kernel(const uint64_t* __restrict__ keys, int64_t nk,
                              const int32_t* __restrict__ deg, int oriented,
                              uint8_t* __restrict__ keep,
                              int32_t* __restrict__ outdeg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const int u = (int)(k >> 32), v = (int)(k & 0xFFFFFFFFu);
    bool kp = true;
    if (oriented) {
      const int du = deg[u], dv = deg[v];
      kp = du < dv || (du == dv && u < v);
    }
    keep[i] = kp;
    if (kp) atomicAdd(&outdeg[u], 1);
  }
}

__global__ void cols_kernel(const uint64_t* __restrict__ keys, int64_t nk,
                            int32_t* __restrict__ cols) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x)
    cols[i] = (int32_t)(keys[i] & 0xFFFFFFFFu);
}

uint64_t host_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

Relabel make_relabel(uint64_t seed, int scale) {
  Relabel r;
  r.mask = scale >= 32 ? 0xFFFFFFFFu : ((1u << scale) - 1u);
  r.sh = (scale + 1) / 2;
  for (int i = 0; i < 3; ++i) {
    r.M[i] = (uint32_t)host_mix64(seed ^ (0x5EC0DE00ull + 2 * i)) | 1u;
    r.A[i] = (uint32_t)host_mix64(seed ^ (0x5EC0DE01ull + 2 * i));
  }
  return r;
}

int gen_grid(int64_t items) {
  int64_t g = (items + 255) / 256, cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace
}  // namespace rst

using namespace rst;

extern "C" reset_status reset_gen_rmat(int32_t scale, int32_t edge_factor,
                                       uint64_t seed, double a, double b,
                                       double c, int32_t options,
                                       int32_t** d_off_out,
                                       int32_t** d_cols_out, int64_t* m_out,
                                       reset_stream_t stream) {
  if (!d_off_out || !d_cols_out || !m_out) return arg_fail("NULL output");
  if (scale < 1 || scale > 30 || edge_factor < 1)
    return arg_fail("scale must be in 1..30, edge_factor >= 1");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return arg_fail("R-MAT probabilities");
  const int32_t oriented = (options & RESET_GEN_SYMMETRIC) ? 0 : 1;
  const int do_relabel = (options & RESET_GEN_KEEP_IDS) ? 0 : 1;
  const int64_t n = (int64_t)1 << scale;
  const int64_t ne = (int64_t)edge_factor << scale;
  if (2 * ne > INT32_MAX) return arg_fail("too many edges for one pass");
  const int ta = (int)(a * 65536.0 + 0.5), tb = (int)((a + b) * 65536.0 + 0.5),
            tc = (int)((a + b + c) * 65536.0 + 0.5);
  cudaStream_t st = as_stream(stream);
  uint64_t *k0 = nullptr, *k1 = nullptr;
  int32_t *deg = nullptr, *outdeg = nullptr, *off = nullptr, *cols = nullptr;
  uint8_t* keep = nullptr;
  int64_t* d_cnt = nullptr;
  void* tmp = nullptr;
  reset_status rs = RESET_OK;
  auto cleanup = [&](bool ok) {
    cudaStreamSynchronize(st);
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(deg);
    cudaFree(outdeg);
    cudaFree(keep);
    cudaFree(d_cnt);
    cudaFree(tmp);
    if (!ok) {
      cudaFree(off);
      cudaFree(cols);
    }
  };
#define GEN_CUDA(call)                                                     \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      rs = cuda_fail(_e, #call, __FILE__, __LINE__);                       \
      cleanup(false);                                                      \
      return rs;                                                           \
    }                                                                      \
  } while (0)
  const int64_t nk = 2 * ne;
  GEN_CUDA(cudaMalloc(&k0, sizeof(uint64_t) * nk));
  GEN_CUDA(cudaMalloc(&k1, sizeof(uint64_t) * nk));
  GEN_CUDA(cudaMalloc(&d_cnt, sizeof(int64_t) * 2));
  note_launch(); rmat_kernel<<<gen_grid(ne), 256, 0, st>>>(seed, scale, ne, ta, tb, tc, do_relabel,
                                                        make_relabel(seed, scale), k0);
  GEN_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> db(k0, k1);
  size_t tb_sort = 0, tb_uniq = 0, tb_flag = 0, tb_scan = 0;
  GEN_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, db, (int)nk, 0, 32 + scale, st));
  GEN_CUDA(cub::DeviceSelect::Unique(nullptr, tb_uniq, k0, k1, d_cnt, (int)nk, st));
  GEN_CUDA(cub::DeviceSelect::Flagged(nullptr, tb_flag, k0, keep, k1, d_cnt, (int)nk, st));
  GEN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, outdeg, outdeg, (int)n + 1, st));
  size_t tbytes = tb_sort;
  if (tb_uniq > tbytes) tbytes = tb_uniq;
  if (tb_flag > tbytes) tbytes = tb_flag;
  if (tb_scan > tbytes) tbytes = tb_scan;
  GEN_CUDA(cudaMalloc(&tmp, tbytes));
  GEN_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb_sort, db, (int)nk, 0, 32 + scale, st));
  uint64_t* sorted = db.Current();
  uint64_t* other = db.Alternate();
  GEN_CUDA(cub::DeviceSelect::Unique(tmp, tb_uniq, sorted, other, d_cnt, (int)nk, st));
  int64_t nu = 0;
  {
    int32_t c32 = 0;
    GEN_CUDA(cudaMemcpyAsync(&c32, d_cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GEN_CUDA(cudaStreamSynchronize(st));
    nu = c32;
    uint64_t last = 0;
    if (nu > 0) {
      GEN_CUDA(cudaMemcpy(&last, other + nu - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost));
      if (last == ~0ull) --nu;  // the self-loop sentinel
    }
  }
  GEN_CUDA(cudaMalloc(&deg, sizeof(int32_t) * n));
  GEN_CUDA(cudaMalloc(&outdeg, sizeof(int32_t) * (n + 1)));
  GEN_CUDA(cudaMalloc(&keep, nu > 0 ? nu : 1));
  GEN_CUDA(cudaMemsetAsync(deg, 0, sizeof(int32_t) * n, st));
  GEN_CUDA(cudaMemsetAsync(outdeg, 0, sizeof(int32_t) * (n + 1), st));
  if (nu > 0) {
    note_launch(); degree_kernel<<<gen_grid(nu), 256, 0, st>>>(other, nu, deg);
    note_launch(); orient_kernel<<<gen_grid(nu), 256, 0, st>>>(other, nu, deg, oriented, keep, outdeg);
    GEN_CUDA(cudaGetLastError());
    GEN_CUDA(cub::DeviceSelect::Flagged(tmp, tb_flag, other, keep, sorted, d_cnt, (int)nu, st));
  } else {
    GEN_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int64_t), st));
  }
  GEN_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb_scan, outdeg, outdeg, (int)n + 1, st));
  int32_t m32 = 0;
  GEN_CUDA(cudaMemcpyAsync(&m32, d_cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  GEN_CUDA(cudaStreamSynchronize(st));
  const int64_t m = nu > 0 ? m32 : 0;
  GEN_CUDA(cudaMalloc(&off, sizeof(int32_t) * (n + 1)));
  GEN_CUDA(cudaMalloc(&cols, sizeof(int32_t) * (m > 0 ? m : 1)));
  GEN_CUDA(cudaMemcpyAsync(off, outdeg, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, st));
  if (m > 0) {
    note_launch(); cols_kernel<<<gen_grid(m), 256, 0, st>>>(sorted, m, cols);
    GEN_CUDA(cudaGetLastError());
  }
#undef GEN_CUDA
  cleanup(true);
  *d_off_out = off;
  *d_cols_out = cols;
  *m_out = m;
  return RESET_OK;
}
