// Token sets for the set-similarity self-join: a seeded synthetic generator
// (stand-in for the reference's SSS datasets) and prefix-filter candidate
// generation, both on the device.
//
// Generator: set i has size ~ Zipf(size_s) on [lo, hi] (discrete inverse
// CDF); its tokens are drawn from a Zipf(1)-like law over U = 2^ulog ranks,
// P(rank = k) = ln((k+2)/(k+1)) / ln(U+1) (rank = floor((U+1)^u) - 1 for a
// uniform u), relabeled by a seeded bijection of [0, U) so token ids carry no
// frequency order; duplicates within a set are removed, rows sorted.
//
// Candidates (Jaccard threshold t = num/den): every token is ranked by
// (global frequency, id) ascending; set x's prefix is its first
// |x| - ceil(t*|x|) + 1 tokens in that order; two sets are candidates iff
// their prefixes share a token and den*min(|x|,|y|) >= num*max(|x|,|y|) (a
// pair with Jaccard >= t always passes both filters).  Output: distinct
// pairs (a < b), sorted.
#include <cub/cub.cuh>

#include <cmath>
#include <vector>

#include "common.cuh"

namespace rst {
namespace {

__device__ __forceinline__ uint64_t dmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t hmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unif(uint64_t seed, uint64_t a, uint64_t b) {
  return (double)(dmix64(seed ^ dmix64(a * 0x100000001B3ull + b)) >> 11) *
         (1.0 / 9007199254740992.0);
}

struct Bij {
  uint32_t M[3], A[3], mask;
  int sh;
};
Bij make_bij(uint64_t seed, int bits) {
  Bij r;
  r.mask = bits >= 32 ? 0xFFFFFFFFu : ((1u << bits) - 1u);
  r.sh = (bits + 1) / 2;
  for (int i = 0; i < 3; ++i) {
    r.M[i] = (uint32_t)hmix64(seed ^ (0x70CE0000ull + 2 * i)) | 1u;
    r.A[i] = (uint32_t)hmix64(seed ^ (0x70CE0001ull + 2 * i));
  }
  return r;
}
__device__ __forceinline__ uint32_t bij(const Bij& r, uint32_t x) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    x = (x * r.M[i]) & r.mask;
    x ^= x >> r.sh;
    x = (x + r.A[i]) & r.mask;
  }
  return x;
}

// Planted near-duplicates: set i > 0 is a child with probability dup_frac;
// its parent is the nearest root (non-child) among the 256 sets before it
// (none: it is a root itself).  A child has its parent's size and keeps
// each of the parent's draws with probability keep_i ~ U(keep_min, 1),
// drawing a fresh token otherwise.
__device__ __forceinline__ bool is_child(uint64_t seed, int64_t i, double dup) {
  return i > 0 && unif(seed, (uint64_t)i, 0xC41DC41Dull) < dup;
}
__device__ __forceinline__ int64_t parent_of(uint64_t seed, int64_t i, double dup) {
  if (!is_child(seed, i, dup)) return -1;
  for (int64_t k = i - 1; k >= 0 && k >= i - 256; --k)
    if (!is_child(seed, k, dup)) return k;
  return -1;
}

__device__ __forceinline__ int root_size(uint64_t seed, int64_t i,
                                         const double* __restrict__ cdf, int ncdf,
                                         int lo) {
  const double u = unif(seed, (uint64_t)i, 0xFFFFFFull);
  int a = 0, b = ncdf - 1;  // first index with cdf >= u
  while (a < b) {
    int mid = (a + b) >> 1;
    if (cdf[mid] >= u) b = mid; else a = mid + 1;
  }
  return lo + a;
}

__global__ void set_sizes_kernel(int32_t n, uint64_t seed,
                                 const double* __restrict__ cdf, int ncdf,
                                 int lo, double dup, int64_t* __restrict__ sizes) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = parent_of(seed, i, dup);
    sizes[i] = root_size(seed, p >= 0 ? p : i, cdf, ncdf, lo);
  }
}

__device__ __forceinline__ uint32_t draw_token(uint64_t seed, int64_t set, int64_t j,
                                               double lnU1, uint64_t U, const Bij& bj) {
  const double u = unif(seed, (uint64_t)set, (uint64_t)j + 1);
  uint64_t rank = (uint64_t)floor(exp(u * lnU1)) - 1;
  if (rank >= U) rank = U - 1;
  return bij(bj, (uint32_t)rank);
}

// One warp per set: its draws as (set << ulog) | token keys.
__global__ void draw_tokens_kernel(int32_t n, uint64_t seed, int ulog, Bij bj,
                                   double dup, double keep_min,
                                   const int64_t* __restrict__ draw_off,
                                   uint64_t* __restrict__ keys) {
  const int lane = threadIdx.x & 31;
  const double lnU1 = log((double)((1ull << ulog) + 1));
  const uint64_t U = 1ull << ulog;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t b0 = draw_off[i], b1 = draw_off[i + 1];
    const int64_t p = parent_of(seed, i, dup);
    const double keep = keep_min + (1.0 - keep_min) * unif(seed, (uint64_t)i, 0xEEEEull);
    for (int64_t j = b0 + lane; j < b1; j += 32) {
      uint32_t tok;
      if (p >= 0 && unif(seed ^ 0x6B6565700000ull, (uint64_t)i, (uint64_t)(j - b0)) < keep)
        tok = draw_token(seed, p, j - b0, lnU1, U, bj);
      else
        tok = draw_token(seed, i, j - b0, lnU1, U, bj);
      keys[j] = ((uint64_t)i << ulog) | tok;
    }
  }
}

__global__ void split_keys_kernel(const uint64_t* __restrict__ keys, int64_t m,
                                  int ulog, int32_t* __restrict__ tokens,
                                  int32_t* __restrict__ counts) {
  const uint64_t mask = (1ull << ulog) - 1;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m;
       j += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[j];
    tokens[j] = (int32_t)(k & mask);
    atomicAdd(&counts[k >> ulog], 1);
  }
}

// ---- prefix filtering -----------------------------------------------------

constexpr int kFreqBits = 19;
constexpr int kSizeBits = 15;

__global__ void token_freq_kernel(const int32_t* __restrict__ tokens, int64_t m,
                                  int32_t* __restrict__ freq) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m;
       j += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&freq[tokens[j]], 1);
}

// (set | min(freq, cap) | token): sorting it orders each set's tokens by
// (frequency, id) -- one global order, the same for every set.
__global__ void canon_keys_kernel(const int32_t* __restrict__ off, int32_t n,
                                  const int32_t* __restrict__ tokens,
                                  const int32_t* __restrict__ freq, int ulog,
                                  uint64_t* __restrict__ keys) {
  const int cap = (1 << kFreqBits) - 1;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int lane = threadIdx.x & 31;
    for (int j = off[i] + lane; j < off[i + 1]; j += 32) {
      const int t = tokens[j];
      const uint64_t f = (uint64_t)min(freq[t], cap);
      keys[j] = ((uint64_t)i << (kFreqBits + ulog)) | (f << ulog) | (uint64_t)t;
    }
  }
}

__global__ void prefix_len_kernel(const int32_t* __restrict__ off, int32_t n,
                                  int num, int den, int64_t* __restrict__ plen) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sz = off[i + 1] - off[i];
    // |x| - ceil(t|x|) + 1, t = num/den; empty sets have no prefix
    const int64_t need = (num * sz + den - 1) / den;
    plen[i] = sz > 0 ? sz - need + 1 : 0;
  }
}

// Prefix entries (token | size | set) of every set.
__global__ void prefix_entries_kernel(const int32_t* __restrict__ off, int32_t n,
                                      const uint64_t* __restrict__ canon,
                                      const int64_t* __restrict__ pre_off, int ulog,
                                      uint64_t* __restrict__ entries) {
  const uint64_t tmask = (1ull << ulog) - 1;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int lane = threadIdx.x & 31;
    const int s0 = off[i], sz = off[i + 1] - s0;
    const int64_t w0 = pre_off[i], p = pre_off[i + 1] - w0;
    for (int j = lane; j < p; j += 32) {
      const uint64_t tok = canon[s0 + j] & tmask;
      entries[w0 + j] = (tok << (kSizeBits + 21)) | ((uint64_t)sz << 21) | (uint64_t)i;
    }
  }
}

// For sorted entry e: partners are the following entries of the same token
// whose size is <= floor(den*size_e/num) (sizes ascend within a token).
__global__ void pair_count_kernel(const uint64_t* __restrict__ ent, int64_t ne,
                                  int num, int den, int64_t* __restrict__ cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ent[e];
    const uint64_t tok = k >> (kSizeBits + 21);
    const int64_t sz = (int64_t)((k >> 21) & ((1u << kSizeBits) - 1));
    const int64_t maxsz = (den * sz) / num;
    const int64_t capsz = maxsz < ((1 << kSizeBits) - 1) ? maxsz : ((1 << kSizeBits) - 1);
    const uint64_t lim = (tok << (kSizeBits + 21)) | ((uint64_t)capsz << 21) |
                         ((1ull << 21) - 1);
    int64_t a = e + 1, b = ne;
    while (a < b) {
      int64_t mid = (a + b) >> 1;
      if (ent[mid] <= lim) a = mid + 1; else b = mid;
    }
    cnt[e] = a - e - 1;
  }
}

__global__ void pair_emit_kernel(const uint64_t* __restrict__ ent, int64_t ne,
                                 const int64_t* __restrict__ cnt_off,
                                 uint64_t* __restrict__ pairs) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t se = (uint32_t)(ent[e] & ((1u << 21) - 1));
    int64_t w = cnt_off[e];
    const int64_t c = cnt_off[e + 1] - w;
    for (int64_t j = 1; j <= c; ++j) {
      const uint32_t sj = (uint32_t)(ent[e + j] & ((1u << 21) - 1));
      const uint32_t lo = se < sj ? se : sj, hi = se < sj ? sj : se;
      pairs[w++] = ((uint64_t)lo << 32) | hi;
    }
  }
}

__global__ void pair_split_kernel(const uint64_t* __restrict__ pairs, int64_t np,
                                  int32_t* __restrict__ pa, int32_t* __restrict__ pb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    pa[i] = (int32_t)(pairs[i] >> 32);
    pb[i] = (int32_t)(pairs[i] & 0xFFFFFFFFu);
  }
}

// Inverted index: draw j of term t is a uniform doc id; term t's draws sit
// at doff[t] .. doff[t+1] (flat over all draws, owner by binary search).
__global__ void draw_postings_kernel(const int64_t* __restrict__ doff, int32_t nterms,
                                     int64_t ndraw, int32_t ndocs, int dbits,
                                     uint64_t seed, uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndraw;
       i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nterms - 1;  // largest t with doff[t] <= i
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (doff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    uint64_t d = (uint64_t)(unif(seed, (uint64_t)lo, (uint64_t)(i - doff[lo])) * ndocs);
    if (d >= (uint64_t)ndocs) d = ndocs - 1;
    keys[i] = ((uint64_t)lo << dbits) | d;
  }
}

int g_grid(int64_t items) {
  int64_t g = (items + 255) / 256, cap = (int64_t)sm_count() * 16;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// Stream-ordered temporaries, freed when the scope ends.
struct Temps {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Temps(cudaStream_t s) : st(s) {}
  ~Temps() {
    for (void* p : ptrs)
      if (p) cudaFreeAsync(p, st);
  }
  template <class T>
  cudaError_t get(T** p, size_t bytes) {
    cudaError_t e = scratch_malloc(reinterpret_cast<void**>(p), bytes ? bytes : 16, st);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

}  // namespace
}  // namespace rst

using namespace rst;

extern "C" reset_status reset_gen_token_sets(int32_t n, int32_t universe_log2,
                                             double size_s, int32_t size_lo,
                                             int32_t size_hi, double dup_frac,
                                             double keep_min, uint64_t seed,
                                             int32_t** d_off_out,
                                             int32_t** d_tokens_out,
                                             int64_t* m_out,
                                             reset_stream_t stream) {
  if (!d_off_out || !d_tokens_out || !m_out) return arg_fail("NULL output");
  if (n < 1 || n >= (1 << 21)) return arg_fail("n must be in 1..2^21-1");
  if (universe_log2 < 4 || universe_log2 > 24) return arg_fail("universe_log2 in 4..24");
  if (size_lo < 1 || size_hi < size_lo || size_hi > 16384) return arg_fail("size range");
  if (!(dup_frac >= 0.0 && dup_frac < 1.0)) return arg_fail("dup_frac must be in [0, 1)");
  if (!(keep_min >= 0.0 && keep_min <= 1.0)) return arg_fail("keep_min must be in [0, 1]");
  cudaStream_t st = as_stream(stream);
  const int ncdf = size_hi - size_lo + 1;
  std::vector<double> cdf(ncdf);
  double acc = 0;
  for (int k = 0; k < ncdf; ++k) {
    acc += std::pow((double)(size_lo + k), -size_s);
    cdf[k] = acc;
  }
  for (auto& c : cdf) c /= acc;
  cdf.back() = 1.0;
  Temps tmp(st);
  double* d_cdf;
  int64_t *d_sizes, *d_doff;
  RST_CUDA(tmp.get(&d_cdf, sizeof(double) * ncdf));
  RST_CUDA(tmp.get(&d_sizes, sizeof(int64_t) * (n + 1)));
  RST_CUDA(tmp.get(&d_doff, sizeof(int64_t) * (n + 1)));
  RST_CUDA(cudaMemcpyAsync(d_cdf, cdf.data(), sizeof(double) * ncdf, cudaMemcpyHostToDevice, st));
  note_launch();
  set_sizes_kernel<<<g_grid(n), 256, 0, st>>>(n, seed, d_cdf, ncdf, size_lo, dup_frac,
                                               d_sizes);
  RST_CUDA(cudaGetLastError());
  RST_CUDA(cudaMemsetAsync(d_sizes + n, 0, sizeof(int64_t), st));
  size_t tb = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_sizes, d_doff, n + 1, st));
  void* d_tb;
  RST_CUDA(tmp.get(&d_tb, tb));
  RST_CUDA(cub::DeviceScan::ExclusiveSum(d_tb, tb, d_sizes, d_doff, n + 1, st));
  int64_t nd = 0;
  RST_CUDA(cudaMemcpyAsync(&nd, d_doff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  uint64_t *k0, *k1;
  RST_CUDA(tmp.get(&k0, sizeof(uint64_t) * nd));
  RST_CUDA(tmp.get(&k1, sizeof(uint64_t) * nd));
  note_launch();
  draw_tokens_kernel<<<g_grid((int64_t)n * 32), 256, 0, st>>>(
      n, seed, universe_log2, make_bij(seed, universe_log2), dup_frac, keep_min, d_doff, k0);
  RST_CUDA(cudaGetLastError());
  const int endbit = universe_log2 + 21;
  cub::DoubleBuffer<uint64_t> db(k0, k1);
  size_t ts = 0, tu = 0;
  int64_t* d_nu;
  RST_CUDA(tmp.get(&d_nu, sizeof(int64_t)));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, ts, db, nd, 0, endbit, st));
  RST_CUDA(cub::DeviceSelect::Unique(nullptr, tu, k0, k1, d_nu, nd, st));
  void* d_ts;
  RST_CUDA(tmp.get(&d_ts, ts > tu ? ts : tu));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(d_ts, ts, db, nd, 0, endbit, st));
  RST_CUDA(cub::DeviceSelect::Unique(d_ts, tu, db.Current(), db.Alternate(), d_nu, nd, st));
  int64_t m = 0;
  RST_CUDA(cudaMemcpyAsync(&m, d_nu, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  if (m > INT32_MAX) return arg_fail("more than 2^31 tokens in total");
  int32_t *off = nullptr, *tok = nullptr, *cnt;
  RST_CUDA(tmp.get(&cnt, sizeof(int32_t) * (n + 1)));
  RST_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st));
  RST_CUDA(cudaMalloc(&off, sizeof(int32_t) * (n + 1)));
  cudaError_t e = cudaMalloc(&tok, sizeof(int32_t) * (m > 0 ? m : 1));
  if (e != cudaSuccess) {
    cudaFree(off);
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  note_launch();
  split_keys_kernel<<<g_grid(m), 256, 0, st>>>(db.Alternate(), m, universe_log2, tok, cnt);
  size_t tb2 = 0;
  e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt, off, n + 1, st);
  void* d_tb2 = nullptr;
  if (e == cudaSuccess) e = tmp.get(&d_tb2, tb2);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(d_tb2, tb2, cnt, off, n + 1, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(off);
    cudaFree(tok);
    return cuda_fail(e, "token sets", __FILE__, __LINE__);
  }
  *d_off_out = off;
  *d_tokens_out = tok;
  *m_out = m;
  return RESET_OK;
}

extern "C" reset_status reset_prefix_candidates(const int32_t* d_off,
                                                const int32_t* d_tokens,
                                                int32_t n, int64_t m,
                                                int32_t universe_log2,
                                                int32_t num, int32_t den,
                                                int32_t** d_pa_out,
                                                int32_t** d_pb_out,
                                                int64_t* np_out,
                                                reset_stream_t stream) {
  if (!d_pa_out || !d_pb_out || !np_out) return arg_fail("NULL output");
  if (n < 1 || n >= (1 << 21)) return arg_fail("n must be in 1..2^21-1");
  if (universe_log2 < 4 || universe_log2 > 24) return arg_fail("universe_log2 in 4..24");
  if (num < 1 || den < num) return arg_fail("threshold num/den must be in (0, 1]");
  cudaStream_t st = as_stream(stream);
  Temps tmp(st);
  const int64_t U = 1ll << universe_log2;
  int32_t* freq;
  uint64_t *ck0, *ck1;
  int64_t *plen, *poff;
  RST_CUDA(tmp.get(&freq, sizeof(int32_t) * U));
  RST_CUDA(cudaMemsetAsync(freq, 0, sizeof(int32_t) * U, st));
  RST_CUDA(tmp.get(&ck0, sizeof(uint64_t) * (m > 0 ? m : 1)));
  RST_CUDA(tmp.get(&ck1, sizeof(uint64_t) * (m > 0 ? m : 1)));
  RST_CUDA(tmp.get(&plen, sizeof(int64_t) * (n + 1)));
  RST_CUDA(tmp.get(&poff, sizeof(int64_t) * (n + 1)));
  note_launch();
  token_freq_kernel<<<g_grid(m), 256, 0, st>>>(d_tokens, m, freq);
  note_launch();
  canon_keys_kernel<<<g_grid((int64_t)n * 32), 256, 0, st>>>(d_off, n, d_tokens, freq,
                                                             universe_log2, ck0);
  RST_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> cb(ck0, ck1);
  size_t ts = 0;
  RST_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, ts, cb, m, 0, 64, st));
  void* d_ts;
  RST_CUDA(tmp.get(&d_ts, ts));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(d_ts, ts, cb, m, 0, 64, st));
  note_launch();
  prefix_len_kernel<<<g_grid(n), 256, 0, st>>>(d_off, n, num, den, plen);
  RST_CUDA(cudaMemsetAsync(plen + n, 0, sizeof(int64_t), st));
  size_t tsc = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tsc, plen, poff, n + 1, st));
  void* d_tsc;
  RST_CUDA(tmp.get(&d_tsc, tsc));
  RST_CUDA(cub::DeviceScan::ExclusiveSum(d_tsc, tsc, plen, poff, n + 1, st));
  int64_t ne = 0;
  RST_CUDA(cudaMemcpyAsync(&ne, poff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  uint64_t *e0, *e1;
  int64_t *cnt, *coff;
  RST_CUDA(tmp.get(&e0, sizeof(uint64_t) * (ne > 0 ? ne : 1)));
  RST_CUDA(tmp.get(&e1, sizeof(uint64_t) * (ne > 0 ? ne : 1)));
  RST_CUDA(tmp.get(&cnt, sizeof(int64_t) * (ne + 1)));
  RST_CUDA(tmp.get(&coff, sizeof(int64_t) * (ne + 1)));
  note_launch();
  prefix_entries_kernel<<<g_grid((int64_t)n * 32), 256, 0, st>>>(
      d_off, n, cb.Current(), poff, universe_log2, e0);
  RST_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> eb(e0, e1);
  size_t te = 0;
  const int ebits = universe_log2 + kSizeBits + 21;
  RST_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, te, eb, ne, 0, ebits, st));
  void* d_te;
  RST_CUDA(tmp.get(&d_te, te));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(d_te, te, eb, ne, 0, ebits, st));
  note_launch();
  pair_count_kernel<<<g_grid(ne), 256, 0, st>>>(eb.Current(), ne, num, den, cnt);
  RST_CUDA(cudaMemsetAsync(cnt + ne, 0, sizeof(int64_t), st));
  size_t tc2 = 0;
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tc2, cnt, coff, ne + 1, st));
  void* d_tc2;
  RST_CUDA(tmp.get(&d_tc2, tc2));
  RST_CUDA(cub::DeviceScan::ExclusiveSum(d_tc2, tc2, cnt, coff, ne + 1, st));
  int64_t nraw = 0;
  RST_CUDA(cudaMemcpyAsync(&nraw, coff + ne, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  uint64_t *p0, *p1;
  int64_t* d_np;
  RST_CUDA(tmp.get(&p0, sizeof(uint64_t) * (nraw > 0 ? nraw : 1)));
  RST_CUDA(tmp.get(&p1, sizeof(uint64_t) * (nraw > 0 ? nraw : 1)));
  RST_CUDA(tmp.get(&d_np, sizeof(int64_t)));
  note_launch();
  pair_emit_kernel<<<g_grid(ne), 256, 0, st>>>(eb.Current(), ne, coff, p0);
  RST_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> pb(p0, p1);
  size_t tp = 0, tu = 0;
  RST_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tp, pb, nraw, 0, 64, st));
  RST_CUDA(cub::DeviceSelect::Unique(nullptr, tu, p0, p1, d_np, nraw, st));
  void* d_tp;
  RST_CUDA(tmp.get(&d_tp, tp > tu ? tp : tu));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(d_tp, tp, pb, nraw, 0, 64, st));
  RST_CUDA(cub::DeviceSelect::Unique(d_tp, tu, pb.Current(), pb.Alternate(), d_np, nraw, st));
  int64_t np = 0;
  RST_CUDA(cudaMemcpyAsync(&np, d_np, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  int32_t *pa = nullptr, *pbb = nullptr;
  RST_CUDA(cudaMalloc(&pa, sizeof(int32_t) * (np > 0 ? np : 1)));
  cudaError_t e = cudaMalloc(&pbb, sizeof(int32_t) * (np > 0 ? np : 1));
  if (e != cudaSuccess) {
    cudaFree(pa);
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  note_launch();
  pair_split_kernel<<<g_grid(np), 256, 0, st>>>(pb.Alternate(), np, pa, pbb);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(pa);
    cudaFree(pbb);
    return cuda_fail(e, "candidate split", __FILE__, __LINE__);
  }
  *d_pa_out = pa;
  *d_pb_out = pbb;
  *np_out = np;
  return RESET_OK;
}

extern "C" reset_status reset_gen_inverted_index(int32_t nterms, int32_t ndocs,
                                                 double zipf_s, int64_t df_max,
                                                 uint64_t seed, int32_t** d_toff_out,
                                                 int32_t** d_docs_out, int64_t* m_out,
                                                 reset_stream_t stream) {
  if (!d_toff_out || !d_docs_out || !m_out) return arg_fail("NULL output");
  if (nterms < 1 || nterms > (1 << 26)) return arg_fail("nterms must be in 1..2^26");
  if (ndocs < 1) return arg_fail("ndocs must be >= 1");
  if (df_max < 1) return arg_fail("df_max must be >= 1");
  if (!(zipf_s >= 0.0)) return arg_fail("zipf_s must be >= 0");
  int dbits = 1;
  while ((1ll << dbits) < ndocs) ++dbits;
  int tbits = 1;
  while ((1ll << tbits) < nterms) ++tbits;
  if (dbits + tbits > 64) return arg_fail("too many terms x docs");
  cudaStream_t st = as_stream(stream);
  std::vector<int64_t> doff((size_t)nterms + 1);
  int64_t tot = 0;
  for (int32_t t = 0; t < nterms; ++t) {
    doff[t] = tot;
    int64_t df = (int64_t)std::llround((double)df_max * std::pow((double)(t + 1), -zipf_s));
    if (df < 1) df = 1;
    if (df > ndocs) df = ndocs;
    tot += df;
  }
  doff[nterms] = tot;
  if (tot > INT32_MAX) return arg_fail("more than 2^31 postings");
  Temps tmp(st);
  int64_t* d_doff;
  uint64_t *k0, *k1;
  int64_t* d_nu;
  RST_CUDA(tmp.get(&d_doff, sizeof(int64_t) * (nterms + 1)));
  RST_CUDA(tmp.get(&k0, sizeof(uint64_t) * tot));
  RST_CUDA(tmp.get(&k1, sizeof(uint64_t) * tot));
  RST_CUDA(tmp.get(&d_nu, sizeof(int64_t)));
  RST_CUDA(cudaMemcpyAsync(d_doff, doff.data(), sizeof(int64_t) * (nterms + 1),
                           cudaMemcpyHostToDevice, st));
  note_launch();
  draw_postings_kernel<<<g_grid(tot), 256, 0, st>>>(d_doff, nterms, tot, ndocs, dbits,
                                                   seed, k0);
  RST_CUDA(cudaGetLastError());
  cub::DoubleBuffer<uint64_t> db(k0, k1);
  size_t ts = 0, tu = 0;
  RST_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, ts, db, tot, 0, dbits + tbits, st));
  RST_CUDA(cub::DeviceSelect::Unique(nullptr, tu, k0, k1, d_nu, tot, st));
  void* d_ts;
  RST_CUDA(tmp.get(&d_ts, ts > tu ? ts : tu));
  RST_CUDA(cub::DeviceRadixSort::SortKeys(d_ts, ts, db, tot, 0, dbits + tbits, st));
  RST_CUDA(cub::DeviceSelect::Unique(d_ts, tu, db.Current(), db.Alternate(), d_nu, tot, st));
  int64_t m = 0;
  RST_CUDA(cudaMemcpyAsync(&m, d_nu, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  int32_t *toff = nullptr, *docs = nullptr, *cnt;
  RST_CUDA(tmp.get(&cnt, sizeof(int32_t) * (nterms + 1)));
  RST_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (nterms + 1), st));
  RST_CUDA(cudaMalloc(&toff, sizeof(int32_t) * (nterms + 1)));
  cudaError_t e = cudaMalloc(&docs, sizeof(int32_t) * (m > 0 ? m : 1));
  if (e != cudaSuccess) {
    cudaFree(toff);
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  note_launch();
  split_keys_kernel<<<g_grid(m), 256, 0, st>>>(db.Alternate(), m, dbits, docs, cnt);
  size_t tb2 = 0;
  e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt, toff, nterms + 1, st);
  void* d_tb2 = nullptr;
  if (e == cudaSuccess) e = tmp.get(&d_tb2, tb2);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(d_tb2, tb2, cnt, toff, nterms + 1, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(toff);
    cudaFree(docs);
    return cuda_fail(e, "inverted index", __FILE__, __LINE__);
  }
  *d_toff_out = toff;
  *d_docs_out = docs;
  *m_out = m;
  return RESET_OK;
}
