// Vertex-staged triangle counting (method 2 of reset_tc_count_ex; used by
// reset_tc_count_noalloc).
//
// Same count as dynamic_triangle_count (triangle-count/TC.cu:128-190): for
// every oriented edge (u, v) the smaller row is probed against the larger
// one (ties: u's keys against v's set), so even rows with repeated entries
// give the reference's number.  What changes is where the bytes come from.
// All out-edges of u share u's row, so u's row is read once into shared
// memory, as a key array K and an open-addressing hash set H:
//   * d(v) <  d(u): v's keys stream from HBM (consecutive lanes read
//     consecutive keys) and are looked up in H -- no table read in HBM;
//   * d(v) >= d(u): u's keys come from K in shared memory and probe v's
//     bucketed table in HBM (reference layout and hash) -- no key read.
// Either way one HBM stream per probe instead of two.
//
// Work classes, all in one persistent launch with dynamic work counters:
//   phase 1  rows with d(u) > kWarpMax: (u, 256-edge segment) units, one CTA
//            each, K/H shared by the CTA (rows above kCtaMax probe the HBM
//            tables on both sides);
//   phase 2  groups of 32 consecutive vertices, one warp each: rows with
//            kTiny <= d(u) <= kWarpMax are staged per warp; tiny rows
//            (d(u) < kTiny) have their edges flattened across the group and
//            then their probes flattened across the warp (thread-granularity
//            work for tiny intersections).
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "probe_common.cuh"

namespace rst {
namespace {

constexpr int kT = 256;
constexpr int kW = kT / 32;
constexpr int kTiny = 32;
constexpr int kWarpMax = 256;
constexpr int kCtaMax = 4096;
constexpr int kSeg = 256;
constexpr int kWarpSmem = 3 * kWarpMax;       // K + H per warp (ints)
constexpr int kCtaSmem = 3 * kCtaMax;         // K + H per CTA (ints)
constexpr int kRounds = 4;                    // probe rounds issued together
static_assert(kW * kWarpSmem <= kCtaSmem, "warp regions must fit the CTA buffer");

__device__ __forceinline__ int hslot(int x, int lgP) {
  return (int)(((unsigned)x * 0x9E3779B1u) >> (32 - lgP));
}

__device__ __forceinline__ void hset_insert(int* H, int lgP, int x) {
  const int P = 1 << lgP;
  int h = hslot(x, lgP);
  for (int t = 0; t < P; ++t) {
    const int old = atomicCAS(&H[h], -1, x);
    if (old == -1 || old == x) return;
    h = (h + 1) & (P - 1);
  }
}

__device__ __forceinline__ bool hset_has(const int* H, int lgP, int x) {
  const int P = 1 << lgP;
  int h = hslot(x, lgP);
  for (int t = 0; t < P; ++t) {
    const int s = H[h];
    if (s == x) return true;
    if (s == -1) return false;
    h = (h + 1) & (P - 1);
  }
  return false;
}

// log2 of the hash capacity for a row of d keys: next power of two >= 2d,
// at least 64.
__device__ __forceinline__ int hset_lg(int d) {
  const int want = 2 * d;
  int lg = 32 - __clz(want - 1);
  return lg < 6 ? 6 : lg;
}

// One batch of up to 32 out-edges of a staged row u (lane i: edge j0+i).
// Keys of u are in K, its set in H (capacity 2^lgP).
template <bool HIER>
__device__ __forceinline__ int staged_batch(
    int j0, int je, int du, const int* K, const int* H, int lgP,
    const int32_t* __restrict__ cols, const int4* __restrict__ desc, int n,
    const int32_t* __restrict__ table, int64_t bn, int b, int lg_max,
    int32_t* status) {
  int hits = 0;
  const int lane = threadIdx.x & 31;
  const int j = j0 + lane;
  const bool valid = j < je;
  int v = valid ? K[j] : 0;
  bool ok = valid;
  if ((unsigned)v >= (unsigned)n) {
    if (valid) atomicOr(status, kErrBadId);
    ok = false;
    v = 0;
  }
  const int4 dv = __ldg(desc + v);
  const bool stream = dv.y < du;  // v is the smaller row: its keys probe u
  const int s = ok ? (stream ? dv.y : du) : 0;
  const int src = dv.x;
  const int64_t toff = desc_toff(dv);
  const int lg = desc_lg(dv);
  int S;
  const int P = warp_excl_scan(s, &S);
  // kRounds rounds at once: key loads (HBM for streamed rows, shared memory
  // for u's own keys), then the first-slot loads of the table probes, then
  // the lookups and continuations.
  for (int base = 0; base < S; base += 32 * kRounds) {
    int x[kRounds], h[kRounds], klg[kRounds], s0[kRounds], s1[kRounds];
    const int32_t* tb[kRounds];
    bool act[kRounds], kst[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      const int f = base + r * 32 + lane;
      const int k = owner_lane(P, f);
      const int kp = __shfl_sync(kFull, P, k);
      const int ks = __shfl_sync(kFull, src, k);
      kst[r] = __shfl_sync(kFull, (int)stream, k);
      klg[r] = __shfl_sync(kFull, lg, k);
      tb[r] = table + __shfl_sync(kFull, toff, k);
      act[r] = f < S;
      const int jj = f - kp;
      x[r] = act[r] ? (kst[r] ? __ldg(cols + ks + jj) : K[jj]) : 0;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      h[r] = home_bucket<HIER>(x[r], klg[r], lg_max);
      const bool g = act[r] && !kst[r];
      s0[r] = g ? __ldg(tb[r] + h[r]) : -1;
      s1[r] = g ? __ldg(tb[r] + h[r] + (b > 1 ? bn : 0)) : -1;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      if (!act[r]) continue;
      bool hit;
      if (kst[r]) {
        hit = hset_has(H, lgP, x[r]);
      } else {
        hit = probe_resolve2<HIER>(x[r], s0[r], s1[r], tb[r], klg[r], h[r], bn, b,
                                   status);
      }
      hits += hit;
    }
  }
  return hits;
}

// One batch of out-edges of an unstaged row u (d(u) > kCtaMax): both sides
// in HBM, as in the reference kernel.
template <bool HIER>
__device__ __forceinline__ int global_batch(
    int j0, int je, int4 du4, const int32_t* __restrict__ cols, int64_t n_cols,
    const int4* __restrict__ desc, int n, const int32_t* __restrict__ table,
    int64_t bn, int b, int lg_max, int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int j = j0 + lane;
  const bool valid = j < je;
  int v = valid ? __ldg(cols + du4.x + j) : 0;
  bool ok = valid;
  if ((unsigned)v >= (unsigned)n) {
    if (valid) atomicOr(status, kErrBadId);
    ok = false;
    v = 0;
  }
  const int4 dv = __ldg(desc + v);
  const bool sw = du4.y > dv.y;
  const int4 A = sw ? dv : du4;
  const int4 B = sw ? du4 : dv;
  return flat_probe<HIER>(cols, n_cols, table, ok ? A.y : 0, A.x, desc_toff(B),
                          desc_lg(B), lg_max, bn, b, status, [](int) {});
}

template <bool HIER>
__global__ void __launch_bounds__(kT, 2)
    tc_staged_kernel(const int4* __restrict__ desc,
                     const int32_t* __restrict__ cols, int64_t n_cols, int32_t n,
                     const int2* __restrict__ units,
                     const int32_t* __restrict__ n_units_p, int units_cap,
                     int32_t* __restrict__ cursors,
                     const int32_t* __restrict__ table, int64_t bn, int b,
                     int lg_max, unsigned long long* __restrict__ count,
                     int32_t* __restrict__ status) {
  extern __shared__ int sm[];
  __shared__ int s_unit;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned long long hits = 0;

  // ---- phase 1: (row, segment) units of long rows, one CTA each
  const int n_units = min(*n_units_p, units_cap);
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(&cursors[0], 1);
    __syncthreads();
    const int ui = s_unit;
    __syncthreads();
    if (ui >= n_units) break;
    const int2 unit = units[ui];
    const int4 du4 = __ldg(desc + unit.x);
    const int du = du4.y;
    const int e0 = unit.y * kSeg;
    const int e1 = min(du, e0 + kSeg);
    if (du <= kCtaMax) {
      int* K = sm;
      int* H = sm + kCtaMax;
      const int lgP = hset_lg(du);
      for (int i = tid; i < (1 << lgP); i += kT) H[i] = -1;
      for (int i = tid; i < du; i += kT) K[i] = __ldg(cols + du4.x + i);
      __syncthreads();
      for (int i = tid; i < du; i += kT) hset_insert(H, lgP, K[i]);
      __syncthreads();
      for (int j0 = e0 + warp * 32; j0 < e1; j0 += kT)
        hits += staged_batch<HIER>(j0, e1, du, K, H, lgP, cols, desc, n, table,
                                   bn, b, lg_max, status);
    } else {
      for (int j0 = e0 + warp * 32; j0 < e1; j0 += kT)
        hits += global_batch<HIER>(j0, e1, du4, cols, n_cols, desc, n, table, bn,
                                   b, lg_max, status);
    }
    __syncthreads();
  }

  // ---- phase 2: groups of 32 vertices, one warp each
  int* K = sm + warp * kWarpSmem;
  int* H = K + kWarpMax;
  const int n_groups = (n + 31) >> 5;
  for (;;) {
    int g = 0;
    if (lane == 0) g = atomicAdd(&cursors[1], 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= n_groups) break;
    const int u = g * 32 + lane;
    const bool vu = u < n;
    const int4 du4 = vu ? __ldg(desc + u) : make_int4(0, 0, 0, 0);
    const int du = du4.y;

    // tiny rows: flatten their edges, then the probes of each 32-edge batch
    {
      const int ecnt = (du > 0 && du < kTiny) ? du : 0;
      int E;
      const int PE = warp_excl_scan(ecnt, &E);
      const int64_t ut = desc_toff(du4);
      const int ulg = desc_lg(du4);
      for (int eb = 0; eb < E; eb += 32) {
        const int fe = eb + lane;
        const int ko = owner_lane(PE, fe);
        const int kpe = __shfl_sync(kFull, PE, ko);
        const int ksu = __shfl_sync(kFull, du4.x, ko);
        const int kdu = __shfl_sync(kFull, du, ko);
        const int64_t kut = __shfl_sync(kFull, ut, ko);
        const int kulg = __shfl_sync(kFull, ulg, ko);
        const bool ve = fe < E;
        int v = ve ? __ldg(cols + ksu + (fe - kpe)) : 0;
        bool ok = ve;
        if ((unsigned)v >= (unsigned)n) {
          if (ve) atomicOr(status, kErrBadId);
          ok = false;
          v = 0;
        }
        const int4 dv = __ldg(desc + v);
        const bool sw = kdu > dv.y;  // TC.cu:148-157
        const int s = ok ? (sw ? dv.y : kdu) : 0;
        const int a_start = sw ? dv.x : ksu;
        const int64_t t_off = sw ? kut : desc_toff(dv);
        const int t_lg = sw ? kulg : desc_lg(dv);
        hits += flat_probe<HIER>(cols, n_cols, table, s, a_start, t_off, t_lg,
                                 lg_max, bn, b, status, [](int) {});
      }
    }
    // medium rows: stage one row at a time in this warp's region
    unsigned msk = __ballot_sync(kFull, vu && du >= kTiny && du <= kWarpMax);
    while (msk) {
      const int src = __ffs(msk) - 1;
      msk &= msk - 1;
      const int rs = __shfl_sync(kFull, du4.x, src);
      const int d = __shfl_sync(kFull, du, src);
      const int lgP = hset_lg(d);
      for (int i = lane; i < (1 << lgP); i += 32) H[i] = -1;
      for (int i = lane; i < d; i += 32) K[i] = __ldg(cols + rs + i);
      __syncwarp();
      for (int i = lane; i < d; i += 32) hset_insert(H, lgP, K[i]);
      __syncwarp();
      for (int j0 = 0; j0 < d; j0 += 32)
        hits += staged_batch<HIER>(j0, d, d, K, H, lgP, cols, desc, n, table,
                                   bn, b, lg_max, status);
      __syncwarp();
    }
  }
  hits = warp_sum_u64(hits);
  if (lane == 0 && hits) atomicAdd(count, hits);
}

// (row, segment) units for rows longer than kWarpMax.
__global__ void tc_plan_kernel(const int4* __restrict__ desc, int32_t n,
                               int2* __restrict__ units,
                               int32_t* __restrict__ n_units, int cap,
                               int32_t* __restrict__ status) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int d = desc[u].y;
    if (d > kWarpMax) {
      const int ns = (d + kSeg - 1) / kSeg;
      const int pos = atomicAdd(n_units, ns);
      if (pos + ns > cap) atomicOr(status, kErrBadId);  // offsets past m
      for (int s = 0; s < ns && pos + s < cap; ++s)
        units[pos + s] = make_int2((int)u, s);
    }
  }
}

}  // namespace

// Launches the staged TC path on `st`; *count must already be zeroed.
reset_status tc_staged(const reset_table* t, const int4* desc,
                       const int32_t* d_cols, int64_t m,
                       unsigned long long* count, cudaStream_t st) {
  const int64_t mm = m > t->m ? m : t->m;
  const int cap = (int)(mm / 128 + 64);
  int2* units = nullptr;
  int32_t* ctr = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&units), sizeof(int2) * cap, st));
  cudaError_t e = scratch_malloc(reinterpret_cast<void**>(&ctr), sizeof(int32_t) * 4, st);
  if (e != cudaSuccess) {
    cudaFreeAsync(units, st);
    return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
  }
  e = cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 4, st);
  if (e == cudaSuccess) {
    const int g1 = (int)std::min<int64_t>((t->n + 255) / 256, (int64_t)sm_count() * 8);
    note_launch();
    tc_plan_kernel<<<g1 > 0 ? g1 : 1, 256, 0, st>>>(desc, t->n, units, ctr + 2, cap,
                                                    t->d_status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const size_t smem = sizeof(int) * kCtaSmem;
    const void* k = t->hier ? (const void*)tc_staged_kernel<true>
                            : (const void*)tc_staged_kernel<false>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kT, smem);
    if (e == cudaSuccess) {
      const int grid = sm_count() * (per_sm > 0 ? per_sm : 1);
      note_launch();
      if (t->hier)
        tc_staged_kernel<true><<<grid, kT, smem, st>>>(
            desc, d_cols, m, t->n, units, ctr + 2, cap, ctr, t->d_table,
            t->bucket_num, t->bucket, t->lg_max, count, t->d_status);
      else
        tc_staged_kernel<false><<<grid, kT, smem, st>>>(
            desc, d_cols, m, t->n, units, ctr + 2, cap, ctr, t->d_table,
            t->bucket_num, t->bucket, t->lg_max, count, t->d_status);
      e = cudaGetLastError();
    }
  }
  cudaFreeAsync(units, st);
  cudaFreeAsync(ctr, st);
  if (e != cudaSuccess) return cuda_fail(e, "tc_staged launch", __FILE__, __LINE__);
  return RESET_OK;
}

}  // namespace rst

// ---------------------------------------------------------------------------
// reset_tc_count_noalloc: the vertex-staged count with its scratch (four work
// counters and the (row, segment) unit list) in a fixed device array instead
// of per-call cudaMallocAsync, for callers that must not allocate device
// memory while they run.  The array is loaded with the library on every GPU
// that uses it and stays until the process exits.
// ---------------------------------------------------------------------------
namespace rst {
namespace {

// Unit capacity: at most m/128 + 64 units are needed for m edges, so the
// entry point accepts up to (kNoAllocUnits - 64) * 128 edges.
constexpr int kNoAllocUnits = 1 << 20;
constexpr int64_t kNoAllocMaxEdges = (int64_t)(kNoAllocUnits - 64) * 128;
// [0] and [1] hold the four int32 counters; units start at [2].  8 MiB.
static __device__ __align__(256) int2 g_tc_noalloc_scratch[kNoAllocUnits + 2];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
int2* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device; looked up once
// per device (the host-side symbol is not a device address).  The cached
// address holds for the life of the device's primary context: a process that
// resets the device (cudaDeviceReset) must not call this entry point again.
reset_status noalloc_scratch(int2** out) {
  int dev = 0;
  RST_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return arg_fail("device ordinal too large");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    RST_CUDA(cudaGetSymbolAddress(&p, g_tc_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<int2*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return RESET_OK;
}

}  // namespace
}  // namespace rst

extern "C" reset_status reset_tc_count_noalloc(const reset_table* t,
                                               const int32_t* d_off,
                                               const int32_t* d_cols,
                                               int64_t m, uint64_t* d_count,
                                               reset_stream_t stream) {
  using namespace rst;
  if (!t || !d_count) return arg_fail("NULL table or count");
  if (m < 0 || m > INT32_MAX) return arg_fail("m out of range");
  if (m > 0 && !d_cols) return arg_fail("NULL cols");
  if (d_off && d_off != t->build_off)
    return arg_fail("reset_tc_count_noalloc needs the offsets the table was built from");
  if (m > kNoAllocMaxEdges || t->m > kNoAllocMaxEdges) {
    set_error("invalid argument: reset_tc_count_noalloc takes at most %lld edges "
              "(its fixed scratch holds %d work units)",
              (long long)kNoAllocMaxEdges, kNoAllocUnits);
    return RESET_ERR_ARG;
  }
  // the kernel walks rows through the table's build-time descriptors, so the
  // column array must be the one of the build CSR (same length)
  if (m != t->m)
    return arg_fail("reset_tc_count_noalloc needs m equal to the table's edge count");
  cudaStream_t st = as_stream(stream);
  int2* scratch = nullptr;
  RST_CHECK(noalloc_scratch(&scratch));
  int32_t* ctr = reinterpret_cast<int32_t*>(scratch);
  int2* units = scratch + 2;
  RST_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st));
  if (m == 0 || t->n == 0) return RESET_OK;
  RST_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 4, st));
  const int g1 = (int)std::min<int64_t>((t->n + 255) / 256, (int64_t)sm_count() * 8);
  note_launch();
  tc_plan_kernel<<<g1 > 0 ? g1 : 1, 256, 0, st>>>(t->d_desc, t->n, units, ctr + 2,
                                                  kNoAllocUnits, t->d_status);
  RST_CUDA(cudaGetLastError());
  const size_t smem = sizeof(int) * kCtaSmem;
  const void* k = t->hier ? (const void*)tc_staged_kernel<true>
                          : (const void*)tc_staged_kernel<false>;
  RST_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  RST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kT, smem));
  const int grid = sm_count() * (per_sm > 0 ? per_sm : 1);
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(d_count);
  note_launch();
  if (t->hier)
    tc_staged_kernel<true><<<grid, kT, smem, st>>>(
        t->d_desc, d_cols, m, t->n, units, ctr + 2, kNoAllocUnits, ctr, t->d_table,
        t->bucket_num, t->bucket, t->lg_max, cnt, t->d_status);
  else
    tc_staged_kernel<false><<<grid, kT, smem, st>>>(
        t->d_desc, d_cols, m, t->n, units, ctr + 2, kNoAllocUnits, ctr, t->d_table,
        t->bucket_num, t->bucket, t->lg_max, cnt, t->d_status);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}
