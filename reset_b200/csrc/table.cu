// Table build: the per-set bucketed hash tables of the reference, built
// deterministically on sm_100a.
//
// Reference: triangle-count/hashtable.cu:21-183 (calculate_length,
// calculate_hash_length, scan, build_hash_table_normal/_hierarchical) and
// baseline/common/hash_table.cu:69-192.  The reference inserts with one
// thread per element and atomicCAS, so slot placement depends on timing.
// Here every set is inserted in CSR order with the same rule (home bucket,
// first empty slot, next bucket when full), so the table is a pure function
// of the input and equals the CPU restatement byte for byte.
//
// Layout of the work:
//  * meta:   len[u] = calc_len(deg u), max_len, and the list of "big" sets
//            whose table does not fit a shared-memory tile.
//  * scan:   off[u] = sum_{w<u} len[w] (64-bit), off[n] = bucket_num.
//  * layout: packed 16-byte per-set descriptors for the probe kernels, the
//            row of every 32-edge chunk, and the first set of every tile.
//  * tile build: one CTA per tile of ~T consecutive buckets.  The tile's
//            b slot planes live in shared memory; small sets (deg <= 8) are
//            inserted by one thread each, larger ones by a warp that
//            inserts 32 keys per round with __match_any_sync, committing
//            the longest prefix of lanes whose placement cannot depend on a
//            later lane (so the result is the sequential one).  The planes
//            are then written to HBM with cp.async.bulk (the TMA engine's
//            1-D bulk copy) -- every table byte is written exactly once and
//            no separate memset pass runs.
//  * big build: one CTA per big set, keys inserted straight into HBM.
#include <cub/cub.cuh>

#include <cstring>
#include <mutex>

#include "common.cuh"

namespace rst {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileThreads = 512;  // threads of a tile-build CTA (3 CTAs, 48 warps per SM)
constexpr int kTileWarps = kTileThreads / 32;
constexpr bool kTileDynamic = true;  // warps take a tile's larger sets from a cursor
constexpr int kThreadSetMax = 8;      // sets with deg <= this: thread per set
constexpr int kTileSmemBudget = 72 * 1024;
constexpr int kBigFillSmemMax = 64 * 1024;  // buckets whose fill bytes fit smem
constexpr int kHugeKeys = 1 << 16;  // sets this long get the parallel build
constexpr int kMaxHuge = 512;       // ... at most this many per table

struct Geom {
  int R_max;  // buckets per shared-memory tile (stride of a slot plane)
  int T;      // buckets assigned per CTA
  int LT;     // largest table length built in a tile
  size_t smem;
};

Geom tile_geom(int b) {
  Geom g;
  int per = 4 * b + 1;
  g.R_max = (kTileSmemBudget / per) & ~7;
  g.LT = 8;
  while (g.LT * 2 <= g.R_max / 3) g.LT *= 2;
  g.T = (g.R_max - g.LT) & ~7;
  g.smem = (size_t)g.R_max * 4 * b + (size_t)g.R_max;
  g.smem = (g.smem + 15) & ~(size_t)15;
  return g;
}

// ------------------------------------------------------------- PTX bits --

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc,
                                           unsigned bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(ssrc);
  asm volatile(
      "cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(
          gdst),
      "r"(s), "r"(bytes)
      : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------------ meta pass --

__global__ void meta_kernel(const int32_t* __restrict__ off, int32_t n,
                            float alpha, int b, int LT,
                            int32_t* __restrict__ len,
                            int64_t* __restrict__ len64,
                            int32_t* __restrict__ info,  // [0]=max_len [1]=big [2]=huge
                            int32_t* __restrict__ big_list,
                            int32_t* __restrict__ huge_list,
                            int32_t* __restrict__ status) {
  int mx = 0;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    int d = off[u + 1] - off[u];
    if (d < 0) {
      atomicOr(status, kErrTableFull);
      d = 0;
    }
    int l = calc_len(d, alpha, b);
    len[u] = l;
    len64[u] = l;
    mx = max(mx, l);
    if (l > LT) {
      // sets of kHugeKeys or more keys (up to kMaxHuge of them) get the
      // parallel build; the rest of the long sets one warp each
      int slot = d >= kHugeKeys ? atomicAdd(&info[2], 1) : kMaxHuge;
      if (slot < kMaxHuge)
        huge_list[slot] = (int32_t)u;
      else
        big_list[atomicAdd(&info[1], 1)] = (int32_t)u;
    }
  }
  mx = __reduce_max_sync(kFull, mx);
  if ((threadIdx.x & 31) == 0 && mx > 0) atomicMax(&info[0], mx);
}

__global__ void finalize_kernel(const int32_t* __restrict__ len,
                                int64_t* __restrict__ off64, int32_t n,
                                int64_t* __restrict__ out_bucket_num) {
  int64_t bn = n > 0 ? off64[n - 1] + len[n - 1] : 0;
  off64[n] = bn;
  *out_bucket_num = bn;
}

// Per-set descriptors, 32-edge chunk rows and the first set of every tile.
__global__ void layout_kernel(const int32_t* __restrict__ off,
                              const int64_t* __restrict__ off64,
                              const int32_t* __restrict__ len, int32_t n,
                              int4* __restrict__ desc,
                              int32_t* __restrict__ chunk_row,
                              int32_t* __restrict__ tile_first, int T,
                              int32_t n_tiles) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int u = (int)i;
    int s = off[u], e = off[u + 1];
    if (chunk_row)
      for (int64_t c = ((int64_t)s + 31) >> 5; c * 32 < e; ++c)
        chunk_row[c] = u;
    if (!off64) continue;
    int64_t toff = off64[u];
    int lg = 31 - __clz(len[u]);
    if (desc)
      desc[u] = make_int4(s, e - s, (int)(uint32_t)toff,
                          (int)(((toff >> 32) & 0xFFFFFF) | ((int64_t)lg << 24)));
    if (tile_first) {
      // tiles whose first set is u: (tile(off64[u-1]), tile(off64[u])]
      int64_t cu = toff / T;
      int64_t cp = u > 0 ? off64[u - 1] / T : -1;
      for (int64_t c = cp + 1; c <= cu && c < n_tiles; ++c) tile_first[c] = u;
      if (u == n - 1)
        for (int64_t c = cu + 1; c <= n_tiles; ++c) tile_first[c] = n;
    }
  }
}

// ------------------------------------------------------- slot storages --

// Shared-memory tile: plane k of the tile at S + k*stride; per-bucket fill
// counts in bytes.
struct SmemSlots {
  int32_t* S;
  int stride;
  unsigned char* fill;
  int base;  // first bucket of the set inside the tile
  __device__ __forceinline__ int get_fill(int bb) const {
    return fill[base + bb];
  }
  __device__ __forceinline__ void set_fill(int bb, int f) const {
    fill[base + bb] = (unsigned char)f;
  }
  __device__ __forceinline__ void put(int bb, int k, int x) const {
    S[k * stride + base + bb] = x;
  }
};

// HBM slots of one set, fill counts in shared memory.
struct GlobalSlotsSmemFill {
  int32_t* G;  // table + off[u]
  int64_t bn;
  unsigned char* fill;
  __device__ __forceinline__ int get_fill(int bb) const { return fill[bb]; }
  __device__ __forceinline__ void set_fill(int bb, int f) const {
    fill[bb] = (unsigned char)f;
  }
  __device__ __forceinline__ void put(int bb, int k, int x) const {
    G[bb + (int64_t)k * bn] = x;
  }
};

// HBM slots of one set; the fill count is re-read from the slots (slots of
// a bucket fill in order, so it is the index of the first -1).
struct GlobalSlotsScan {
  int32_t* G;
  int64_t bn;
  int b;
  __device__ __forceinline__ int get_fill(int bb) const {
    int k = 0;
    while (k < b && __ldcg(G + bb + (int64_t)k * bn) != -1) ++k;
    return k;
  }
  __device__ __forceinline__ void set_fill(int, int) const {}
  __device__ __forceinline__ void put(int bb, int k, int x) const {
    __stcg(G + bb + (int64_t)k * bn, x);
  }
};

// One thread inserts one set sequentially (triangle-count/hashtable.cu:65-74
// rule, CSR order).
template <bool HIER, class Slots>
__device__ void insert_set_thread(const int32_t* __restrict__ keys, int d,
                                  int lg, int lg_max, int b, const Slots& sl,
                                  int32_t* status) {
  const int l = 1 << lg;
  for (int j = 0; j < d; ++j) {
    int x = keys[j];
    int bb = home_bucket<HIER>(x, lg, lg_max);
    int f = sl.get_fill(bb);
    int guard = 0;
    while (f >= b && guard < l) {
      bb = (bb + 1) & (l - 1);
      f = sl.get_fill(bb);
      ++guard;
    }
    if (guard >= l) {
      atomicOr(status, kErrTableFull);
      continue;
    }
    sl.put(bb, f, x);
    sl.set_fill(bb, f + 1);
  }
}

// A warp inserts one set, 32 keys per batch, with the result of sequential
// CSR-order insertion.  Per round, every pending lane finds the first
// non-full bucket B from its current bucket and the fill k0 there; lanes
// aiming at the same bucket are ranked by lane order (match_any).  Lanes
// below the first lane that would overflow its bucket are committed: none of
// them lands outside its bucket, so none can change another's placement.
// The lowest pending lane never overflows, so every round makes progress.
template <bool HIER, class Slots>
__device__ void insert_set_warp(const int32_t* __restrict__ keys, int d,
                                int lg, int lg_max, int b, const Slots& sl,
                                int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int l = 1 << lg;
  const unsigned lt = lanemask_lt(), gt = lanemask_gt();
  // the next round's keys are loaded before this round is inserted, so the
  // load latency overlaps the insertion (long sets take many rounds)
  int xn = lane < d ? __ldg(keys + lane) : 0;
  for (int j0 = 0; j0 < d; j0 += 32) {
    const int j = j0 + lane;
    const bool valid = j < d;
    const int x = xn;
    if (j + 32 < d) xn = __ldg(keys + j + 32);
    int h = valid ? home_bucket<HIER>(x, lg, lg_max) : 0;
    unsigned pending = __ballot_sync(kFull, valid);
    while (pending) {
      const bool me = (pending >> lane) & 1u;
      int B = -1 - lane;  // unique for lanes not in this round
      int k0 = 0;
      bool dropped = false;
      if (me) {
        int f = sl.get_fill(h);
        int guard = 0;
        while (f >= b && guard < l) {
          h = (h + 1) & (l - 1);
          f = sl.get_fill(h);
          ++guard;
        }
        if (guard >= l) {
          atomicOr(status, kErrTableFull);
          dropped = true;
          B = -100 - lane;
        } else {
          B = h;
          k0 = f;
        }
      }
      const unsigned grp = __match_any_sync(kFull, B);
      const int rank = __popc(grp & pending & lt);
      const bool over = me && !dropped && (k0 + rank >= b);
      const unsigned ov = __ballot_sync(kFull, over);
      const unsigned below = ov ? ((1u << (__ffs(ov) - 1)) - 1u) : kFull;
      const bool commit = me && ((below >> lane) & 1u);
      const unsigned cm = __ballot_sync(kFull, commit);
      if (commit && !dropped) {
        sl.put(B, k0 + rank, x);
        if ((grp & cm & gt) == 0) sl.set_fill(B, k0 + rank + 1);
      }
      __syncwarp();
      pending &= ~cm;
    }
  }
}

// Reads one set's slots back in bucket order (slot-major within the set)
// and appends the non-empty ones to out (baseline/common/utils.cu:105-131).
template <class Get>
__device__ void extract_set_warp(int l, int b, int32_t* __restrict__ out,
                                 const Get& get) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  int w = 0;
  const int total = l * b;
  for (int i0 = 0; i0 < total; i0 += 32) {
    int i = i0 + lane;
    int v = -1;
    if (i < total) v = get(i / b, i % b);
    unsigned msk = __ballot_sync(kFull, v != -1);
    if (v != -1) out[w + __popc(msk & lt)] = v;
    w += __popc(msk);
  }
}

// ----------------------------------------------------------- tile build --

template <bool HIER>
__global__ void __launch_bounds__(kTileThreads)
    tile_build_kernel(const int32_t* __restrict__ off,
                      const int32_t* __restrict__ elems,
                      const int32_t* __restrict__ len,
                      const int64_t* __restrict__ off64,
                      const int32_t* __restrict__ tile_first,
                      int64_t bucket_num, int b, int lg_max, int R_max, int LT,
                      int32_t* __restrict__ table,
                      int32_t* __restrict__ hash_out,
                      int32_t* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char smem[];
  int32_t* S = reinterpret_cast<int32_t*>(smem);
  unsigned char* fill = smem + (size_t)R_max * 4 * b;
  __shared__ int s_span[kTileWarps];
  __shared__ int s_wnext;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int s0 = tile_first[blockIdx.x], s1 = tile_first[blockIdx.x + 1];
  int u = s0;
  while (u < s1) {
    // Next segment: big sets are skipped (built by big_build_kernel or
    // build_huge); a run is the maximal span of consecutive tile-sized
    // sets.  Every warp finds it (the same answer, from L1-cached lengths),
    // so no barrier waits for one warp's scan.
    int r = u;
    if (len[u] > LT) {
      r = -(u + 1);
    } else {
      for (;;) {
        int idx = r + lane;
        bool stop = idx >= s1 || len[idx] > LT;
        unsigned msk = __ballot_sync(kFull, stop);
        if (msk) {
          r += __ffs(msk) - 1;
          break;
        }
        r += 32;
      }
    }
    if (r < 0) {  // a big set
      u = -r;
      continue;
    }
    const int64_t RA = off64[u];
    const int R = (int)(off64[r] - RA);  // multiple of 8, <= R_max

    // 1. clear the tile: b planes of R slots to -1, R fill bytes to 0.
    {
      const int4 neg = make_int4(-1, -1, -1, -1);
      const int q = R >> 2;
      for (int k = 0; k < b; ++k) {
        int4* P = reinterpret_cast<int4*>(S + (size_t)k * R_max);
        for (int i = tid; i < q; i += kTileThreads) P[i] = neg;
      }
      int32_t* F = reinterpret_cast<int32_t*>(fill);
      for (int i = tid; i < q; i += kTileThreads) F[i] = 0;
      if (tid == 0) s_wnext = 0;
    }
    __syncthreads();

    // 2a. small sets, one thread each.
    for (int s = u + tid; s < r; s += kTileThreads) {
      int rs = off[s], d = off[s + 1] - rs;
      if (d > kThreadSetMax || d == 0) continue;
      int lg = 31 - __clz(len[s]);
      SmemSlots sl{S, R_max, fill, (int)(off64[s] - RA)};
      insert_set_thread<HIER>(elems + rs, d, lg, lg_max, b, sl, status);
    }
    // 2b. larger sets, one warp each, taken from a shared cursor (a fixed
    // round-robin left warps with one long set waiting at the barrier)
    for (int wround = 0;; ++wround) {
      int s = 0;
      if (kTileDynamic) {
        if (lane == 0) s = u + atomicAdd(&s_wnext, 1);
        s = __shfl_sync(kFull, s, 0);
      } else {
        s = u + warp + kTileWarps * wround;
      }
      if (s >= r) break;
      int rs = off[s], d = off[s + 1] - rs;
      if (d <= kThreadSetMax) continue;
      int lg = 31 - __clz(len[s]);
      SmemSlots sl{S, R_max, fill, (int)(off64[s] - RA)};
      insert_set_warp<HIER>(elems + rs, d, lg, lg_max, b, sl, status);
    }
    fence_proxy_async_smem();
    __syncthreads();

    // 3. planes -> HBM through the bulk-copy engine.
    if (tid == 0) {
      for (int k = 0; k < b; ++k)
        bulk_store(table + (int64_t)k * bucket_num + RA, S + (size_t)k * R_max,
                   (unsigned)R * 4u);
      bulk_commit();
    }
    // 4. optional: rows in bucket order, read from the tile.  The run's sets
    // are consecutive in the tile and their rows consecutive in the CSR, so
    // the rows in bucket order are the tile's non-empty slots in (bucket,
    // slot) order, compacted into hash_out[off[u] .. off[r]): each warp
    // counts a contiguous span of slots, then writes its keys after the
    // spans before it.
    if (hash_out) {
      const int total = R * b;
      const int span = (((total + kTileWarps - 1) / kTileWarps) + 31) & ~31;
      const int i_lo = min(total, warp * span), i_hi = min(total, i_lo + span);
      auto slot = [&](int i) {
        return b == 1 ? S[i] : S[(i % b) * R_max + i / b];
      };
      int c = 0;
      for (int i0 = i_lo; i0 < i_hi; i0 += 32) {
        const int i = i0 + lane;
        c += __popc(__ballot_sync(kFull, i < i_hi && slot(i) != -1));
      }
      if (lane == 0) s_span[warp] = c;
      __syncthreads();
      int w = off[u];
      for (int k = 0; k < warp; ++k) w += s_span[k];
      const unsigned lt = lanemask_lt();
      for (int i0 = i_lo; i0 < i_hi; i0 += 32) {
        const int i = i0 + lane;
        const int v = i < i_hi ? slot(i) : -1;
        const unsigned msk = __ballot_sync(kFull, v != -1);
        if (v != -1) hash_out[w + __popc(msk & lt)] = v;
        w += __popc(msk);
      }
    }
    if (tid == 0) bulk_wait_read_all();
    __syncthreads();
    u = r;
  }
  if (tid == 0) bulk_wait_all();
}

// ------------------------------------------------------------ big build --

template <bool HIER>
__global__ void __launch_bounds__(kThreads)
    big_build_kernel(const int32_t* __restrict__ off,
                     const int32_t* __restrict__ elems,
                     const int32_t* __restrict__ len,
                     const int64_t* __restrict__ off64,
                     const int32_t* __restrict__ big_list, int64_t bucket_num,
                     int b, int lg_max, int32_t* __restrict__ table,
                     int32_t* __restrict__ hash_out,
                     int32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char fill[];
  const int u = big_list[blockIdx.x];
  const int l = len[u];
  const int lg = 31 - __clz(l);
  const int64_t toff = off64[u];
  int32_t* G = table + toff;
  const int tid = threadIdx.x;
  {
    const int4 neg = make_int4(-1, -1, -1, -1);
    for (int k = 0; k < b; ++k) {
      int4* P = reinterpret_cast<int4*>(G + (int64_t)k * bucket_num);
      for (int i = tid; i < (l >> 2); i += kThreads) P[i] = neg;
    }
    if (l <= kBigFillSmemMax) {
      int32_t* F = reinterpret_cast<int32_t*>(fill);
      for (int i = tid; i < (l >> 2); i += kThreads) F[i] = 0;
    }
  }
  __syncthreads();
  const int rs = off[u], d = off[u + 1] - rs;
  if (tid < 32) {
    if (l <= kBigFillSmemMax)
      insert_set_warp<HIER>(elems + rs, d, lg, lg_max, b,
                            GlobalSlotsSmemFill{G, bucket_num, fill}, status);
    else
      insert_set_warp<HIER>(elems + rs, d, lg, lg_max, b,
                            GlobalSlotsScan{G, bucket_num, b}, status);
  }
  __syncthreads();
  if (hash_out && tid < 32 && d > 0)
    extract_set_warp(l, b, hash_out + rs, [&](int bb, int k) {
      return __ldcg(G + bb + (int64_t)k * bucket_num);
    });
}

// ----------------------------------------------------------- huge build --
//
// One set of d >= kHugeKeys keys, built in parallel with exactly the slots
// of sequential CSR-order insertion:
//  1. home bucket of every key, keys per home bucket (cnt);
//  2. the final fills: in linear probing they do not depend on the
//     insertion order -- the keys carried from bucket h to h+1 are
//     c(h+1) = max(0, c(h) + cnt(h) - b), a max-plus recurrence solved by
//     one scan (c -> max(P, c + Q) composes); the table is circular and
//     holds fewer keys than slots, so the carry into bucket 0 is the P of
//     the whole composition;
//  3. clusters = runs of buckets a carry flows through (a bucket with carry
//     0 starts one); keys never leave their home bucket's cluster;
//  4. keys stably sorted by cluster (so CSR order within each), then one
//     thread per cluster replays the sequential rule on its keys.

struct CarryFn {  // c -> max(p, c + q)
  long long p, q;
};
struct ComposeCarry {  // apply a, then b
  __host__ __device__ CarryFn operator()(const CarryFn& a, const CarryFn& b) const {
    return CarryFn{max(b.p, a.p + b.q), a.q + b.q};
  }
};
struct MaxI32 {
  __host__ __device__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

template <bool HIER>
__global__ void huge_home_kernel(const int32_t* __restrict__ keys, int64_t d, int lg,
                                 int lg_max, int32_t* __restrict__ home,
                                 int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int h = home_bucket<HIER>(__ldg(keys + i), lg, lg_max);
    home[i] = h;
    atomicAdd(cnt + h, 1);
  }
}

// Carry functions of the buckets; nxt[h] = the next bucket (circular).
__global__ void huge_fn_kernel(const int32_t* __restrict__ cnt, int64_t l, int b,
                               CarryFn* __restrict__ fn, int32_t* __restrict__ nxt) {
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < l;
       h += (int64_t)gridDim.x * blockDim.x) {
    fn[h] = CarryFn{0, (long long)cnt[h] - b};
    nxt[h] = (int32_t)((h + 1) & (l - 1));
  }
}

// start[h] = h where the carry into bucket h is 0, else -1 (fn holds the
// inclusive prefix compositions).
__global__ void huge_start_kernel(const CarryFn* __restrict__ fn, int64_t l,
                                  int32_t* __restrict__ start) {
  const long long c0 = fn[l - 1].p;
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < l;
       h += (int64_t)gridDim.x * blockDim.x) {
    const long long c = h == 0 ? c0 : max(fn[h - 1].p, c0 + fn[h - 1].q);
    start[h] = c == 0 ? (int32_t)h : -1;
  }
}

// Cluster of every key: the last carry-free bucket at or before its home
// (before bucket 0: the last one of the table, the cluster that wraps).
__global__ void huge_cluster_kernel(const int32_t* __restrict__ home, int64_t d,
                                    const int32_t* __restrict__ cstart, int64_t l,
                                    int32_t* __restrict__ cid, int32_t* __restrict__ idx) {
  const int32_t wrap = cstart[l - 1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cstart[home[i]];
    cid[i] = c >= 0 ? c : wrap;
    idx[i] = (int32_t)i;
  }
}

// One thread per cluster: its keys (sorted_idx[seg .. seg + len), CSR
// order) inserted by the sequential rule; fill[] starts at 0.
__global__ void huge_place_kernel(const int32_t* __restrict__ keys,
                                  const int32_t* __restrict__ home,
                                  const int32_t* __restrict__ sorted_idx,
                                  const int32_t* __restrict__ run_len,
                                  const int32_t* __restrict__ run_off,
                                  const int32_t* __restrict__ n_runs, int64_t l, int b,
                                  int64_t bn, int32_t* __restrict__ fill,
                                  int32_t* __restrict__ nxt, int32_t* __restrict__ G,
                                  int32_t* __restrict__ status) {
  const int64_t nr = *n_runs;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nr;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s0 = run_off[r], s1 = s0 + run_len[r];
    for (int32_t j = s0; j < s1; ++j) {
      const int32_t i = sorted_idx[j];
      // first bucket with room at or after the home bucket: full buckets
      // point further along (nxt, compressed on the way), so a run of
      // repeated keys does not rescan its cluster for every key
      int64_t h = home[i];
      int64_t guard = 0;
      while (fill[h] >= b && guard < l) {
        h = nxt[h];
        ++guard;
      }
      if (guard >= l) {
        atomicOr(status, kErrTableFull);
        continue;
      }
      for (int64_t x = home[i]; x != h && fill[x] >= b;) {  // compress
        const int64_t y = nxt[x];
        nxt[x] = (int32_t)h;
        x = y;
      }
      const int k = fill[h]++;
      G[h + (int64_t)k * bn] = keys[i];
    }
  }
}

// A huge set's rows in bucket order: its non-empty slots in (bucket, slot)
// order, compacted.  Block k covers indices [k*kHugeChunk, (k+1)*kHugeChunk)
// of the l*b (bucket, slot) pairs, each warp a contiguous span of them.
constexpr int kHugeChunk = 8192;

__device__ __forceinline__ int32_t huge_slot(const int32_t* G, int64_t bn, int b, int64_t i) {
  return b == 1 ? G[i] : G[i / b + (i % b) * bn];
}

__device__ __forceinline__ int huge_warp_count(const int32_t* G, int64_t bn, int b,
                                               int64_t lo, int64_t hi) {
  const int lane = threadIdx.x & 31;
  int c = 0;
  for (int64_t i0 = lo; i0 < hi; i0 += 32) {
    const int64_t i = i0 + lane;
    c += __popc(__ballot_sync(kFull, i < hi && huge_slot(G, bn, b, i) != -1));
  }
  return c;
}

__global__ void __launch_bounds__(kThreads)
    huge_count_kernel(const int32_t* __restrict__ G, int64_t bn, int b, int64_t total,
                      int32_t* __restrict__ blk_cnt) {
  __shared__ int s_c[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = (int64_t)blockIdx.x * kHugeChunk;
  const int span = kHugeChunk / kWarps;
  const int64_t lo = min(total, base + (int64_t)warp * span), hi = min(total, lo + span);
  const int c = huge_warp_count(G, bn, b, lo, hi);
  if (lane == 0) s_c[warp] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kWarps; ++w) t += s_c[w];
    blk_cnt[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kThreads)
    huge_write_kernel(const int32_t* __restrict__ G, int64_t bn, int b, int64_t total,
                      const int32_t* __restrict__ blk_off, int32_t* __restrict__ out) {
  __shared__ int s_c[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = (int64_t)blockIdx.x * kHugeChunk;
  const int span = kHugeChunk / kWarps;
  const int64_t lo = min(total, base + (int64_t)warp * span), hi = min(total, lo + span);
  const int c = huge_warp_count(G, bn, b, lo, hi);
  if (lane == 0) s_c[warp] = c;
  __syncthreads();
  int64_t w = blk_off[blockIdx.x];
  for (int k = 0; k < warp; ++k) w += s_c[k];
  const unsigned lt = lanemask_lt();
  for (int64_t i0 = lo; i0 < hi; i0 += 32) {
    const int64_t i = i0 + lane;
    const int32_t v = i < hi ? huge_slot(G, bn, b, i) : -1;
    const unsigned msk = __ballot_sync(kFull, v != -1);
    if (v != -1) out[w + __popc(msk & lt)] = v;
    w += __popc(msk);
  }
}

// (row start, keys, table length, table offset) of each huge set.
__global__ void huge_info_kernel(const int32_t* __restrict__ off,
                                 const int32_t* __restrict__ len,
                                 const int64_t* __restrict__ off64,
                                 const int32_t* __restrict__ huge_list, int nh,
                                 int64_t* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh) return;
  const int u = huge_list[k];
  out[4 * k + 0] = off[u];
  out[4 * k + 1] = (int64_t)off[u + 1] - off[u];
  out[4 * k + 2] = len[u];
  out[4 * k + 3] = off64[u];
}

// ------------------------------------------------- standalone extraction --

__global__ void __launch_bounds__(kThreads)
    extract_kernel(const int32_t* __restrict__ off,
                   const int64_t* __restrict__ off64, int32_t n,
                   const int32_t* __restrict__ table, int64_t bucket_num,
                   int b, int32_t* __restrict__ out) {
  const int warps = gridDim.x * kWarps;
  for (int s = blockIdx.x * kWarps + (threadIdx.x >> 5); s < n; s += warps) {
    int rs = off[s], d = off[s + 1] - rs;
    if (d <= 0) continue;
    int64_t toff = off64[s];
    int l = (int)(off64[s + 1] - toff);
    const int32_t* G = table + toff;
    extract_set_warp(l, b, out + rs, [&](int bb, int k) {
      return __ldg(G + bb + (int64_t)k * bucket_num);
    });
  }
}

int grid_for(int64_t items, int threads, int per_sm = 8) {
  int64_t g = (items + threads - 1) / threads;
  int64_t cap = (int64_t)sm_count() * per_sm;
  if (g > cap) g = cap;
  return (int)(g > 0 ? g : 1);
}

}  // namespace

reset_status make_chunk_rows(const int32_t* d_off, int32_t n, int64_t m,
                             int32_t** d_rows_out, cudaStream_t st) {
  int64_t nc = (m + 31) / 32;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(d_rows_out),
                           sizeof(int32_t) * (nc > 0 ? nc : 1), st));
  RST_CUDA(cudaMemsetAsync(*d_rows_out, 0, sizeof(int32_t) * (nc > 0 ? nc : 1), st));
  note_launch(); layout_kernel<<<grid_for(n, 256), 256, 0, st>>>(
      d_off, nullptr, nullptr, n, nullptr, *d_rows_out, nullptr, 1, 0);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

// Descriptors for offsets other than the build CSR; the table offsets and
// lengths still come from the table.
__global__ void redesc_kernel(const int32_t* __restrict__ off,
                              const int4* __restrict__ src, int32_t n,
                              int4* __restrict__ dst) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    int4 d = src[u];
    int s = off[u];
    d.x = s;
    d.y = off[u + 1] - s;
    dst[u] = d;
  }
}

reset_status make_desc(const reset_table* t, const int32_t* d_off,
                       int4** d_desc_out, cudaStream_t st) {
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(d_desc_out),
                           sizeof(int4) * (t->n > 0 ? t->n : 1), st));
  note_launch(); redesc_kernel<<<grid_for(t->n, 256), 256, 0, st>>>(d_off, t->d_desc, t->n,
                                                     *d_desc_out);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

// Table memory comes from a library-owned stream-ordered pool per device
// whose release threshold is unlimited: freeing a table keeps its pages
// mapped for the next build, so rebuilding a multi-GB table costs no
// cudaMalloc/cudaFree page mapping (reset_release_cached_memory() returns
// them).
namespace {
constexpr int kPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kPoolDevices] = {};
}  // namespace

reset_status table_pool(cudaMemPool_t* out) {
  int dev = 0;
  RST_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kPoolDevices) return arg_fail("device ordinal too large");
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    RST_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    RST_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return RESET_OK;
}

cudaError_t scratch_malloc(void** p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool;
  if (table_pool(&pool) != RESET_OK) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

void release_pools() {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  for (int d = 0; d < kPoolDevices; ++d)
    if (g_pool[d]) cudaMemPoolTrimTo(g_pool[d], 0);
}

}  // namespace rst

using namespace rst;

namespace {

void destroy(reset_table* t) {
  if (!t) return;
  // stream-ordered frees into the table pool (callers synchronise first)
  void* ptrs[] = {t->d_table, t->d_len, t->d_off64, t->d_desc, t->d_chunk_row,
                  t->d_status};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, 0);
  delete t;
}

// The parallel build of one huge set (see huge_home_kernel): row start rs,
// d keys, table length l (a power of two) at offset toff.  Scratch comes
// from the table pool, stream-ordered; no host synchronisation.
template <bool HIER>
reset_status build_huge(const reset_table* t, const int32_t* d_elems, int64_t rs, int64_t d,
                        int64_t l, int64_t toff, int32_t* d_hash_out, cudaStream_t st) {
  const int b = t->bucket;
  const int64_t bn = t->bucket_num;
  const int lg = 63 - __builtin_clzll((unsigned long long)l);
  int32_t* G = t->d_table + toff;
  for (int k = 0; k < b; ++k)
    RST_CUDA(cudaMemsetAsync(G + (int64_t)k * bn, 0xFF, sizeof(int32_t) * (size_t)l, st));
  if (d <= 0) return RESET_OK;
  const int di = (int)d, li = (int)l;
  const int64_t total = l * b;
  const int64_t nblk = (total + kHugeChunk - 1) / kHugeChunk;
  const int32_t* keys = d_elems + rs;
  // CUB temporary sizes
  size_t tb[6] = {0, 0, 0, 0, 0, 0};
  CarryFn* nf = nullptr;
  int32_t* ni = nullptr;
  RST_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tb[0], nf, nf, ComposeCarry(), li, st));
  RST_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tb[1], ni, ni, MaxI32(), li, st));
  RST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb[2], ni, ni, ni, ni, di, 0,
                                           std::max(lg, 1), st));
  RST_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tb[3], ni, ni, ni, ni, di, st));
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb[4], ni, ni, di, st));
  RST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb[5], ni, ni, (int)nblk, st));
  size_t tmp = 0;
  for (size_t x : tb) tmp = std::max(tmp, x);
  // one scratch block: 8 arrays of d ints, 5 of l ints, l carry functions
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t sd = al(4 * (size_t)d), sl = al(4 * (size_t)l);
  const size_t bytes = 8 * sd + 5 * sl + al(sizeof(CarryFn) * (size_t)l) +
                       2 * al(4 * (size_t)(nblk + 1)) + al(16) + al(tmp);
  char* base = nullptr;
  RST_CUDA(scratch_malloc(reinterpret_cast<void**>(&base), bytes, st));
  char* q = base;
  auto carve = [&q](size_t n) {
    char* r = q;
    q += n;
    return r;
  };
  int32_t* home = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* cid = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* idx = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* cid_s = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* idx_s = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* runs = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* run_len = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* run_off = reinterpret_cast<int32_t*>(carve(sd));
  int32_t* cnt = reinterpret_cast<int32_t*>(carve(sl));
  int32_t* start = reinterpret_cast<int32_t*>(carve(sl));
  int32_t* cstart = reinterpret_cast<int32_t*>(carve(sl));
  int32_t* fill = reinterpret_cast<int32_t*>(carve(sl));
  int32_t* nxt = reinterpret_cast<int32_t*>(carve(sl));
  CarryFn* fn = reinterpret_cast<CarryFn*>(carve(al(sizeof(CarryFn) * (size_t)l)));
  int32_t* blk = reinterpret_cast<int32_t*>(carve(al(4 * (size_t)(nblk + 1))));
  int32_t* blk_off = reinterpret_cast<int32_t*>(carve(al(4 * (size_t)(nblk + 1))));
  int32_t* n_runs = reinterpret_cast<int32_t*>(carve(al(16)));
  void* ctmp = carve(al(tmp));

  reset_status rs_out = RESET_OK;
  auto run = [&]() -> reset_status {
    RST_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)l, st));
    RST_CUDA(cudaMemsetAsync(fill, 0, 4 * (size_t)l, st));
    note_launch();
    huge_home_kernel<HIER><<<grid_for(d, kThreads), kThreads, 0, st>>>(keys, d, lg, t->lg_max,
                                                                      home, cnt);
    note_launch();
    huge_fn_kernel<<<grid_for(l, kThreads), kThreads, 0, st>>>(cnt, l, b, fn, nxt);
    size_t x = tmp;
    RST_CUDA(cub::DeviceScan::InclusiveScan(ctmp, x, fn, fn, ComposeCarry(), li, st));
    note_launch();
    huge_start_kernel<<<grid_for(l, kThreads), kThreads, 0, st>>>(fn, l, start);
    x = tmp;
    RST_CUDA(cub::DeviceScan::InclusiveScan(ctmp, x, start, cstart, MaxI32(), li, st));
    note_launch();
    huge_cluster_kernel<<<grid_for(d, kThreads), kThreads, 0, st>>>(home, d, cstart, l, cid,
                                                                    idx);
    x = tmp;
    RST_CUDA(cub::DeviceRadixSort::SortPairs(ctmp, x, cid, cid_s, idx, idx_s, di, 0,
                                             std::max(lg, 1), st));
    x = tmp;
    RST_CUDA(cub::DeviceRunLengthEncode::Encode(ctmp, x, cid_s, runs, run_len, n_runs, di, st));
    x = tmp;
    RST_CUDA(cub::DeviceScan::ExclusiveSum(ctmp, x, run_len, run_off, di, st));
    note_launch();
    huge_place_kernel<<<grid_for(d, kThreads), kThreads, 0, st>>>(
        keys, home, idx_s, run_len, run_off, n_runs, l, b, bn, fill, nxt, G, t->d_status);
    RST_CUDA(cudaGetLastError());
    if (d_hash_out) {
      note_launch();
      huge_count_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(G, bn, b, total, blk);
      x = tmp;
      RST_CUDA(cub::DeviceScan::ExclusiveSum(ctmp, x, blk, blk_off, (int)nblk, st));
      note_launch();
      huge_write_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(G, bn, b, total, blk_off,
                                                             d_hash_out + rs);
      RST_CUDA(cudaGetLastError());
    }
    return RESET_OK;
  };
  rs_out = run();
  cudaFreeAsync(base, st);
  return rs_out;
}

template <bool HIER>
reset_status launch_builds(const reset_table* t, const int32_t* d_off,
                           const int32_t* d_elems, const int32_t* d_tile_first,
                           int32_t n_tiles, const int32_t* d_big, int32_t n_big,
                           const Geom& g, int32_t* d_hash_out, cudaStream_t st) {
  if (n_tiles > 0) {
    RST_CUDA(cudaFuncSetAttribute(tile_build_kernel<HIER>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)g.smem));
    note_launch(); tile_build_kernel<HIER><<<n_tiles, kTileThreads, g.smem, st>>>(
        d_off, d_elems, t->d_len, t->d_off64, d_tile_first, t->bucket_num,
        t->bucket, t->lg_max, g.R_max, g.LT, t->d_table, d_hash_out,
        t->d_status);
    RST_CUDA(cudaGetLastError());
  }
  if (n_big > 0) {
    size_t sm = kBigFillSmemMax;
    RST_CUDA(cudaFuncSetAttribute(big_build_kernel<HIER>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    note_launch(); big_build_kernel<HIER><<<n_big, kThreads, sm, st>>>(
        d_off, d_elems, t->d_len, t->d_off64, d_big, t->bucket_num, t->bucket,
        t->lg_max, t->d_table, d_hash_out, t->d_status);
    RST_CUDA(cudaGetLastError());
  }
  return RESET_OK;
}

}  // namespace

extern "C" {

reset_status reset_table_build(const int32_t* d_off, const int32_t* d_elems,
                               int32_t n, int64_t m, const reset_params* params,
                               int32_t hierarchical, int32_t* d_hash_out,
                               reset_table** out, reset_stream_t stream) {
  if (!out) return arg_fail("out is NULL");
  *out = nullptr;
  reset_params p;
  reset_params_default(&p);
  if (params) p = *params;
  if (n < 0 || m < 0) return arg_fail("negative n or m");
  if (!d_off) return arg_fail("d_off is NULL");
  if (m > 0 && !d_elems) return arg_fail("d_elems is NULL");
  if (!(p.alpha > 0.f && p.alpha <= 1.f))
    return arg_fail("alpha must be in (0, 1]");
  if (p.bucket < 1 || p.bucket > 16) return arg_fail("bucket must be in 1..16");
  if (m > INT32_MAX) return arg_fail("m exceeds the int32 CSR range");
  cudaStream_t st = as_stream(stream);
  const Geom g = tile_geom(p.bucket);

  reset_table* t = new reset_table();
  t->n = n;
  t->m = m;
  t->bucket = p.bucket;
  t->alpha = p.alpha;
  t->hier = hierarchical ? 1 : 0;
  t->build_off = d_off;
  cudaGetDevice(&t->device);

  int32_t* d_info = nullptr;
  int32_t* d_big = nullptr;
  int32_t* d_huge = nullptr;
  int64_t* d_huge_info = nullptr;
  int32_t* d_tile_first = nullptr;
  int64_t* d_bn = nullptr;
  void* d_tmp = nullptr;
  reset_status rs = RESET_OK;
  auto fail = [&](reset_status s) {
    cudaStreamSynchronize(st);
    if (d_info) cudaFreeAsync(d_info, st);
    if (d_big) cudaFreeAsync(d_big, st);
    if (d_huge) cudaFreeAsync(d_huge, st);
    if (d_huge_info) cudaFreeAsync(d_huge_info, st);
    if (d_tile_first) cudaFreeAsync(d_tile_first, st);
    if (d_bn) cudaFreeAsync(d_bn, st);
    if (d_tmp) cudaFreeAsync(d_tmp, st);
    cudaStreamSynchronize(st);
    destroy(t);
    return s;
  };
#define BUILD_CUDA(call)                                                   \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) return fail(cuda_fail(_e, #call, __FILE__, __LINE__)); \
  } while (0)

  cudaMemPool_t pool;
  {
    reset_status ps = table_pool(&pool);
    if (ps != RESET_OK) return fail(ps);
  }
#define POOL_ALLOC(ptr, bytes) \
  BUILD_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&(ptr)), (bytes), pool, st))
  POOL_ALLOC(t->d_status, sizeof(int32_t));
  BUILD_CUDA(cudaMemsetAsync(t->d_status, 0, sizeof(int32_t), st));
  POOL_ALLOC(t->d_len, sizeof(int32_t) * (n > 0 ? n : 1));
  POOL_ALLOC(t->d_off64, sizeof(int64_t) * (n + 1));
  POOL_ALLOC(d_info, sizeof(int32_t) * 4);
  POOL_ALLOC(d_bn, sizeof(int64_t));
  BUILD_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int32_t) * 4, st));
  POOL_ALLOC(d_big, sizeof(int32_t) * (n > 0 ? n : 1));
  POOL_ALLOC(d_huge, sizeof(int32_t) * kMaxHuge);

  if (n > 0) {
    note_launch(); meta_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_off, n, p.alpha, p.bucket,
                                                   g.LT, t->d_len, t->d_off64,
                                                   d_info, d_big, d_huge, t->d_status);
    BUILD_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    BUILD_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, t->d_off64,
                                             t->d_off64, n, st));
    POOL_ALLOC(d_tmp, tmp_bytes);
    BUILD_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, t->d_off64,
                                             t->d_off64, n, st));
  }
  note_launch(); finalize_kernel<<<1, 1, 0, st>>>(t->d_len, t->d_off64, n, d_bn);
  BUILD_CUDA(cudaGetLastError());
  int32_t info[4];
  int64_t bn = 0;
  BUILD_CUDA(cudaMemcpyAsync(info, d_info, sizeof(info), cudaMemcpyDeviceToHost, st));
  BUILD_CUDA(cudaMemcpyAsync(&bn, d_bn, sizeof(bn), cudaMemcpyDeviceToHost, st));
  BUILD_CUDA(cudaStreamSynchronize(st));
  t->bucket_num = bn;
  t->max_len = n > 0 ? info[0] : 8;
  t->lg_max = 31 - __builtin_clz((unsigned)t->max_len);
  const int32_t n_big = info[1];
  const int n_huge = std::min(info[2], kMaxHuge);
  if (bn >= ((int64_t)1 << 56)) return fail(arg_fail("table too large"));
  // huge sets: their rows and table places on the host (one more sync,
  // only for tables that have such sets)
  int64_t huge[4 * kMaxHuge];
  if (n_huge > 0) {
    POOL_ALLOC(d_huge_info, sizeof(int64_t) * 4 * kMaxHuge);
    note_launch(); huge_info_kernel<<<1, kMaxHuge, 0, st>>>(d_off, t->d_len, t->d_off64,
                                                            d_huge, n_huge, d_huge_info);
    BUILD_CUDA(cudaGetLastError());
    BUILD_CUDA(cudaMemcpyAsync(huge, d_huge_info, sizeof(int64_t) * 4 * n_huge,
                               cudaMemcpyDeviceToHost, st));
    BUILD_CUDA(cudaStreamSynchronize(st));
  }

  size_t tbytes = sizeof(int32_t) * (size_t)bn * p.bucket;
  POOL_ALLOC(t->d_table, tbytes > 0 ? tbytes : 16);
  POOL_ALLOC(t->d_desc, sizeof(int4) * (n > 0 ? n : 1));
  t->n_chunks = (m + 31) / 32;
  POOL_ALLOC(t->d_chunk_row, sizeof(int32_t) * (t->n_chunks > 0 ? t->n_chunks : 1));
  const int64_t n_tiles64 = (bn + g.T - 1) / g.T;
  if (n_tiles64 > INT32_MAX) return fail(arg_fail("too many tiles"));
  const int32_t n_tiles = (int32_t)n_tiles64;
  POOL_ALLOC(d_tile_first, sizeof(int32_t) * (n_tiles + 1));
  if (n > 0) {
    note_launch(); layout_kernel<<<grid_for(n, 256), 256, 0, st>>>(
        d_off, t->d_off64, t->d_len, n, t->d_desc, t->d_chunk_row,
        d_tile_first, g.T, n_tiles);
    BUILD_CUDA(cudaGetLastError());
    if (t->hier)
      rs = launch_builds<true>(t, d_off, d_elems, d_tile_first, n_tiles, d_big,
                               n_big, g, d_hash_out, st);
    else
      rs = launch_builds<false>(t, d_off, d_elems, d_tile_first, n_tiles,
                                d_big, n_big, g, d_hash_out, st);
    if (rs != RESET_OK) return fail(rs);
    for (int k = 0; k < n_huge && rs == RESET_OK; ++k) {
      const int64_t* h = huge + 4 * k;
      rs = t->hier ? build_huge<true>(t, d_elems, h[0], h[1], h[2], h[3], d_hash_out, st)
                   : build_huge<false>(t, d_elems, h[0], h[1], h[2], h[3], d_hash_out, st);
    }
    if (rs != RESET_OK) return fail(rs);
  }
  cudaFreeAsync(d_info, st);
  cudaFreeAsync(d_big, st);
  cudaFreeAsync(d_huge, st);
  if (d_huge_info) cudaFreeAsync(d_huge_info, st);
  cudaFreeAsync(d_tile_first, st);
  cudaFreeAsync(d_bn, st);
  if (d_tmp) cudaFreeAsync(d_tmp, st);
#undef POOL_ALLOC
#undef BUILD_CUDA
  *out = t;
  return RESET_OK;
}

reset_status reset_table_info(const reset_table* t, reset_table_view* v) {
  if (!t || !v) return arg_fail("NULL table or view");
  v->n = t->n;
  v->bucket = t->bucket;
  v->max_len = t->max_len;
  v->hierarchical = t->hier;
  v->bucket_num = t->bucket_num;
  v->m = t->m;
  v->alpha = t->alpha;
  v->pad = 0;
  v->d_table = t->d_table;
  v->d_len = t->d_len;
  v->d_off = t->d_off64;
  return RESET_OK;
}

reset_status reset_table_free(reset_table* t) {
  if (!t) return RESET_OK;
  cudaError_t e = cudaDeviceSynchronize();
  destroy(t);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize", __FILE__, __LINE__);
  return RESET_OK;
}

reset_status reset_table_free_async(reset_table* t, reset_stream_t stream) {
  if (!t) return RESET_OK;
  cudaStream_t st = as_stream(stream);
  void* ptrs[] = {t->d_table, t->d_len, t->d_off64, t->d_desc, t->d_chunk_row,
                  t->d_status};
  cudaError_t e = cudaSuccess;
  for (void* p : ptrs)
    if (p) {
      cudaError_t e2 = cudaFreeAsync(p, st);
      if (e == cudaSuccess) e = e2;
    }
  delete t;
  if (e != cudaSuccess) return cuda_fail(e, "cudaFreeAsync", __FILE__, __LINE__);
  return RESET_OK;
}

reset_status reset_release_cached_memory(void) {
  RST_CUDA(cudaDeviceSynchronize());
  release_pools();
  return RESET_OK;
}

reset_status reset_table_check(reset_table* t, reset_stream_t stream) {
  if (!t) return arg_fail("NULL table");
  cudaStream_t st = as_stream(stream);
  int32_t bits = 0;
  RST_CUDA(cudaMemcpyAsync(&bits, t->d_status, sizeof(bits),
                           cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaStreamSynchronize(st));
  if (bits) {
    RST_CUDA(cudaMemsetAsync(t->d_status, 0, sizeof(int32_t), st));
    RST_CUDA(cudaStreamSynchronize(st));
  }
  if (bits & kErrTableFull) {
    set_error("a set did not fit its table (or a CSR row had negative length)");
    return RESET_ERR_TABLE_FULL;
  }
  if (bits & kErrProbeLimit) {
    set_error("a probe walked a whole table without finding an empty slot");
    return RESET_ERR_PROBE_LIMIT;
  }
  if (bits & kErrBadId) {
    set_error("invalid argument: a row, pair or query id was outside [0, n)");
    return RESET_ERR_ARG;
  }
  if (bits & kErrStageTimeout) {
    set_error("a bounded wait for a shared-memory bulk copy gave up");
    return RESET_ERR_TIMEOUT;
  }
  return RESET_OK;
}

reset_status reset_csr_hash_order(const reset_table* t, const int32_t* d_off,
                                  int32_t* d_cols_out, reset_stream_t stream) {
  if (!t || !d_off || (!d_cols_out && t->m > 0))
    return arg_fail("NULL table, offsets or output");
  if (t->n == 0) return RESET_OK;
  cudaStream_t st = as_stream(stream);
  note_launch(); extract_kernel<<<grid_for((int64_t)t->n * 32, kThreads), kThreads, 0, st>>>(
      d_off, t->d_off64, t->n, t->d_table, t->bucket_num, t->bucket,
      d_cols_out);
  RST_CUDA(cudaGetLastError());
  return RESET_OK;
}

}  // extern "C"
