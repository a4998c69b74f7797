// Device helpers of the owner-grouped probe kernels (tc_owner.cu,
// sss_owner.cu): 1-D bulk copies of a set's table into shared memory
// (cp.async.bulk completing on an mbarrier, with bounded waits), the
// reference probe rule walked in the staged copy, and the flattened 16-byte
// key streaming of up to 32 probing rows against one staged table.
#pragma once

#include "common.cuh"
#include "probe_common.cuh"

namespace rst {

constexpr int kWaitLimit = 1 << 22;  // polls of a bulk-copy barrier before giving up

// Launch shape and bins of the owner-grouped kernels.
constexpr int kOT = 512;                 // threads per CTA (2 CTAs, 32 warps per SM)
constexpr int kOW = kOT / 32;            // warps per CTA
// Ints of shared memory per CTA for staged tables (80 KB): every power-of-two
// plane size with b = 1, 2, 4 or 5 slots that 96 KB held still fits, and the
// 16 KB saved doubles the pending-probe queues of the triangle count.
constexpr int kCtaTab = 20480;
constexpr int kWarpTab = kCtaTab / kOW;  // a warp's region (1280 ints)
constexpr int kCtaSeg = 8192;            // probers per CTA work unit
// Probers a warp takes at a time from a CTA unit.  A unit averages a few
// hundred probers of ~100-300 keys each; taking 32 at a time left 16 warps
// with one or two uneven batches, so the CTA waited ~1/3 of each unit at
// its closing barrier (modelled on the scale-20 groups: 65% balance at 32,
// 92% at 8).  Each batch still flattens its rows' keys across the lanes.
constexpr int kGrab = 8;
constexpr int kBigGroup = 256;           // groups above this are CTA work
constexpr int kCtaWork = 32768;          // probes that make a smaller group CTA work
constexpr int kDirSeg = 256;             // probers per direct work unit

// Bin of every owner w with a non-empty group ent[goff[w] .. goff[w+1])
// ({row start, row length} of each prober): 0 = CTA work (units (w, seg)
// of kCtaSeg probers), 1 = warp work, 2 = direct probes into the HBM table
// (staging does not pay, or the table does not fit shared memory) for
// groups of at most 32 probers, 3 = the same for larger groups, cut into
// units (w, seg) of kDirSeg probers so that no warp serialises a hub's
// whole group.  ctr[0..2] and ctr[6] count the four lists.  Grid-stride
// over owners, block-uniform loop (warp collectives inside).
__device__ __forceinline__ void classify_owners(const int4* __restrict__ desc,
                                                const int32_t* __restrict__ goff,
                                                const int2* __restrict__ ent, int32_t n, int b,
                                                int2* __restrict__ units,
                                                int32_t* __restrict__ wlist,
                                                int32_t* __restrict__ dlist,
                                                int2* __restrict__ dunits,
                                                int32_t* __restrict__ ctr) {
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
          bin = P > 32 ? 3 : 2;
          if (bin == 3) nunits = (P + kDirSeg - 1) / kDirSeg;
        } else if (big || T > kWarpTab) {
          bin = 0;
          nunits = (P + kCtaSeg - 1) / kCtaSeg;
        } else {
          bin = 1;
        }
      }
    }
    // warp-aggregated appends
#pragma unroll
    for (int which = 0; which <= 3; which += 3) {
      int tot;
      const int pre = warp_excl_scan(bin == which ? nunits : 0, &tot);
      int* c = ctr + (which == 0 ? 0 : 6);
      int b0 = 0;
      if (lane == 0 && tot) b0 = atomicAdd(c, tot);
      b0 = __shfl_sync(kFull, b0, 0);
      int2* u = which == 0 ? units : dunits;
      if (bin == which)
        for (int s = 0; s < nunits; ++s) u[b0 + pre + s] = make_int2((int)w, s);
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

// Issues the bulk copies of one set's table (b planes of 1 << lg ints, plane
// k at table + toff + k*bn in HBM) into S, plane k at S + k * (1 << lg).
__device__ __forceinline__ void stage_table(int* S, const int32_t* __restrict__ table,
                                            int64_t toff, int lg, int64_t bn, int b,
                                            uint64_t* bar) {
  const int L = 1 << lg;
  const uint32_t plane = (uint32_t)L * 4u;
  fence_proxy_async_smem();
  mbar_expect_tx(bar, plane * (uint32_t)b);
  for (int k = 0; k < b; ++k) bulk_g2s(S + (int64_t)k * L, table + toff + k * bn, plane, bar);
}

// Continues search_in_hashtable (TC.cu:11-31) in a staged table (plane k at
// S + k*L) from slot k of bucket h (k == b: the next bucket's slot 0); the
// slots before it held other keys.  Same bound as probe_key (the table).
__device__ __forceinline__ unsigned smem_walk(int x, const int* S, int L, int h, int k, int b,
                                              int32_t* status) {
  const int cap = L * b;
  for (int t = 0; t < cap; ++t) {
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

// Pending probes one round of 32 lanes x 4 keys can queue.
constexpr int kQueue = 128;

// Waits (bounded) for a staged table; with one slot per bucket the writer
// then appends a copy of bucket 0 after the last bucket (S[L] = S[0]), so
// the home bucket's successor is S[h + 1] without a wrap.  Neither region
// size (kCtaTab, kWarpTab) is a power of two, so a staged b = 1 table (a
// power of two) ends strictly inside its region and S[L] is in it too.  The
// caller's barrier publishes the copy.
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity, int* S, int lg, int b,
                                           bool writer) {
  const bool ok = mbar_wait(bar, parity);
  if (ok && writer && b == 1) S[1 << lg] = S[0];
  return ok;
}

// Walks queued keys q[0, nq) of one staged table (all lanes, nq
// warp-uniform): each key's first two probe slots held other keys, so its
// walk resumes after them -- slot 2 of its home bucket, or with one slot per
// bucket the bucket after the next.  Returns this lane's hits.
template <bool HIER>
__device__ __forceinline__ unsigned walk_keys(const int* q, int nq, const int* S, int lg,
                                              int lg_max, int b, int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int L = 1 << lg;
  const unsigned hmask = HIER ? ((1u << lg_max) - 1u) : (unsigned)(L - 1);
  const int hsh = HIER ? (lg_max - lg) : 0;
  const int inc1 = b > 1 ? 0 : 1;
  const int kcont = b > 1 ? 2 : 1;
  unsigned hits = 0;
  __syncwarp();
  for (int i = lane; i < nq; i += 32) {
    const int x = q[i];
    const int h = (int)(((unsigned)x & hmask) >> hsh);
    hits += smem_walk(x, S, L, h + inc1, kcont, b, status);
  }
  __syncwarp();
  return hits;
}

// Largest lane k < NR with P_k <= f (P nondecreasing across lanes, P_0 = 0;
// every row at or past NR is empty).
template <int NR>
__device__ __forceinline__ int owner_lane_n(int P, int f) {
  int k = 0;
#pragma unroll
  for (int step = NR / 2; step >= 1; step >>= 1) {
    const int pk = __shfl_sync(kFull, P, k + step);
    if (pk <= f) k += step;
  }
  return k;
}

// The keys of up to NR probing rows (NR a power of two <= 32; lane i:
// ent[i] = {row start, row length} in cols) looked up in one staged table
// (plane k at S + k*L; with b = 1 padded by stage_wait).  The rows' 16-byte
// chunks are flattened across the lanes (round r: lane i loads chunk 32r+i
// of the concatenation, its row found by a shuffle binary search over the NR
// rows) and R rounds are in flight at once.  Elements of a chunk outside its
// row become the sentinel -2, which matches no slot (keys are >= 0, empty
// slots -1), so every element is probed without a validity test.  Every
// key's first two probe slots (slots 0 and 1 of its home bucket; with one
// slot per bucket, the home and next bucket) are read and resolved without
// branching; probes that both slots leave open are queued in this warp's
// shared-memory queue (qx, qh: QCAP entries each, QCAP >= kQueue) and walked
// by all lanes together once more than QCAP - kQueue are pending (and before
// returning), so the rare long walks neither idle the warp nor run with few
// lanes.  Returns this lane's hits; with PAIRS, the hits of row i are also
// added to s_cnt[i] (32 shared-memory counters of this warp, zeroed by the
// caller).
//
// KEEP (counting only): the queue holds keys alone (their walk restarts from
// the hash) and outlives the call: *nq_keep carries its length from call to
// call over one staged table, and the caller walks the rest with walk_keys
// before the table changes.
//
// PF: the next R chunks of keys are loaded before the current ones are
// probed (software pipelining across rounds).
//
// CW: keys per lane and round (4: one 16-byte load; 8: two, so the row
// search and chunk bookkeeping are paid once per 8 keys).
template <bool HIER, int R, bool PAIRS = false, int NR = 32, int QCAP = kQueue,
          bool KEEP = false, bool PF = false, int CW = 4>
__device__ __forceinline__ unsigned staged_keys(const int2* __restrict__ ent, int cnt,
                                                const int32_t* __restrict__ cols, int64_t m,
                                                const int* S, int lg, int lg_max, int b,
                                                int32_t* status, int* qx, int* qh,
                                                int* s_cnt = nullptr, int* nq_keep = nullptr) {
  static_assert(NR >= 1 && NR <= 32 && (NR & (NR - 1)) == 0, "NR: a power of two <= 32");
  static_assert(CW == 4 || CW == 8, "chunks of 4 or 8 keys");
  static_assert(QCAP >= 32 * CW, "the queue must hold one round");
  constexpr int kShift = CW == 8 ? 3 : 2;
  static_assert(!(KEEP && PAIRS), "a kept queue carries no rows");
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int2 e = lane < cnt ? __ldg(ent + lane) : make_int2(0, 0);
  const int64_t end = (int64_t)e.x + e.y;
  const int nc = e.y > 0 ? (int)(((end + CW - 1) >> kShift) - (e.x >> kShift)) : 0;
  int total;
  const int P = warp_excl_scan(nc, &total);
  const int L = 1 << lg;
  const unsigned hmask = HIER ? ((1u << lg_max) - 1u) : (unsigned)(L - 1);
  const int hsh = HIER ? (lg_max - lg) : 0;
  // the second probe slot: slot 1 of the home bucket, or (b = 1) the next
  // bucket, S[h + 1] in the padded copy; a queued walk continues from slot
  // kcont of bucket h + inc1
  const int off1 = b > 1 ? L : 1;
  const int inc1 = b > 1 ? 0 : 1;
  const int kcont = b > 1 ? 2 : 1;
  const int4* __restrict__ cols4 = reinterpret_cast<const int4*>(cols);
  const int64_t full = m >> kShift;  // chunks that lie wholly inside cols
  unsigned hits = 0;
  int nq = KEEP ? *nq_keep : 0;  // queued probes (warp-uniform)
  auto walk_queue = [&]() {
    if (KEEP) {
      hits += walk_keys<HIER>(qx, nq, S, lg, lg_max, b, status);
      nq = 0;
      return;
    }
    __syncwarp();
    for (int i = lane; i < nq; i += 32) {
      const int v = qh[i];
      const unsigned hit = smem_walk(qx[i], S, L, v >> 10, (v >> 5) & 31, b, status);
      if (PAIRS) {
        if (hit) atomicAdd(s_cnt + (v & 31), 1);
      } else {
        hits += hit;
      }
    }
    __syncwarp();
    nq = 0;
  };
  // Loads the R chunks of rounds [base, base + 32R) of this lane: keys in
  // x (-2 outside rows), rows in kk (-1 if none).
  auto load = [&](int base, int (&x)[R][CW], int (&kk)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      kk[r] = -1;
#pragma unroll
      for (int j = 0; j < CW; ++j) x[r][j] = -2;
      if (base + r * 32 < total) {  // warp-uniform
        const int f = base + r * 32 + lane;
        const int k = owner_lane_n<NR>(P, f);
        const int kp = __shfl_sync(kFull, P, k);
        const int kb = __shfl_sync(kFull, e.x, k);
        const int kd = __shfl_sync(kFull, e.y, k);
        if (f < total) {
          kk[r] = k;
          // m <= 2^31 - 16 (checked on the host): CW*c + CW - 1 fits an int
          const int c = (kb >> kShift) + (f - kp);
          const int i0 = c * CW;
          const int lo = kb - i0;       // elements j < lo precede the row
          const int hi = kb + kd - i0;  // elements j >= hi follow it
          if (c < full) {
#pragma unroll
            for (int v = 0; v < CW / 4; ++v) {
              const int4 q = __ldg(cols4 + (CW / 4) * c + v);
              x[r][4 * v + 0] = q.x;
              x[r][4 * v + 1] = q.y;
              x[r][4 * v + 2] = q.z;
              x[r][4 * v + 3] = q.w;
            }
          } else {
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (j >= lo && j < hi) x[r][j] = __ldg(cols + i0 + j);
          }
          if (lo > 0 || hi < CW) {  // the first or last chunk of its row
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (j < lo || j >= hi) x[r][j] = -2;
          }
        }
      }
    }
  };
  // Probes the keys of rounds [base, base + 32R).
  auto probe = [&](int base, const int (&x)[R][CW], const int (&kk)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (base + r * 32 >= total) break;  // warp-uniform
      unsigned hr = 0;
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        const int xx = x[r][j];
        const int h = (int)(((unsigned)xx & hmask) >> hsh);
        const int s0 = S[h];
        const int s1 = S[h + off1];
        hr += (unsigned)((s0 == xx) | ((s0 != -1) & (s1 == xx)));
        const bool pend = (s0 != xx) & (s0 != -1) & (s1 != xx) & (s1 != -1);
        const unsigned pm = __ballot_sync(kFull, pend);
        if (pend) {
          // continue at slot 2 of the home bucket (or, one slot per bucket,
          // at the bucket after h + 1); the row rides along for PAIRS
          const int pos = nq + __popc(pm & lt);
          qx[pos] = xx;
          if (!KEEP) qh[pos] = ((h + inc1) << 10) | (kcont << 5) | (kk[r] & 31);
        }
        nq += __popc(pm);
      }
      if (nq > QCAP - 32 * CW) walk_queue();
      hits += hr;
      if (PAIRS) {
        const unsigned grp = __match_any_sync(kFull, kk[r]);
        const unsigned sum = __reduce_add_sync(grp, hr);
        if (kk[r] >= 0 && lane == __ffs(grp) - 1 && sum) atomicAdd(s_cnt + kk[r], (int)sum);
      }
    }
  };
  if (PF) {
    // the next R chunks are loaded before this round's keys are probed,
    // so their latency hides behind the probes
    int xn[R][CW], kn[R];
    if (total > 0) load(0, xn, kn);
    for (int base = 0; base < total; base += 32 * R) {
      int x[R][CW], kk[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        kk[r] = kn[r];
#pragma unroll
        for (int j = 0; j < CW; ++j) x[r][j] = xn[r][j];
      }
      if (base + 32 * R < total) load(base + 32 * R, xn, kn);
      probe(base, x, kk);
    }
  } else {
    for (int base = 0; base < total; base += 32 * R) {
      int x[R][CW], kk[R];
      load(base, x, kk);
      probe(base, x, kk);
    }
  }
  if (KEEP)
    *nq_keep = nq;
  else if (nq)
    walk_queue();
  return hits;
}

}  // namespace rst
