// Served form: a request loop over device-resident indexes with continuous
// batching.
//
// Requests (IR queries, set-similarity pair lists, three-way intersections,
// per-vertex triangle counts, raw pair intersections) are queued on the host
// as they arrive.  One scheduler thread owns `streams` slots; whenever a slot
// is free it drains the queue into a batch -- FIFO, bounded by the batch
// limit and by device memory: every request is charged its device bytes
// against a budget (a share of the free device memory at start-up), and the
// queue head waits while in-flight batches hold the rest.  The batch's
// requests are grouped by (kind, index, threshold); each group gets dense
// input arrays (one pinned buffer, one H2D copy for the whole batch), its
// kernels, and dense outputs (one D2H copy), then an event is recorded.
// Batches on different slots overlap on the GPU; a batch's requests are
// unpacked when its event completes.  A request's result depends only on
// its own inputs and the index, so it is the same alone and in any mix.
//
// Kernels: the planned IR slice kernels of reset_ir, the pair kernel of
// reset_sss, and here a three-way probe and an order-independent table build
// for raw pairs (|A ∩ B| counted with A's multiplicity, the rule of
// set_size/intersection.cu:154-181).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "probe_common.cuh"

namespace rst {
reset_status ir_launch_planned(const reset_table* t, const int32_t* docs,
                               const int32_t* query, const int32_t* qoff,
                               int32_t nq, const int64_t* sl_off,
                               int64_t total_slices, const int64_t* res_off,
                               int32_t* res, int32_t* stage, int32_t* sl_cnt,
                               int64_t* pos, int32_t* cnt, int64_t* packed_off,
                               cudaStream_t st, bool yield = false);
int ir_slice_size();
}  // namespace rst

using namespace rst;

namespace {

constexpr int kThreadsS = 256;

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// ---------------------------------------------------------------- kernels --

// |N(a) ∩ N(b) ∩ N(c)| per triple: the smallest set's keys are probed into
// the middle set's table and, on a hit, into the largest set's table.  One
// warp per triple, lanes over the keys.
template <bool HIER>
__global__ void __launch_bounds__(kThreadsS)
    triple_kernel(const int4* __restrict__ desc, int32_t n,
                  const int32_t* __restrict__ elems,
                  const int32_t* __restrict__ table, int64_t bn, int b,
                  int lg_max, const int32_t* __restrict__ tri, int64_t nt,
                  int32_t* __restrict__ out, int32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = gw; i < nt; i += nw) {
    const int v0 = tri[3 * i], v1 = tri[3 * i + 1], v2 = tri[3 * i + 2];
    if ((unsigned)v0 >= (unsigned)n || (unsigned)v1 >= (unsigned)n ||
        (unsigned)v2 >= (unsigned)n) {
      if (lane == 0) {
        out[i] = 0;
        atomicOr(status, kErrBadId);
      }
      continue;
    }
    int4 d0 = __ldg(desc + v0), d1 = __ldg(desc + v1), d2 = __ldg(desc + v2);
    if (d1.y < d0.y) { int4 t = d0; d0 = d1; d1 = t; }
    if (d2.y < d1.y) { int4 t = d1; d1 = d2; d2 = t; }
    if (d1.y < d0.y) { int4 t = d0; d0 = d1; d1 = t; }
    const int32_t* tb1 = table + desc_toff(d1);
    const int32_t* tb2 = table + desc_toff(d2);
    const int lg1 = desc_lg(d1), lg2 = desc_lg(d2);
    int hits = 0;
    for (int j = lane; j < d0.y; j += 32) {
      const int x = __ldg(elems + d0.x + j);
      if (probe_key<HIER>(x, tb1, lg1, lg_max, bn, b, status) &&
          probe_key<HIER>(x, tb2, lg2, lg_max, bn, b, status))
        ++hits;
    }
    hits = __reduce_add_sync(kFull, hits);
    if (lane == 0) out[i] = hits;
  }
}

// Expands per-vertex triangle requests into (v, w) pairs, w in N(v): pair
// j of vertex k sits at pofs[k] + j.
__global__ void expand_kernel(const int32_t* __restrict__ verts, int64_t nv,
                              const int64_t* __restrict__ pofs,
                              const int32_t* __restrict__ off,
                              const int32_t* __restrict__ cols,
                              int32_t* __restrict__ pa, int32_t* __restrict__ pb) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = gw; k < nv; k += nw) {
    const int v = verts[k];
    const int64_t p0 = pofs[k], np = pofs[k + 1] - p0;
    const int r0 = off[v];
    for (int64_t j = lane; j < np; j += 32) {
      pa[p0 + j] = v;
      pb[p0 + j] = cols[r0 + j];
    }
  }
}

// Raw pairs: B's table (normal hash; slot k of bucket h at h + k*len)
// filled by CAS in any order -- membership does not depend on the order --
// then A probed with the reference's rule.
__global__ void raw_insert_kernel(const int32_t* __restrict__ keys, int64_t nk,
                                  int32_t* __restrict__ tb, int lg, int b,
                                  int32_t* __restrict__ status) {
  const int64_t len = 1ll << lg;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = keys[i];
    int64_t h = x & (len - 1);
    bool placed = false;
    for (int64_t t = 0; t < len && !placed; ++t) {
      for (int k = 0; k < b; ++k) {
        const int old = atomicCAS(tb + h + k * len, -1, x);
        if (old == -1) {
          placed = true;
          break;
        }
      }
      h = (h + 1) & (len - 1);
    }
    if (!placed) atomicOr(status, kErrTableFull);
  }
}

__global__ void raw_probe_kernel(const int32_t* __restrict__ keys, int64_t nk,
                                 const int32_t* __restrict__ tb, int lg, int b,
                                 unsigned long long* __restrict__ count,
                                 int32_t* __restrict__ status) {
  unsigned long long hits = 0;
  const int64_t len = 1ll << lg;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk;
       i += (int64_t)gridDim.x * blockDim.x)
    hits += probe_key<false>(keys[i], tb, lg, lg, len, b, status);
  hits = warp_sum_u64(hits);
  if ((threadIdx.x & 31) == 0 && hits) atomicAdd(count, hits);
}

int grid_for_items(int64_t items, int per_block) {
  int64_t g = (items + per_block - 1) / per_block;
  const int64_t cap = (int64_t)sm_count() * 8;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}

// ------------------------------------------------------------- host side --

struct Index {
  const reset_table* t = nullptr;
  const int32_t* d_off = nullptr;
  const int32_t* d_elems = nullptr;
  std::vector<int32_t> h_off;
  int32_t n() const { return (int32_t)h_off.size() - 1; }
};

// The pinned host arena IR survivors are copied into: one allocation made
// when the server starts, carved first-fit into 256-byte aligned ranges.
// A batch's range is a lease its requests share; the last release returns
// it, so results are handed out without copying and no pinned memory is
// allocated or freed (cudaFreeHost synchronises the device) while serving.
class PinnedArena {
 public:
  ~PinnedArena() {
    if (base_) cudaFreeHost(base_);
  }
  cudaError_t init(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    cudaError_t e = cudaHostAlloc(&base_, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      base_ = nullptr;
      return e;
    }
    free_[0] = bytes;
    return cudaSuccess;
  }
  // A range of `bytes`, or nullptr when none is free.
  char* take(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    std::lock_guard<std::mutex> lk(mu_);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      return static_cast<char*>(base_) + off;
    }
    return nullptr;
  }
  void give(char* p, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    size_t off = (size_t)(p - static_cast<char*>(base_));
    std::lock_guard<std::mutex> lk(mu_);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + bytes == next->first) {  // merge right
      bytes += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {  // merge left
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += bytes;
        return;
      }
    }
    free_[off] = bytes;
  }

 private:
  void* base_ = nullptr;
  std::mutex mu_;
  std::map<size_t, size_t> free_;  // offset -> length
};

struct Lease {
  PinnedArena* arena;
  char* p;
  size_t bytes;
  ~Lease() { arena->give(p, bytes); }
};
using LeaseP = std::shared_ptr<Lease>;

struct Req {
  uint64_t id = 0;
  int32_t kind = 0, index = 0, num = 7, den = 10;
  std::vector<int32_t> a, b;
  int64_t t_arr = 0, t_start = 0, t_done = 0;
  int64_t dev_bytes = 0;
  int64_t cost = 0;  // estimated probes (batch formation)
  int64_t aux = 0;  // IR: df(first term); TC: number of (v, w) pairs; RAW: len
  reset_status status = RESET_OK;
  // IR: what holds the survivors `docs` points into -- an arena lease, or
  // the batch's pageable buffer when the arena was full -- shared by the
  // batch's requests
  std::shared_ptr<const void> docs_owner;
  const int32_t* docs = nullptr;
  std::vector<int64_t> values;
  std::vector<uint8_t> flags;
  int64_t count = 0;
  int64_t batch_id = -1;
  int32_t batch_size = 0;
  bool done = false;
  // placement in its group
  size_t group = 0;
  int64_t item0 = 0;  // first query / pair / triple / vertex of the group
  int64_t res0 = 0;   // IR: first result slot; TC: first pair
};
using ReqP = std::shared_ptr<Req>;

// A growable pinned staging buffer of one slot.  Outgrown buffers are kept
// until the server is destroyed: cudaFreeHost synchronises the device, which
// would stall every batch in flight.
struct Pinned {
  void* p = nullptr;
  size_t cap = 0;
  std::vector<void*> retired;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    const size_t c = std::max(n, cap * 2);
    void* q = nullptr;
    cudaError_t e = cudaHostAlloc(&q, c, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    if (p) retired.push_back(p);
    p = q;
    cap = c;
    return cudaSuccess;
  }
  void release() {
    for (void* q : retired) cudaFreeHost(q);
    retired.clear();
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};


struct Group {
  int32_t kind = 0, index = 0, num = 0, den = 0;
  std::vector<Req*> reqs;
  int64_t items = 0;  // queries / pairs / triples / vertices (RAW: |A|)
  int64_t aux = 0;    // IR: result slots; TC: pairs; RAW: |B|
  int64_t aux2 = 0;   // IR: slices; RAW: len
  size_t in[4] = {0, 0, 0, 0};
  size_t out[2] = {0, 0};
  size_t sc[3] = {0, 0, 0};
  size_t sc3 = 0;
  int64_t dense_n = 0;      // IR: survivors packed on the device
  size_t dense_host = 0;    // IR: their offset (ints) in the slot's result buffer
};

struct Batch {
  int64_t id = 0;
  std::vector<ReqP> reqs;
  std::vector<Group> groups;
  void* d_buf = nullptr;
  size_t in_bytes = 0, out_begin = 0, out_end = 0, d_bytes = 0;
  int64_t reserved = 0;
  int64_t t_launch = 0;
  int phase = 0;  // 0: kernels + small outputs in flight; 1: IR survivors in flight
  bool heavy = false;  // one request above the cost cap
  cudaStream_t st = nullptr;  // the slot stream the batch runs on
  // where the IR survivors land (phase 1): an arena range, or a pageable
  // buffer of the batch when the arena is full
  std::shared_ptr<const void> res;
  const int32_t* res_ptr = nullptr;
  reset_status status = RESET_OK;
};

struct Slot {
  cudaStream_t st = nullptr;     // light batches (highest priority)
  cudaStream_t st_lo = nullptr;  // heavy batches (lowest priority)
  cudaEvent_t ev = nullptr;
  Pinned in, out;
  void* arena = nullptr;  // device buffer reused by this slot's batches
  size_t arena_cap = 0;
  std::unique_ptr<Batch> batch;  // set while its kernels or copies are in flight
  bool busy = false;  // a batch is in flight or with a finisher thread
};

}  // namespace

struct reset_server {
  reset_server_config cfg{};
  int device = 0;
  cudaMemPool_t pool = nullptr;
  std::vector<Index> indexes;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_fin;
  std::deque<ReqP> pending;
  std::unordered_map<uint64_t, ReqP> reqs;
  uint64_t next_id = 1;
  int64_t next_batch = 0;
  int64_t budget = 0, in_use = 0;
  bool stop = false, fin_stop = false;
  std::thread worker;
  // Finished kernels (slot, batch) for the finisher threads, which enqueue
  // the IR survivor copies and hand results out, so that host copies of
  // large results never hold up the scheduler thread.
  std::deque<std::pair<int, std::unique_ptr<Batch>>> finished;
  std::vector<std::thread> finishers;
  int64_t n_done = 0, n_batches = 0, sum_batch = 0, max_batch = 0;
  int64_t max_in_use = 0, max_inflight = 0, inflight = 0, heavy_inflight = 0;
  int64_t launch_ns = 0, batch_ns = 0, max_launch_ns = 0, max_finish_ns = 0;
  PinnedArena results;  // IR survivors handed out without a copy
};

namespace {

constexpr int64_t kReqSlack = 8 * 256;  // alignment slack charged per request

// Validates a request against its index and computes its device bytes.
reset_status plan_request(const reset_server* s, Req* r) {
  const int64_t slice = ir_slice_size();
  if (r->kind != RESET_REQ_RAW &&
      (r->index < 0 || r->index >= (int32_t)s->indexes.size()))
    return arg_fail("unknown index");
  switch (r->kind) {
    case RESET_REQ_IR: {
      const Index& ix = s->indexes[r->index];
      for (int32_t t : r->a)
        if (t < 0 || t >= ix.n()) return arg_fail("IR term out of range");
      const int64_t df = r->a.empty() ? 0 : ix.h_off[r->a[0] + 1] - ix.h_off[r->a[0]];
      r->aux = df;
      const int64_t ns = (df + slice - 1) / slice;
      r->dev_bytes = 4 * (int64_t)r->a.size() + 32 + 4 * df + (4 * slice + 12) * ns;
      // the first list is read and probed against each further term
      r->cost = df * std::max<int64_t>(1, (int64_t)r->a.size() - 1);
      break;
    }
    case RESET_REQ_PAIRS: {
      const Index& ix = s->indexes[r->index];
      if (r->a.size() % 2) return arg_fail("PAIRS takes (a, b) pairs");
      if (r->den <= 0 || r->num < 0) return arg_fail("threshold num/den");
      for (int32_t v : r->a)
        if (v < 0 || v >= ix.n()) return arg_fail("set id out of range");
      r->dev_bytes = 13 * (int64_t)(r->a.size() / 2);
      for (size_t i = 0; i + 1 < r->a.size(); i += 2)
        r->cost += 1 + std::min(ix.h_off[r->a[i] + 1] - ix.h_off[r->a[i]],
                                ix.h_off[r->a[i + 1] + 1] - ix.h_off[r->a[i + 1]]);
      break;
    }
    case RESET_REQ_TRIPLES: {
      const Index& ix = s->indexes[r->index];
      if (r->a.size() % 3) return arg_fail("TRIPLES takes (a, b, c) triples");
      for (int32_t v : r->a)
        if (v < 0 || v >= ix.n()) return arg_fail("set id out of range");
      r->dev_bytes = 16 * (int64_t)(r->a.size() / 3);
      for (size_t i = 0; i + 2 < r->a.size(); i += 3) {
        int64_t lo = INT64_MAX;
        for (int j = 0; j < 3; ++j)
          lo = std::min(lo, (int64_t)(ix.h_off[r->a[i + j] + 1] - ix.h_off[r->a[i + j]]));
        r->cost += 1 + 2 * lo;
      }
      break;
    }
    case RESET_REQ_TC_VERTEX: {
      const Index& ix = s->indexes[r->index];
      int64_t P = 0;
      for (int32_t v : r->a) {
        if (v < 0 || v >= ix.n()) return arg_fail("vertex out of range");
        const int64_t d = ix.h_off[v + 1] - ix.h_off[v];
        P += d;
        r->cost += 1 + d * std::min<int64_t>(d, 256);  // each (v, w) probes <= d keys
      }
      r->aux = P;
      r->dev_bytes = 12 * (int64_t)r->a.size() + 13 * P;
      break;
    }
    case RESET_REQ_RAW: {
      const int64_t nb = (int64_t)r->b.size();
      if (nb > (1ll << 28)) return arg_fail("raw set B too large (at most 2^28 keys)");
      for (int32_t x : r->a)
        if (x < 0) return arg_fail("raw keys must be >= 0");
      for (int32_t x : r->b)
        if (x < 0) return arg_fail("raw keys must be >= 0");
      r->aux = calc_len((int)nb, 0.2f, 5);
      r->dev_bytes = 4 * (int64_t)(r->a.size() + nb) + 20 * r->aux + 16;
      // B's table is cleared (5 slots per bucket) and built (an atomic
      // insertion per key) before A probes it: a large pair is heavy work
      r->cost = (int64_t)r->a.size() + 4 * nb + 5 * r->aux;
      break;
    }
    default:
      return arg_fail("unknown request kind");
  }
  r->dev_bytes += kReqSlack;
  return RESET_OK;
}

bool trivially_empty(const Req& r) {
  switch (r.kind) {
    case RESET_REQ_IR: return r.a.empty();
    case RESET_REQ_PAIRS: case RESET_REQ_TRIPLES: case RESET_REQ_TC_VERTEX:
      return r.a.empty();
    case RESET_REQ_RAW: return r.a.empty() || r.b.empty();
  }
  return false;
}

// Groups, lays out, fills the pinned input, allocates, copies in, launches,
// copies out and records the slot's event.
LeaseP take_lease(reset_server* s, size_t bytes);

// IR batches whose survivors can take at most this many bytes bring them
// back with the small outputs (one round trip instead of two).
constexpr size_t kOnePhaseBytes = size_t(1) << 20;

reset_status launch_batch(reset_server* s, Slot& sl, Batch& bt) {
  const int64_t slice = ir_slice_size();
  // ---- groups
  std::vector<Req*> order;
  for (auto& r : bt.reqs) order.push_back(r.get());
  std::stable_sort(order.begin(), order.end(), [](const Req* x, const Req* y) {
    if (x->kind != y->kind) return x->kind < y->kind;
    if (x->index != y->index) return x->index < y->index;
    if (x->num != y->num) return x->num < y->num;
    return x->den < y->den;
  });
  for (Req* r : order) {
    Group* g = bt.groups.empty() ? nullptr : &bt.groups.back();
    const bool join = g && r->kind != RESET_REQ_RAW && g->kind == r->kind &&
                      g->index == r->index &&
                      (r->kind != RESET_REQ_PAIRS || (g->num == r->num && g->den == r->den));
    if (!join) {
      bt.groups.emplace_back();
      g = &bt.groups.back();
      g->kind = r->kind;
      g->index = r->index;
      g->num = r->num;
      g->den = r->den;
    }
    r->group = bt.groups.size() - 1;
    g->reqs.push_back(r);
    switch (r->kind) {
      case RESET_REQ_IR:
        r->item0 = g->items;
        r->res0 = g->aux;
        g->items += 1;
        g->aux += r->aux;
        g->aux2 += (r->aux + slice - 1) / slice;
        break;
      case RESET_REQ_PAIRS:
        r->item0 = g->items;
        g->items += (int64_t)r->a.size() / 2;
        break;
      case RESET_REQ_TRIPLES:
        r->item0 = g->items;
        g->items += (int64_t)r->a.size() / 3;
        break;
      case RESET_REQ_TC_VERTEX:
        r->item0 = g->items;
        r->res0 = g->aux;
        g->items += (int64_t)r->a.size();
        g->aux += r->aux;
        break;
      case RESET_REQ_RAW:
        g->items = (int64_t)r->a.size();
        g->aux = (int64_t)r->b.size();
        g->aux2 = r->aux;
        break;
    }
  }
  // ---- layout: inputs, outputs, scratch
  size_t p = 0;
  auto take = [&p](size_t bytes) {
    const size_t at = p;
    p = align256(p + std::max<size_t>(bytes, 4));
    return at;
  };
  for (auto& g : bt.groups) {
    switch (g.kind) {
      case RESET_REQ_IR: {
        size_t terms = 0;
        for (Req* r : g.reqs) terms += r->a.size();
        g.in[0] = take(4 * terms);            // terms
        g.in[1] = take(4 * (g.items + 1));    // qoff
        g.in[2] = take(8 * (g.items + 1));    // res_off
        g.in[3] = take(8 * (g.items + 1));    // sl_off
        break;
      }
      case RESET_REQ_PAIRS:
        g.in[0] = take(4 * g.items);
        g.in[1] = take(4 * g.items);
        break;
      case RESET_REQ_TRIPLES:
        g.in[0] = take(12 * g.items);
        break;
      case RESET_REQ_TC_VERTEX:
        g.in[0] = take(4 * g.items);          // vertices
        g.in[1] = take(8 * (g.items + 1));    // pair offsets
        break;
      case RESET_REQ_RAW:
        g.in[0] = take(4 * g.items);
        g.in[1] = take(4 * g.aux);
        break;
    }
  }
  bt.in_bytes = p;
  bt.out_begin = p;
  for (auto& g : bt.groups) {
    switch (g.kind) {
      case RESET_REQ_IR:
        g.out[0] = take(4 * g.items);        // counts
        g.out[1] = take(8 * (g.items + 1));  // dense offsets (last = total)
        break;
      case RESET_REQ_PAIRS:
        g.out[0] = take(4 * g.items);  // intersection sizes
        g.out[1] = take(g.items);      // flags
        break;
      case RESET_REQ_TRIPLES:
        g.out[0] = take(4 * g.items);
        break;
      case RESET_REQ_TC_VERTEX:
        g.out[0] = take(4 * g.aux);    // intersection size per (v, w)
        break;
      case RESET_REQ_RAW:
        g.out[0] = take(16);           // count (u64) + status (i32)
        break;
    }
  }
  bt.out_end = p;
  for (auto& g : bt.groups) {
    switch (g.kind) {
      case RESET_REQ_IR:
        g.sc[0] = take(4 * g.aux2);                      // slice counts
        g.sc[1] = take(4 * (size_t)g.aux2 * slice);      // slice stage
        g.sc[2] = take(4 * g.aux);                       // survivors, packed
        g.sc3 = take(8 * ((size_t)g.aux2 + 1));          // slice positions
        break;
      case RESET_REQ_TC_VERTEX:
        g.sc[0] = take(4 * g.aux);  // pa
        g.sc[1] = take(4 * g.aux);  // pb
        g.sc[2] = take(g.aux);      // flags
        break;
      case RESET_REQ_RAW: g.sc[0] = take(20 * (size_t)g.aux2); break;  // table
      default: break;
    }
  }
  bt.d_bytes = p;

  // ---- pinned input
  const int64_t t_plan = now_ns();
  if (sl.in.ensure(bt.in_bytes) != cudaSuccess || sl.out.ensure(bt.out_end - bt.out_begin) != cudaSuccess)
    return cuda_fail(cudaErrorMemoryAllocation, "pinned staging", __FILE__, __LINE__);
  const int64_t t_pinned = now_ns();
  char* hp = static_cast<char*>(sl.in.p);
  for (auto& g : bt.groups) {
    switch (g.kind) {
      case RESET_REQ_IR: {
        int32_t* terms = reinterpret_cast<int32_t*>(hp + g.in[0]);
        int32_t* qoff = reinterpret_cast<int32_t*>(hp + g.in[1]);
        int64_t* roff = reinterpret_cast<int64_t*>(hp + g.in[2]);
        int64_t* soff = reinterpret_cast<int64_t*>(hp + g.in[3]);
        int32_t pos = 0;
        int64_t q = 0, ro = 0, so = 0;
        for (Req* r : g.reqs) {
          std::memcpy(terms + pos, r->a.data(), 4 * r->a.size());
          qoff[q] = pos;
          roff[q] = ro;
          soff[q] = so;
          pos += (int32_t)r->a.size();
          ro += r->aux;
          so += (r->aux + slice - 1) / slice;
          ++q;
        }
        qoff[q] = pos;
        roff[q] = ro;
        soff[q] = so;
        break;
      }
      case RESET_REQ_PAIRS: {
        int32_t* pa = reinterpret_cast<int32_t*>(hp + g.in[0]);
        int32_t* pb = reinterpret_cast<int32_t*>(hp + g.in[1]);
        for (Req* r : g.reqs) {
          const int64_t k = (int64_t)r->a.size() / 2;
          for (int64_t i = 0; i < k; ++i) {
            pa[r->item0 + i] = r->a[2 * i];
            pb[r->item0 + i] = r->a[2 * i + 1];
          }
        }
        break;
      }
      case RESET_REQ_TRIPLES: {
        int32_t* tri = reinterpret_cast<int32_t*>(hp + g.in[0]);
        for (Req* r : g.reqs) std::memcpy(tri + 3 * r->item0, r->a.data(), 4 * r->a.size());
        break;
      }
      case RESET_REQ_TC_VERTEX: {
        int32_t* verts = reinterpret_cast<int32_t*>(hp + g.in[0]);
        int64_t* pofs = reinterpret_cast<int64_t*>(hp + g.in[1]);
        const Index& ix = s->indexes[g.index];
        int64_t v = 0, pp = 0;
        for (Req* r : g.reqs)
          for (int32_t x : r->a) {
            verts[v] = x;
            pofs[v++] = pp;
            pp += ix.h_off[x + 1] - ix.h_off[x];
          }
        pofs[v] = pp;
        break;
      }
      case RESET_REQ_RAW: {
        Req* r = g.reqs[0];
        std::memcpy(hp + g.in[0], r->a.data(), 4 * r->a.size());
        std::memcpy(hp + g.in[1], r->b.data(), 4 * r->b.size());
        break;
      }
    }
  }

  // ---- device work
  bt.st = bt.heavy ? sl.st_lo : sl.st;
  cudaStream_t st = bt.st;
  if (bt.d_bytes > sl.arena_cap) {  // grow (stream-ordered; the slot is idle)
    if (sl.arena) RST_CUDA(cudaFreeAsync(sl.arena, st));
    sl.arena = nullptr;
    sl.arena_cap = 0;
    const size_t cap = std::max(bt.d_bytes + bt.d_bytes / 4, (size_t)(1u << 20));
    RST_CUDA(cudaMallocFromPoolAsync(&sl.arena, cap, s->pool, st));
    sl.arena_cap = cap;
  }
  bt.d_buf = sl.arena;
  char* dp = static_cast<char*>(bt.d_buf);
  const int64_t t_arena = now_ns();
  RST_CUDA(cudaMemcpyAsync(dp, hp, bt.in_bytes, cudaMemcpyHostToDevice, st));
  for (auto& g : bt.groups) {
    switch (g.kind) {
      case RESET_REQ_IR: {
        const Index& ix = s->indexes[g.index];
        RST_CHECK(ir_launch_planned(
            ix.t, ix.d_elems, reinterpret_cast<int32_t*>(dp + g.in[0]),
            reinterpret_cast<int32_t*>(dp + g.in[1]), (int32_t)g.items,
            reinterpret_cast<int64_t*>(dp + g.in[3]), g.aux2, nullptr,
            reinterpret_cast<int32_t*>(dp + g.sc[2]),
            reinterpret_cast<int32_t*>(dp + g.sc[1]),
            reinterpret_cast<int32_t*>(dp + g.sc[0]),
            reinterpret_cast<int64_t*>(dp + g.sc3),
            reinterpret_cast<int32_t*>(dp + g.out[0]),
            reinterpret_cast<int64_t*>(dp + g.out[1]), st, /*yield=*/bt.heavy));
        break;
      }
      case RESET_REQ_PAIRS: {
        const Index& ix = s->indexes[g.index];
        RST_CHECK(reset_sss(ix.t, nullptr, ix.d_elems,
                            reinterpret_cast<int32_t*>(dp + g.in[0]),
                            reinterpret_cast<int32_t*>(dp + g.in[1]), g.items, g.num,
                            g.den, reinterpret_cast<uint8_t*>(dp + g.out[1]),
                            reinterpret_cast<int32_t*>(dp + g.out[0]), st));
        break;
      }
      case RESET_REQ_TRIPLES: {
        const Index& ix = s->indexes[g.index];
        const reset_table* t = ix.t;
        const int grid = grid_for_items(g.items * 32, kThreadsS);
        note_launch();
        if (t->hier)
          triple_kernel<true><<<grid, kThreadsS, 0, st>>>(
              t->d_desc, t->n, ix.d_elems, t->d_table, t->bucket_num, t->bucket,
              t->lg_max, reinterpret_cast<int32_t*>(dp + g.in[0]), g.items,
              reinterpret_cast<int32_t*>(dp + g.out[0]), t->d_status);
        else
          triple_kernel<false><<<grid, kThreadsS, 0, st>>>(
              t->d_desc, t->n, ix.d_elems, t->d_table, t->bucket_num, t->bucket,
              t->lg_max, reinterpret_cast<int32_t*>(dp + g.in[0]), g.items,
              reinterpret_cast<int32_t*>(dp + g.out[0]), t->d_status);
        RST_CUDA(cudaGetLastError());
        break;
      }
      case RESET_REQ_TC_VERTEX: {
        const Index& ix = s->indexes[g.index];
        int32_t* pa = reinterpret_cast<int32_t*>(dp + g.sc[0]);
        int32_t* pb = reinterpret_cast<int32_t*>(dp + g.sc[1]);
        note_launch();
        expand_kernel<<<grid_for_items(g.items * 32, kThreadsS), kThreadsS, 0, st>>>(
            reinterpret_cast<int32_t*>(dp + g.in[0]), g.items,
            reinterpret_cast<int64_t*>(dp + g.in[1]), ix.d_off, ix.d_elems, pa, pb);
        RST_CUDA(cudaGetLastError());
        if (g.aux > 0)
          RST_CHECK(reset_sss(ix.t, nullptr, ix.d_elems, pa, pb, g.aux, 1, 1,
                              reinterpret_cast<uint8_t*>(dp + g.sc[2]),
                              reinterpret_cast<int32_t*>(dp + g.out[0]), st));
        break;
      }
      case RESET_REQ_RAW: {
        int32_t* tab = reinterpret_cast<int32_t*>(dp + g.sc[0]);
        unsigned long long* cnt = reinterpret_cast<unsigned long long*>(dp + g.out[0]);
        int32_t* status = reinterpret_cast<int32_t*>(dp + g.out[0] + 8);
        const int lg = 31 - __builtin_clz((unsigned)g.aux2);
        RST_CUDA(cudaMemsetAsync(tab, 0xFF, 20 * (size_t)g.aux2, st));
        RST_CUDA(cudaMemsetAsync(dp + g.out[0], 0, 16, st));
        note_launch();
        raw_insert_kernel<<<grid_for_items(g.aux, kThreadsS), kThreadsS, 0, st>>>(
            reinterpret_cast<int32_t*>(dp + g.in[1]), g.aux, tab, lg, 5, status);
        note_launch();
        raw_probe_kernel<<<grid_for_items(g.items, kThreadsS), kThreadsS, 0, st>>>(
            reinterpret_cast<int32_t*>(dp + g.in[0]), g.items, tab, lg, 5, cnt, status);
        RST_CUDA(cudaGetLastError());
        break;
      }
    }
  }
  // Small IR batches: copy each group's whole survivor region (bounded by
  // the first terms' lengths) into an arena range now, so the batch
  // completes in one phase; larger ones copy only the survivors once their
  // number is known (enqueue_results).
  size_t ir_bound = 0;
  for (auto& g : bt.groups)
    if (g.kind == RESET_REQ_IR) ir_bound += 4 * (size_t)g.aux;
  if (ir_bound > 0 && ir_bound <= kOnePhaseBytes) {
    if (LeaseP lease = take_lease(s, ir_bound)) {
      size_t at = 0;
      for (auto& g : bt.groups) {
        if (g.kind != RESET_REQ_IR) continue;
        g.dense_host = at / 4;
        if (g.aux > 0)
          RST_CUDA(cudaMemcpyAsync(lease->p + at, dp + g.sc[2], 4 * (size_t)g.aux,
                                   cudaMemcpyDeviceToHost, st));
        at += 4 * (size_t)g.aux;
      }
      bt.res_ptr = reinterpret_cast<const int32_t*>(lease->p);
      bt.res = std::move(lease);
      bt.phase = 1;
    }
  }
  RST_CUDA(cudaMemcpyAsync(sl.out.p, dp + bt.out_begin, bt.out_end - bt.out_begin,
                           cudaMemcpyDeviceToHost, st));
  RST_CUDA(cudaEventRecord(sl.ev, st));
  // RESET_SERVER_TRACE=<ms>: report launches slower than that, by phase
  static const double trace_ms = [] {
    const char* v = std::getenv("RESET_SERVER_TRACE");
    return v ? std::atof(v) : -1.0;
  }();
  const int64_t t_end = now_ns();
  if (trace_ms >= 0 && (t_end - bt.t_launch) / 1e6 > trace_ms)
    std::fprintf(stderr,
                 "reset_server: batch %lld (%zu requests, %zu device bytes, %s) launched in "
                 "%.3f ms: plan %.3f, pinned staging %.3f, arena %.3f, copies + kernels %.3f\n",
                 (long long)bt.id, bt.reqs.size(), bt.d_bytes, bt.heavy ? "heavy" : "light",
                 (t_end - bt.t_launch) / 1e6, (t_plan - bt.t_launch) / 1e6,
                 (t_pinned - t_plan) / 1e6, (t_arena - t_pinned) / 1e6, (t_end - t_arena) / 1e6);
  return RESET_OK;
}

// Copies a finished batch's outputs into its requests (no lock held).
void unpack_batch(const reset_server* s, Slot& sl, Batch& bt) {
  const char* hp = static_cast<const char*>(sl.out.p);
  auto at = [&](size_t off) { return hp + (off - bt.out_begin); };
  for (auto& rp : bt.reqs) {
    Req* r = rp.get();
    const Group& g = bt.groups[r->group];
    switch (r->kind) {
      case RESET_REQ_IR: {
        const int32_t c = reinterpret_cast<const int32_t*>(at(g.out[0]))[r->item0];
        const int64_t o = reinterpret_cast<const int64_t*>(at(g.out[1]))[r->item0];
        r->count = c;
        const int32_t* src = bt.res_ptr + g.dense_host + o;
        if (c == 0) {
          r->docs = nullptr;
        } else {  // hand out the batch's buffer itself
          r->docs_owner = bt.res;
          r->docs = src;
        }
        break;
      }
      case RESET_REQ_PAIRS: {
        const int64_t k = (int64_t)r->a.size() / 2;
        const int32_t* in = reinterpret_cast<const int32_t*>(at(g.out[0])) + r->item0;
        const uint8_t* fl = reinterpret_cast<const uint8_t*>(at(g.out[1])) + r->item0;
        r->values.assign(in, in + k);
        r->flags.assign(fl, fl + k);
        int64_t c = 0;
        for (int64_t i = 0; i < k; ++i) c += fl[i];
        r->count = c;
        break;
      }
      case RESET_REQ_TRIPLES: {
        const int64_t k = (int64_t)r->a.size() / 3;
        const int32_t* o = reinterpret_cast<const int32_t*>(at(g.out[0])) + r->item0;
        r->values.assign(o, o + k);
        int64_t c = 0;
        for (int64_t i = 0; i < k; ++i) c += o[i];
        r->count = c;
        break;
      }
      case RESET_REQ_TC_VERTEX: {
        const int32_t* o = reinterpret_cast<const int32_t*>(at(g.out[0])) + r->res0;
        const Index& ix = s->indexes[r->index];
        r->values.resize(r->a.size());
        int64_t p = 0, c = 0;
        for (size_t i = 0; i < r->a.size(); ++i) {
          const int32_t v = r->a[i];
          int64_t sum = 0;
          for (int64_t j = 0; j < ix.h_off[v + 1] - ix.h_off[v]; ++j) sum += o[p++];
          r->values[i] = sum;
          c += sum;
        }
        r->count = c;
        break;
      }
      case RESET_REQ_RAW: {
        const char* o = at(g.out[0]);
        uint64_t c;
        int32_t stt;
        std::memcpy(&c, o, 8);
        std::memcpy(&stt, o + 8, 4);
        r->count = (int64_t)c;
        if (stt) r->status = RESET_ERR_TABLE_FULL;
        break;
      }
    }
  }
}

// A lease of `bytes` in the server's result arena, or nullptr when the
// arena is full (results still held by clients).
LeaseP take_lease(reset_server* s, size_t bytes) {
  char* p = s->results.take(bytes);
  if (!p) return nullptr;
  try {
    return LeaseP(new Lease{&s->results, p, bytes});
  } catch (const std::bad_alloc&) {
    s->results.give(p, bytes);
    return nullptr;
  }
}

// After the kernels (finisher thread): copies every IR group's packed
// survivors (sizes now known on the host) into an arena range, or, when the
// arena is full, into a pageable buffer of the batch.  Returns true if
// copies were enqueued (the batch completes at the next event).
bool enqueue_results(reset_server* s, Slot& sl, Batch& bt) {
  const char* hp = static_cast<const char*>(sl.out.p);
  size_t total = 0;
  for (auto& g : bt.groups) {
    if (g.kind != RESET_REQ_IR) continue;
    g.dense_n = reinterpret_cast<const int64_t*>(hp + (g.out[1] - bt.out_begin))[g.items];
    g.dense_host = total;
    total += (size_t)g.dense_n;
  }
  if (total == 0) return false;
  if (LeaseP lease = take_lease(s, 4 * total)) {
    bt.res_ptr = reinterpret_cast<const int32_t*>(lease->p);
    bt.res = std::move(lease);
  } else {
    // Arena full (clients still hold results): a pageable buffer of the
    // batch.  Its copies return once done (pageable destination), which
    // only this finisher thread waits for; pinned memory is never
    // allocated while serving (cudaHostAlloc can stall other CUDA calls).
    try {
      auto buf = std::make_shared<std::vector<int32_t>>(total);
      bt.res_ptr = buf->data();
      bt.res = std::move(buf);
    } catch (const std::bad_alloc&) {
      bt.status = RESET_ERR_OOM;
      return false;
    }
  }
  const char* dp = static_cast<const char*>(bt.d_buf);
  for (auto& g : bt.groups) {
    if (g.kind != RESET_REQ_IR || g.dense_n == 0) continue;
    cudaError_t e = cudaMemcpyAsync(const_cast<int32_t*>(bt.res_ptr) + g.dense_host,
                                    dp + g.sc[2], 4 * (size_t)g.dense_n,
                                    cudaMemcpyDeviceToHost, bt.st);
    if (e != cudaSuccess) {
      bt.status = cuda_fail(e, "result copy", __FILE__, __LINE__);
      return false;
    }
  }
  cudaError_t e = cudaEventRecord(sl.ev, bt.st);
  if (e != cudaSuccess) {
    bt.status = cuda_fail(e, "cudaEventRecord", __FILE__, __LINE__);
    return false;
  }
  bt.phase = 1;
  return true;
}

void worker_main(reset_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool progressed = false;
    // completions go to the finisher threads (the slot stays busy)
    for (size_t i = 0; i < s->slots.size(); ++i) {
      Slot& sl = s->slots[i];
      if (!sl.batch) continue;
      cudaError_t q = cudaEventQuery(sl.ev);
      if (q == cudaErrorNotReady) continue;
      std::unique_ptr<Batch> bt = std::move(sl.batch);
      if (q != cudaSuccess) bt->status = cuda_fail(q, "server batch", __FILE__, __LINE__);
      s->finished.emplace_back((int)i, std::move(bt));
      s->cv_fin.notify_one();
      progressed = true;
    }
    // launches
    for (auto& sl : s->slots) {
      if (sl.busy || s->pending.empty()) continue;
      auto bt = std::make_unique<Batch>();
      int64_t bytes = 0, cost = 0;
      // Requests are taken in arrival order while the batch's estimated
      // probes stay under the cap.  A request above the cap is "heavy": it
      // runs alone, and only while another slot stays open for the rest;
      // when it cannot start, lighter requests behind it (within a window)
      // may pass it.
      const int64_t cap = s->cfg.max_batch_cost > 0 ? s->cfg.max_batch_cost : INT64_MAX;
      const bool heavy_room = s->slots.size() == 1 ||
                              s->heavy_inflight + 1 < (int64_t)s->slots.size();
      int passed = 0;
      for (auto it = s->pending.begin();
           it != s->pending.end() && (int64_t)bt->reqs.size() < s->cfg.max_batch_requests;) {
        ReqP r = *it;
        if (r->dev_bytes > s->budget) {  // can never fit: fail it
          r->status = RESET_ERR_OOM;
          r->t_done = now_ns();
          r->done = true;
          ++s->n_done;
          it = s->pending.erase(it);
          progressed = true;
          s->cv_done.notify_all();
          continue;
        }
        if (r->cost > cap) {
          if (bt->reqs.empty() && heavy_room) {
            if (s->in_use + r->dev_bytes > s->budget) break;  // wait for memory
            bytes = r->dev_bytes;
            bt->reqs.push_back(r);
            bt->heavy = true;
            it = s->pending.erase(it);
            break;
          }
          if (!bt->reqs.empty() || ++passed > 64) break;  // a light batch ends here
          ++it;  // pass the heavy request it cannot start now
          continue;
        }
        if (!bt->reqs.empty() && cost + r->cost > cap) break;
        if (s->in_use + bytes + r->dev_bytes > s->budget) break;  // wait for memory
        bytes += r->dev_bytes;
        cost += r->cost;
        bt->reqs.push_back(r);
        it = s->pending.erase(it);
      }
      if (bt->reqs.empty()) continue;
      if (bt->heavy) ++s->heavy_inflight;
      bt->id = s->next_batch++;
      bt->reserved = bytes;
      s->in_use += bytes;
      s->max_in_use = std::max(s->max_in_use, s->in_use);
      ++s->inflight;
      s->max_inflight = std::max(s->max_inflight, s->inflight);
      ++s->n_batches;
      s->sum_batch += (int64_t)bt->reqs.size();
      s->max_batch = std::max<int64_t>(s->max_batch, (int64_t)bt->reqs.size());
      const int64_t t = now_ns();
      for (auto& r : bt->reqs) {
        r->t_start = t;
        r->batch_id = bt->id;
        r->batch_size = (int32_t)bt->reqs.size();
      }
      sl.busy = true;
      lk.unlock();
      bt->t_launch = t;
      reset_status rs = launch_batch(s, sl, *bt);
      const int64_t t_launched = now_ns();
      if (rs != RESET_OK) {
        bt->status = rs;
        cudaEventRecord(sl.ev, bt->st ? bt->st : sl.st);  // completes once the slot drains
      }
      lk.lock();
      s->launch_ns += t_launched - t;
      s->max_launch_ns = std::max(s->max_launch_ns, t_launched - t);
      sl.batch = std::move(bt);
      progressed = true;
    }
    if (s->stop && s->pending.empty() && s->inflight == 0) break;
    if (!progressed) {
      if (s->inflight > 0)
        s->cv_work.wait_for(lk, std::chrono::microseconds(20));
      else
        s->cv_work.wait(lk, [s] { return s->stop || !s->pending.empty(); });
    }
  }
}

// Finisher thread: takes batches whose event completed; a phase-0 batch with
// IR survivors gets their copies enqueued and goes back in flight, any other
// has its results handed to its requests, and its slot is freed.
void finisher_main(reset_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_fin.wait(lk, [s] { return s->fin_stop || !s->finished.empty(); });
    if (s->finished.empty()) break;  // fin_stop: the scheduler has drained
    const int i = s->finished.front().first;
    std::unique_ptr<Batch> bt = std::move(s->finished.front().second);
    s->finished.pop_front();
    Slot& sl = s->slots[i];
    lk.unlock();
    const int64_t t0 = now_ns();
    if (bt->status == RESET_OK && bt->phase == 0 && enqueue_results(s, sl, *bt)) {
      const int64_t t1 = now_ns();
      lk.lock();
      s->max_finish_ns = std::max(s->max_finish_ns, t1 - t0);
      sl.batch = std::move(bt);  // survivors in flight; the scheduler polls the event
      s->cv_work.notify_one();
      continue;
    }
    if (bt->status == RESET_OK) unpack_batch(s, sl, *bt);
    const int64_t t = now_ns();
    lk.lock();
    s->max_finish_ns = std::max(s->max_finish_ns, t - t0);
    s->batch_ns += t - bt->t_launch;
    for (auto& r : bt->reqs) {
      if (bt->status != RESET_OK) r->status = bt->status;
      r->t_done = t;
      r->done = true;
      ++s->n_done;
    }
    s->in_use -= bt->reserved;
    --s->inflight;
    if (bt->heavy) --s->heavy_inflight;
    sl.busy = false;
    s->cv_done.notify_all();
    s->cv_work.notify_one();
  }
}

}  // namespace

extern "C" {

void reset_server_config_default(reset_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->streams = 4;
  c->max_batch_requests = 1024;
  c->max_batch_cost = int64_t(1) << 22;
  c->mem_budget_bytes = 0;
  c->pinned_result_bytes = int64_t(256) << 20;
}

int64_t reset_now_ns(void) { return now_ns(); }

reset_status reset_server_create(const reset_server_config* cfg, reset_server** out) {
  if (!out) return arg_fail("NULL output");
  *out = nullptr;
  reset_server_config c;
  reset_server_config_default(&c);
  if (cfg) c = *cfg;
  if (c.streams < 1 || c.streams > 64) return arg_fail("streams must be in 1..64");
  if (c.max_batch_requests < 1) return arg_fail("max_batch_requests must be >= 1");
  if (c.mem_budget_bytes < 0) return arg_fail("negative memory budget");
  if (c.max_batch_cost < 0) return arg_fail("negative max_batch_cost");
  if (c.pinned_result_bytes < 0) return arg_fail("negative pinned_result_bytes");
  if (c.pinned_result_bytes == 0) c.pinned_result_bytes = int64_t(256) << 20;
  std::unique_ptr<reset_server> s;
  try {
    s.reset(new reset_server());
  } catch (const std::bad_alloc&) {
    return RESET_ERR_OOM;
  }
  s->cfg = c;
  RST_CUDA(cudaGetDevice(&s->device));
  size_t freeb = 0, totalb = 0;
  RST_CUDA(cudaMemGetInfo(&freeb, &totalb));
  s->budget = c.mem_budget_bytes > 0 ? c.mem_budget_bytes : (int64_t)(freeb / 2);
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->device;
  RST_CUDA(cudaMemPoolCreate(&s->pool, &props));
  uint64_t keep = UINT64_MAX;
  RST_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  s->slots.resize(c.streams);
  // light batches run at the highest stream priority, heavy ones at the
  // lowest, so blocks of light batches are scheduled first as SMs free up
  int prio_lo = 0, prio_hi = 0;
  RST_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  for (auto& sl : s->slots) {
    RST_CUDA(cudaStreamCreateWithPriority(&sl.st, cudaStreamNonBlocking, prio_hi));
    RST_CUDA(cudaStreamCreateWithPriority(&sl.st_lo, cudaStreamNonBlocking, prio_lo));
    RST_CUDA(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
  }
  RST_CUDA(s->results.init((size_t)c.pinned_result_bytes));
  // finisher threads (one per slot, at most four), then the scheduler
  try {
    const int nf = std::min(c.streams, 4);
    for (int i = 0; i < nf; ++i) s->finishers.emplace_back(finisher_main, s.get());
    s->worker = std::thread(worker_main, s.get());
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = s->fin_stop = true;
    }
    s->cv_fin.notify_all();
    for (auto& f : s->finishers) f.join();
    return arg_fail("cannot start the server threads");
  }
  *out = s.release();
  return RESET_OK;
}

reset_status reset_server_add_index(reset_server* s, const reset_table* t,
                                    const int32_t* d_off, const int32_t* d_elems,
                                    int32_t* index_out) {
  if (!s || !t || !index_out) return arg_fail("NULL argument");
  if (d_off != t->build_off) return arg_fail("d_off must be the offsets the table was built on");
  if (!d_elems && t->m > 0) return arg_fail("NULL elements");
  Index ix;
  ix.t = t;
  ix.d_off = d_off;
  ix.d_elems = d_elems;
  try {
    ix.h_off.resize((size_t)t->n + 1);
  } catch (const std::bad_alloc&) {
    return RESET_ERR_OOM;
  }
  RST_CUDA(cudaMemcpy(ix.h_off.data(), d_off, 4 * ((size_t)t->n + 1), cudaMemcpyDeviceToHost));
  // Device bytes of the largest single request on this index (an IR query
  // of up to six terms whose first list is the longest set).  Slot arenas
  // are grown to it now: growing one while serving maps new pool memory in
  // the scheduler thread, which stalled every arrival behind a heavy
  // request by 20-60 ms.
  int64_t max_len = 0;
  for (int32_t u = 0; u < t->n; ++u)
    max_len = std::max<int64_t>(max_len, ix.h_off[u + 1] - ix.h_off[u]);
  const int64_t slice = ir_slice_size();
  const size_t need = (size_t)(4 * 6 + 32 + 4 * max_len +
                               (4 * slice + 12) * ((max_len + slice - 1) / slice)) +
                      (size_t(1) << 16);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->inflight == 0) {  // slots idle: grow their arenas (stream-ordered, then waited for)
    for (auto& sl : s->slots) {
      if (sl.busy || sl.arena_cap >= need) continue;
      if (sl.arena) RST_CUDA(cudaFreeAsync(sl.arena, sl.st));
      sl.arena = nullptr;
      sl.arena_cap = 0;
      RST_CUDA(cudaMallocFromPoolAsync(&sl.arena, need, s->pool, sl.st));
      RST_CUDA(cudaStreamSynchronize(sl.st));
      sl.arena_cap = need;
    }
  }
  s->indexes.push_back(std::move(ix));
  *index_out = (int32_t)s->indexes.size() - 1;
  return RESET_OK;
}

reset_status reset_server_submit(reset_server* s, const reset_request* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return arg_fail("NULL argument");
  if (q->nargs < 0 || q->nargs2 < 0) return arg_fail("negative argument count");
  if ((q->nargs > 0 && !q->args) || (q->nargs2 > 0 && !q->args2)) return arg_fail("NULL arguments");
  ReqP r;
  try {
    r = std::make_shared<Req>();
    r->a.assign(q->args, q->args + q->nargs);
    if (q->kind == RESET_REQ_RAW) r->b.assign(q->args2, q->args2 + q->nargs2);
  } catch (const std::bad_alloc&) {
    return RESET_ERR_OOM;
  }
  r->kind = q->kind;
  r->index = q->index;
  r->num = q->num;
  r->den = q->den;
  if (r->kind != RESET_REQ_PAIRS) r->num = r->den = 0;
  r->t_arr = q->arrival_ns > 0 ? q->arrival_ns : now_ns();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return RESET_ERR_BUSY;
  reset_status ps = plan_request(s, r.get());
  if (ps != RESET_OK) return ps;
  r->id = s->next_id++;
  s->reqs[r->id] = r;
  *ticket = r->id;
  if (trivially_empty(*r)) {
    const int64_t t = now_ns();
    r->t_start = r->t_done = t;
    if (r->kind == RESET_REQ_TC_VERTEX) r->values.assign(r->a.size(), 0);
    r->done = true;
    ++s->n_done;
    s->cv_done.notify_all();
    return RESET_OK;
  }
  s->pending.push_back(r);
  s->cv_work.notify_one();
  return RESET_OK;
}

reset_status reset_server_wait(reset_server* s, uint64_t ticket, int32_t timeout_ms,
                               reset_result* out) {
  if (!s || !out) return arg_fail("NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return arg_fail("unknown ticket");
  ReqP r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return RESET_ERR_TIMEOUT;
  std::memset(out, 0, sizeof(*out));
  out->status = r->status;
  out->kind = r->kind;
  out->count = r->count;
  out->docs = r->docs;
  out->ndocs = r->docs ? r->count : 0;
  out->values = r->values.empty() ? nullptr : r->values.data();
  out->nvalues = (int64_t)r->values.size();
  out->flags = r->flags.empty() ? nullptr : r->flags.data();
  out->queue_us = (r->t_start - r->t_arr) / 1e3;
  out->service_us = (r->t_done - r->t_start) / 1e3;
  out->latency_us = (r->t_done - r->t_arr) / 1e3;
  out->batch_id = r->batch_id;
  out->batch_size = r->batch_size;
  return RESET_OK;
}

reset_status reset_server_release(reset_server* s, uint64_t ticket) {
  if (!s) return arg_fail("NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return arg_fail("unknown ticket");
  if (!it->second->done) return RESET_ERR_BUSY;
  s->reqs.erase(it);
  return RESET_OK;
}

reset_status reset_server_stats(reset_server* s, reset_server_counters* st) {
  if (!s || !st) return arg_fail("NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  st->completed = s->n_done;
  st->batches = s->n_batches;
  st->max_batch = s->max_batch;
  st->mean_batch = s->n_batches ? (double)s->sum_batch / s->n_batches : 0.0;
  st->pending = (int64_t)s->pending.size();
  st->inflight_batches = s->inflight;
  st->max_inflight_batches = s->max_inflight;
  st->budget_bytes = s->budget;
  st->in_use_bytes = s->in_use;
  st->max_in_use_bytes = s->max_in_use;
  st->launch_host_us = s->launch_ns / 1e3;
  st->batch_us = s->batch_ns / 1e3;
  st->max_launch_us = s->max_launch_ns / 1e3;
  st->max_finish_us = s->max_finish_ns / 1e3;
  int64_t arena = 0;
  for (auto& sl : s->slots) arena += (int64_t)sl.arena_cap;
  st->arena_bytes = arena;
  return RESET_OK;
}

reset_status reset_server_destroy(reset_server* s) {
  if (!s) return RESET_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();  // returns once nothing is in flight
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->fin_stop = true;
  }
  s->cv_fin.notify_all();
  for (auto& f : s->finishers)
    if (f.joinable()) f.join();
  cudaError_t e = cudaSuccess;
  for (auto& sl : s->slots) {
    for (cudaStream_t* p : {&sl.st, &sl.st_lo}) {
      if (!*p) continue;
      cudaError_t e2 = cudaStreamSynchronize(*p);
      if (e == cudaSuccess) e = e2;
      cudaStreamDestroy(*p);
    }
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.arena) cudaFree(sl.arena);
    sl.in.release();
    sl.out.release();
  }
  s->reqs.clear();  // their leases go back to the arena, freed with the server
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
  if (e != cudaSuccess) return cuda_fail(e, "reset_server_destroy", __FILE__, __LINE__);
  return RESET_OK;
}

}  // extern "C"
