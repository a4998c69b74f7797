// Internal definitions shared by the libreset translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "reset.h"

namespace rst {

// ---------------------------------------------------------------- errors --

// Records a message for reset_last_error_string() on this host thread.
void set_error(const char* fmt, ...);
// Maps a CUDA error to a status (and records it).
reset_status cuda_fail(cudaError_t e, const char* what, const char* file,
                       int line);
reset_status arg_fail(const char* what);

#define RST_CUDA(call)                                                  \
  do {                                                                  \
    cudaError_t _e = (call);                                            \
    if (_e != cudaSuccess)                                              \
      return ::rst::cuda_fail(_e, #call, __FILE__, __LINE__);           \
  } while (0)

#define RST_CHECK(expr)                                                 \
  do {                                                                  \
    reset_status _s = (expr);                                           \
    if (_s != RESET_OK) return _s;                                      \
  } while (0)

// Device-side error bits (OR-ed into reset_table::d_status).
enum : int32_t {
  kErrTableFull = 1,
  kErrProbeLimit = 2,
  kErrBadId = 4,       // a row or pair id outside [0, n)
  kErrStageTimeout = 8,  // a bounded wait for a bulk copy into shared memory gave up
};

constexpr uint32_t kFull = 0xffffffffu;

inline cudaStream_t as_stream(reset_stream_t s) {
  return reinterpret_cast<cudaStream_t>(s);
}

// ------------------------------------------------------- per-set layout --

// Packed per-set descriptor, one 16-byte load per set on the probe path:
//   x = first element of the set's row in the CSR
//   y = number of elements (row length)
//   z = low 32 bits of the set's table offset (in buckets)
//   w = bits 32..55 of the table offset | log2(len) << 24
__host__ __device__ __forceinline__ int64_t desc_toff(int4 d) {
  return (int64_t)(uint32_t)d.z | ((int64_t)(d.w & 0xFFFFFF) << 32);
}
__host__ __device__ __forceinline__ int desc_lg(int4 d) {
  return (int)((uint32_t)d.w >> 24);
}

// calculate_length (triangle-count/hashtable.cu:21-36): float division,
// truncation, strict next power of two, at least 8.
__host__ __device__ __forceinline__ int calc_len(int degree, float alpha,
                                                 int bucket) {
  float q = (float)degree / alpha;
  int total = (int)q;
  int length = total / bucket;
  if (length == 0) return 8;
  length |= length >> 1;
  length |= length >> 2;
  length |= length >> 4;
  length |= length >> 8;
  length |= length >> 16;
  length++;
  if (length < 8) length = 8;
  return length;
}

// Home bucket.  Normal: x & (len-1) (TC.cuh:48-52).  Hierarchical:
// (x & (max_len-1)) >> (log2 max_len - log2 len) (TC.cuh:40-46), written
// with logs since both lengths are powers of two.
template <bool HIER>
__device__ __forceinline__ int home_bucket(int x, int lg, int lg_max) {
  if (HIER) return (x & ((1 << lg_max) - 1)) >> (lg_max - lg);
  return x & ((1 << lg) - 1);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned lanemask_gt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_gt;" : "=r"(r));
  return r;
}

}  // namespace rst

// ------------------------------------------------------------ the table --

struct reset_table {
  int32_t n = 0;
  int32_t bucket = 5;
  int32_t max_len = 8;
  int32_t lg_max = 3;
  int32_t hier = 1;
  float alpha = 0.2f;
  int64_t bucket_num = 0;
  int64_t m = 0;
  int device = 0;
  int32_t* d_table = nullptr;    // bucket * bucket_num
  int32_t* d_len = nullptr;      // n
  int64_t* d_off64 = nullptr;    // n + 1
  int4* d_desc = nullptr;        // n packed descriptors (see desc_toff)
  int32_t* d_chunk_row = nullptr;  // row of edge 32*c, for c < n_chunks
  int64_t n_chunks = 0;
  const int32_t* build_off = nullptr;  // CSR offsets the table was built on
  int32_t* d_status = nullptr;   // device error bits
};

namespace rst {
// Descriptor + chunk-row arrays for a CSR other than the build CSR (used when
// a probe call passes offsets that are not the ones the table was built
// from).  Allocated on `stream` with cudaMallocAsync; the caller frees.
reset_status make_desc(const reset_table* t, const int32_t* d_off,
                       int4** d_desc_out, cudaStream_t stream);
reset_status make_chunk_rows(const int32_t* d_off, int32_t n, int64_t m,
                             int32_t** d_rows_out, cudaStream_t stream);
int sm_count();
// Process-wide kernel tuning knobs (reset_set_tuning).
reset_tuning tuning();
// The library-owned table memory pool of the current device.
reset_status table_pool(cudaMemPool_t* out);
// Stream-ordered scratch from the same pool (it keeps freed pages mapped,
// unlike the device's default pool, which unmaps them at every sync).
cudaError_t scratch_malloc(void** p, size_t bytes, cudaStream_t st);
// Vertex-staged triangle counting (tc_staged.cu); *count must be zeroed.
reset_status tc_staged(const reset_table* t, const int4* desc,
                       const int32_t* d_cols, int64_t m,
                       unsigned long long* count, cudaStream_t st);
// Owner-grouped triangle counting (tc_owner.cu): sum over the edges (u, v)
// of the edge CSR of |K(u) ∩ K(v)|, K = the key CSR t was built on (the
// graph itself for plain TC); tables staged in shared memory, keys streamed
// with 16-byte loads (kcols 16-byte aligned); *count must be zeroed.  With
// owner_hits (n zeroed u64), every owner's hits are also added there.
reset_status tc_owner(const reset_table* t, const int4* kdesc, const int32_t* koff,
                      const int32_t* kcols, int64_t mk, const int32_t* eoff,
                      const int32_t* ecols, const int32_t* echunk_rows, int64_t me,
                      unsigned long long* count, cudaStream_t st,
                      unsigned long long* owner_hits = nullptr);
// Owner-grouped pair decisions (sss_owner.cu).  Scratch for n sets and up to
// `cap` pairs comes from one stream-ordered allocation.
struct PairOwnerScratch {
  int32_t *cnt = nullptr, *goff = nullptr, *pidx = nullptr, *wlist = nullptr,
          *dlist = nullptr, *ctr = nullptr;
  int2 *ent = nullptr, *units = nullptr, *dunits = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  void* base = nullptr;
};
reset_status pair_owner_alloc(int32_t n, int64_t cap, PairOwnerScratch* s, cudaStream_t st);
void pair_owner_free(PairOwnerScratch* s, cudaStream_t st);
// Decisions for the pairs p < cap (or p < *np_dev); elems 16-byte aligned,
// cap <= INT32_MAX.  No allocation, no host synchronisation.
reset_status pair_owner_launch(const reset_table* t, const int4* desc, const int32_t* elems,
                               int64_t m, const int32_t* pa, const int32_t* pb, int64_t cap,
                               const int64_t* np_dev, bool float_rule, int32_t num, int32_t den,
                               float thr, uint8_t* flags, int32_t* inter,
                               const PairOwnerScratch& s, cudaStream_t st);
// pair_owner_alloc + launch + stream-ordered free.
reset_status sss_owner(const reset_table* t, const int4* desc, const int32_t* elems, int64_t m,
                       const int32_t* pa, const int32_t* pb, int64_t np, bool float_rule,
                       int32_t num, int32_t den, float thr, uint8_t* flags, int32_t* inter,
                       cudaStream_t st);
// Counts launches of libreset's own kernels (reset_kernel_launches()).
void note_launch(int k = 1);
}  // namespace rst
