// Batched set-similarity form: one persistent, CUDA-graph-captured launch
// that decides thousands of pairs of uneven sizes.
//
// reset_batch owns device buffers for up to `capacity` pairs and a CUDA graph
// of three nodes: a 4-byte memset that writes the pair count, a memset that
// clears the work cursor, and the persistent pair kernel (dynamic 32-pair
// chunks; pairs with a warp's worth of keys probed by a whole warp, smaller
// ones flattened across lanes).  A run patches the count into the
// instantiated graph (cudaGraphExecMemsetNodeSetParams, which only affects
// later launches) and replays it: no host synchronisation, allocation or
// per-batch launch setup.  Same decisions as reset_sss (den*I >= num*U).
#include "common.cuh"

namespace rst {
reset_status sss_launch_persistent(const reset_table* t, const int32_t* elems,
                                   const int32_t* pa, const int32_t* pb,
                                   const int64_t* np_dev,
                                   unsigned long long* cursor, int64_t capacity,
                                   int32_t num, int32_t den, uint8_t* flags,
                                   int32_t* inter, bool decisions_only,
                                   cudaStream_t st);
}

struct reset_batch {
  const reset_table* t = nullptr;
  const int32_t* elems = nullptr;
  int64_t capacity = 0;
  int32_t num = 7, den = 10;
  int32_t *pa = nullptr, *pb = nullptr, *inter = nullptr;
  uint8_t* flags = nullptr;
  int64_t* np_dev = nullptr;
  unsigned long long* cursor = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphNode_t count_node = nullptr;
  cudaMemsetParams count_params{};
  cudaGraphExec_t exec = nullptr;
  rst::PairOwnerScratch owner{};  // RESET_BATCH_OWNER_GROUPED: grouping scratch
};

using namespace rst;

namespace {
void batch_destroy(reset_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->pa);
  cudaFree(b->pb);
  cudaFree(b->inter);
  cudaFree(b->flags);
  cudaFree(b->np_dev);
  cudaFree(b->cursor);
  if (b->owner.base) {
    pair_owner_free(&b->owner, nullptr);
    cudaStreamSynchronize(nullptr);
  }
  delete b;
}
}  // namespace

extern "C" {

reset_status reset_batch_create(const reset_table* t, const int32_t* d_elems,
                                int64_t capacity, int32_t num, int32_t den,
                                reset_batch** out, reset_stream_t stream) {
  return reset_batch_create_ex(t, d_elems, capacity, num, den, 0, out, stream);
}

reset_status reset_batch_create_ex(const reset_table* t, const int32_t* d_elems,
                                   int64_t capacity, int32_t num, int32_t den,
                                   int32_t options, reset_batch** out,
                                   reset_stream_t stream) {
  if (options & ~(RESET_BATCH_DECISIONS_ONLY | RESET_BATCH_OWNER_GROUPED))
    return arg_fail("unknown batch option");
  if (!t || !out) return arg_fail("NULL table or output");
  if (!d_elems && t->m > 0) return arg_fail("NULL elements");
  const bool owner = (options & RESET_BATCH_OWNER_GROUPED) != 0;
  if (owner && ((reinterpret_cast<uintptr_t>(d_elems) & 15) != 0 || t->m > INT32_MAX - 4))
    return arg_fail("owner-grouped batches need 16-byte aligned elements, at most 2^31 - 5");
  if (capacity < 1 || capacity > INT32_MAX) return arg_fail("capacity must be in 1..2^31-1");
  if (den <= 0 || num < 0) return arg_fail("threshold num/den");
  *out = nullptr;
  reset_batch* b = new reset_batch();
  b->t = t;
  b->elems = d_elems;
  b->capacity = capacity;
  b->num = num;
  b->den = den;
  (void)stream;
  cudaError_t e = cudaMalloc(&b->pa, sizeof(int32_t) * capacity);
  if (e == cudaSuccess) e = cudaMalloc(&b->pb, sizeof(int32_t) * capacity);
  if (e == cudaSuccess) e = cudaMalloc(&b->inter, sizeof(int32_t) * capacity);
  if (e == cudaSuccess) e = cudaMalloc(&b->flags, capacity);
  if (e == cudaSuccess) e = cudaMalloc(&b->np_dev, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&b->cursor, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    batch_destroy(b);
    return cuda_fail(e, "reset_batch_create allocation", __FILE__, __LINE__);
  }
  // np_dev's high word stays 0; the count node writes the low word
  e = cudaMemset(b->np_dev, 0, sizeof(int64_t));
  if (e == cudaSuccess && owner) {  // grouping scratch for `capacity` pairs
    reset_status ps = pair_owner_alloc(t->n, capacity, &b->owner, nullptr);
    if (ps == RESET_OK) e = cudaStreamSynchronize(nullptr);
    if (ps != RESET_OK) {
      batch_destroy(b);
      return ps;
    }
  }
  // capture the kernel, then put the two memset nodes in front of it
  cudaStream_t cap = nullptr;
  reset_status rs = RESET_OK;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    if (owner)
      rs = pair_owner_launch(t, t->d_desc, d_elems, t->m, b->pa, b->pb, capacity, b->np_dev,
                             false, num, den, 0.f, b->flags, b->inter, b->owner, cap);
    else
      rs = sss_launch_persistent(t, d_elems, b->pa, b->pb, b->np_dev, b->cursor, capacity,
                                 num, den, b->flags, b->inter,
                                 (options & RESET_BATCH_DECISIONS_ONLY) != 0, cap);
    cudaError_t e2 = cudaStreamEndCapture(cap, &b->graph);
    if (e == cudaSuccess) e = e2;
  }
  if (cap) cudaStreamDestroy(cap);
  size_t nroots = 0;
  cudaGraphNode_t root = nullptr;
  if (e == cudaSuccess && rs == RESET_OK) e = cudaGraphGetRootNodes(b->graph, nullptr, &nroots);
  if (e == cudaSuccess && rs == RESET_OK && nroots != 1) rs = arg_fail("unexpected batch graph");
  if (e == cudaSuccess && rs == RESET_OK) e = cudaGraphGetRootNodes(b->graph, &root, &nroots);
  cudaGraphNode_t cursor_node = nullptr;
  if (e == cudaSuccess && rs == RESET_OK) {
    b->count_params.dst = b->np_dev;
    b->count_params.value = 0;
    b->count_params.elementSize = 4;
    b->count_params.width = 1;
    b->count_params.height = 1;
    b->count_params.pitch = 0;
    e = cudaGraphAddMemsetNode(&b->count_node, b->graph, nullptr, 0, &b->count_params);
  }
  if (e == cudaSuccess && rs == RESET_OK) {
    cudaMemsetParams cp{};
    cp.dst = b->cursor;
    cp.value = 0;
    cp.elementSize = 4;
    cp.width = 2;
    cp.height = 1;
    e = cudaGraphAddMemsetNode(&cursor_node, b->graph, nullptr, 0, &cp);
  }
  if (e == cudaSuccess && rs == RESET_OK) {
    cudaGraphNode_t from[2] = {b->count_node, cursor_node};
    cudaGraphNode_t to[2] = {root, root};
    e = cudaGraphAddDependencies(b->graph, from, to, 2);
  }
  if (e == cudaSuccess && rs == RESET_OK) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (rs != RESET_OK || e != cudaSuccess) {
    batch_destroy(b);
    if (rs != RESET_OK) return rs;
    return cuda_fail(e, "reset_batch_create graph", __FILE__, __LINE__);
  }
  *out = b;
  return RESET_OK;
}

reset_status reset_batch_buffers(reset_batch* b, int32_t** d_pair_a,
                                 int32_t** d_pair_b, uint8_t** d_flags,
                                 int32_t** d_inter) {
  if (!b) return arg_fail("NULL batch");
  if (d_pair_a) *d_pair_a = b->pa;
  if (d_pair_b) *d_pair_b = b->pb;
  if (d_flags) *d_flags = b->flags;
  if (d_inter) *d_inter = b->inter;
  return RESET_OK;
}

reset_status reset_batch_run(reset_batch* b, int64_t npairs,
                             reset_stream_t stream) {
  if (!b) return arg_fail("NULL batch");
  if (npairs < 0 || npairs > b->capacity) return arg_fail("npairs exceeds the batch capacity");
  cudaStream_t st = as_stream(stream);
  b->count_params.value = (unsigned int)npairs;
  RST_CUDA(cudaGraphExecMemsetNodeSetParams(b->exec, b->count_node, &b->count_params));
  note_launch();
  RST_CUDA(cudaGraphLaunch(b->exec, st));
  return RESET_OK;
}

reset_status reset_batch_destroy(reset_batch* b) {
  if (!b) return RESET_OK;
  cudaError_t e = cudaDeviceSynchronize();
  batch_destroy(b);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize", __FILE__, __LINE__);
  return RESET_OK;
}

}  // extern "C"
