/*
 * reset.hpp -- C++ host side over the C ABI of libreset.so.
 *
 * Mirrors the reference's host classes so C++ callers keep their code shape:
 *   reset::CSRGraph / reset::InvertedIndex  <- baseline/common/graph_data.cuh:42-97
 *   reset::HashTableBuilder                 <- baseline/common/hash_table.cuh:12-95
 *   reset::TCBaseline                       <- baseline/tc/tc.cuh:15-59
 *   reset::SSSBaseline                      <- baseline/sss/sss.cuh:12-69
 *   reset::IRBaseline                       <- baseline/ir/ir.cuh:13-87
 * and wraps the batched and served forms (reset::Batch, reset::Server).
 * Same names, argument meaning and return values (pairs of result and
 * kernel milliseconds).  Launch-shape arguments of the reference (CHUNK_SIZE,
 * grid_size, block_size) are accepted and ignored: the library sizes its own
 * persistent grids.  Errors throw reset::Error (the reference exit()s or
 * throws std::runtime_error, baseline/common/utils.cu:9-18).
 * Header-only; link with -lreset -lcudart.
 */
#ifndef RESET_HPP
#define RESET_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "reset.h"

namespace reset {

struct Error : std::runtime_error {
  reset_status status;
  Error(reset_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(reset_status s) {
  if (s != RESET_OK)
    throw Error(s, std::string(reset_status_string(s)) + ": " + reset_last_error_string());
}

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Error(RESET_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Reference on-disk format (preprocess/util.py:12-20): a u64 element count
// followed by int32 payload; scalars are a bare int32.
inline std::vector<int> read_i32_vec(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error(RESET_ERR_ARG, "cannot open file: " + path);
  uint64_t n = 0;
  in.read(reinterpret_cast<char*>(&n), sizeof(n));
  std::vector<int> v(n);
  in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(int)));
  if (!in) throw Error(RESET_ERR_ARG, "truncated file: " + path);
  return v;
}

inline int read_int_binary(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error(RESET_ERR_ARG, "cannot open file: " + path);
  int v = 0;
  in.read(reinterpret_cast<char*>(&v), sizeof(v));
  if (!in) throw Error(RESET_ERR_ARG, "truncated file: " + path);
  return v;
}

template <class T>
struct DeviceBuffer {
  T* p = nullptr;
  size_t n = 0;
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t count) { alloc(count); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  ~DeviceBuffer() { cudaFree(p); }
  void alloc(size_t count) {
    cudaFree(p);
    p = nullptr;
    n = count;
    check_cuda(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), "cudaMalloc");
  }
  void upload(const std::vector<T>& h) {
    alloc(h.size());
    if (!h.empty())
      check_cuda(cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice), "H2D");
  }
  std::vector<T> download() const {
    std::vector<T> h(n);
    if (n) check_cuda(cudaMemcpy(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost), "D2H");
    return h;
  }
};

// A CSR held on host and device (graph_data.cuh:72-97).
class CSRGraph {
 public:
  CSRGraph(const std::string& offsets_path, const std::string& columns_path)
      : off_(read_i32_vec(offsets_path)), cols_(read_i32_vec(columns_path)) {
    if (off_.empty() || (size_t)off_.back() != cols_.size())
      throw Error(RESET_ERR_ARG, "inconsistent CSR files");
    d_off_.upload(off_);
    d_cols_.upload(cols_);
  }
  CSRGraph(std::vector<int> off, std::vector<int> cols) : off_(std::move(off)), cols_(std::move(cols)) {
    d_off_.upload(off_);
    d_cols_.upload(cols_);
  }
  int get_num_nodes() const { return (int)off_.size() - 1; }
  int get_num_elements() const { return (int)cols_.size(); }
  const std::vector<int>& get_host_offsets() const { return off_; }
  const std::vector<int>& get_host_elements() const { return cols_; }
  int* get_device_offsets() const { return d_off_.p; }
  int* get_device_elements() const { return d_cols_.p; }

 private:
  std::vector<int> off_, cols_;
  DeviceBuffer<int> d_off_, d_cols_;
};

// An inverted index: terms are rows, documents are columns (graph_data.cuh:42-68).
using InvertedIndex = CSRGraph;

// Builds the hierarchical and the normal table over one CSR
// (HashTableBuilder::build_hash_tables, baseline/common/hash_table.cu:187-310).
class HashTableBuilder {
 public:
  HashTableBuilder() = default;
  HashTableBuilder(const HashTableBuilder&) = delete;
  HashTableBuilder& operator=(const HashTableBuilder&) = delete;
  virtual ~HashTableBuilder() { free_hash_tables(); }

  void build_hash_tables(int num_nodes, const std::vector<int>& h_offsets,
                         const std::vector<int>& h_elements, float load_factor,
                         int bucket_size) {
    free_hash_tables();
    if ((int)h_offsets.size() != num_nodes + 1) throw Error(RESET_ERR_ARG, "offsets size");
    d_off_.upload(h_offsets);
    d_elems_.upload(h_elements);
    d_hash_order_.alloc(h_elements.size());
    reset_params p;
    reset_params_default(&p);
    p.alpha = load_factor;
    p.bucket = bucket_size;
    check(reset_table_build(d_off_.p, d_elems_.p, num_nodes, (int64_t)h_elements.size(), &p,
                            1, d_hash_order_.p, &hier_, nullptr));
    check(reset_table_build(d_off_.p, d_elems_.p, num_nodes, (int64_t)h_elements.size(), &p,
                            0, nullptr, &norm_, nullptr));
    check(reset_table_info(hier_, &vh_));
    check(reset_table_info(norm_, &vn_));
  }

  void free_hash_tables() {
    if (hier_) reset_table_free(hier_);
    if (norm_) reset_table_free(norm_);
    hier_ = norm_ = nullptr;
  }

  int* get_d_hash_hierarchical() const { return vh_.d_table; }
  int* get_d_hash_normal() const { return vn_.d_table; }
  int* get_d_hash_length() const { return vh_.d_len; }
  long long* get_d_hash_tables_offset() const { return reinterpret_cast<long long*>(vh_.d_off); }
  int get_max_length() const { return vh_.max_len; }
  long long get_bucket_num() const { return vh_.bucket_num; }

  const reset_table* hierarchical_table() const { return hier_; }
  const reset_table* normal_table() const { return norm_; }
  // Rows read back in hierarchical bucket order (built in the same pass as
  // the table; what reorder_csr_by_hash_layout produces in the reference).
  int* get_d_hash_ordered_elements() const { return d_hash_order_.p; }
  int* get_d_offsets() const { return d_off_.p; }
  int* get_d_elements() const { return d_elems_.p; }

 protected:
  reset_table* hier_ = nullptr;
  reset_table* norm_ = nullptr;
  reset_table_view vh_{}, vn_{};
  DeviceBuffer<int> d_off_, d_elems_, d_hash_order_;
};

namespace detail {
struct EventTimer {
  cudaEvent_t a, b;
  EventTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
  }
  float stop() {
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
  }
};
}  // namespace detail

// Triangle counting over an oriented CSR (baseline/tc/tc.cuh:15-59).
class TCBaseline : public HashTableBuilder {
 public:
  void build(const CSRGraph& g, float load_factor = 0.2f, int bucket_size = 5) {
    build_hash_tables(g.get_num_nodes(), g.get_host_offsets(), g.get_host_elements(),
                      load_factor, bucket_size);
  }
  std::pair<unsigned long long, float> run_hierarchical(CSRGraph& g, int = 0, int = 0,
                                                        int = 0, int = 0, bool sorted = true) {
    const int* cols = sorted ? get_d_hash_ordered_elements() : get_d_elements();
    return run(hier_, g, cols);
  }
  std::pair<unsigned long long, float> run_normal(CSRGraph& g, int = 0, int = 0, int = 0,
                                                  int = 0, bool = false) {
    return run(norm_, g, get_d_elements());
  }

 private:
  std::pair<unsigned long long, float> run(reset_table* t, CSRGraph& g, const int* cols) {
    DeviceBuffer<uint64_t> cnt(1);
    detail::EventTimer tm;
    check(reset_tc_count(t, get_d_offsets(), cols, g.get_num_elements(), cnt.p, nullptr));
    float ms = tm.stop();
    check(reset_table_check(t, nullptr));
    return {(unsigned long long)cnt.download()[0], ms};
  }
};

// Set-similarity search over explicit pairs (baseline/sss/sss.cuh:12-69).
// The reference's pairs are the CSR entries (vertexs[e], csr_cols[e]).
class SSSBaseline : public HashTableBuilder {
 public:
  void build(const CSRGraph& g, float load_factor = 0.2f, int bucket_size = 5) {
    build_hash_tables(g.get_num_nodes(), g.get_host_offsets(), g.get_host_elements(),
                      load_factor, bucket_size);
  }
  void load_vertex_pairs(const std::vector<int>& a, const std::vector<int>& b) {
    if (a.size() != b.size()) throw Error(RESET_ERR_ARG, "pair arrays differ in length");
    d_a_.upload(a);
    d_b_.upload(b);
    d_flags_.alloc(a.size());
    np_ = (int64_t)a.size();
  }
  // Float rule of sss.cu:139-141: returns (number of similar pairs, ms).
  std::pair<int, float> run_hierarchical(CSRGraph&, int, int, int, int, float threshold,
                                         bool = true) {
    return run(hier_, threshold, true);
  }
  std::pair<int, float> run_normal(CSRGraph&, int, int, int, int, float threshold,
                                   bool = false) {
    return run(norm_, threshold, false);
  }
  // Exact integer rule den*I >= num*U.
  std::pair<int, float> run_exact(int num, int den) {
    detail::EventTimer tm;
    check(reset_sss(hier_, get_d_offsets(), get_d_elements(), d_a_.p, d_b_.p, np_, num, den,
                    d_flags_.p, nullptr, nullptr));
    float ms = tm.stop();
    return {count_flags(), ms};
  }
  std::vector<uint8_t> flags() const { return d_flags_.download(); }

 private:
  std::pair<int, float> run(reset_table* t, float thr, bool) {
    detail::EventTimer tm;
    check(reset_sss_float(t, get_d_offsets(), get_d_elements(), d_a_.p, d_b_.p, np_, thr,
                          d_flags_.p, nullptr, nullptr));
    float ms = tm.stop();
    return {count_flags(), ms};
  }
  int count_flags() const {
    int s = 0;
    for (uint8_t f : d_flags_.download()) s += f;
    return s;
  }
  DeviceBuffer<int> d_a_, d_b_;
  DeviceBuffer<uint8_t> d_flags_;
  int64_t np_ = 0;
};

// Conjunctive retrieval (baseline/ir/ir.cuh:13-87).  Result slot q is sized
// for df(first term), as information-retrieval/ir.cu:324-330 does.
class IRBaseline : public HashTableBuilder {
 public:
  void build(const InvertedIndex& idx, float load_factor = 0.2f, int bucket_size = 5) {
    build_hash_tables(idx.get_num_nodes(), idx.get_host_offsets(), idx.get_host_elements(),
                      load_factor, bucket_size);
    toff_ = idx.get_host_offsets();
  }
  void load_queries(const std::vector<int>& query, const std::vector<int>& query_offsets) {
    q_ = query;
    qoff_ = query_offsets;
    nq_ = (int)qoff_.size() - 1;
    std::vector<int64_t> roff(nq_ + 1, 0);
    for (int q = 0; q < nq_; q++) {
      int64_t df = 0;
      if (qoff_[q + 1] > qoff_[q]) {
        int t0 = q_[qoff_[q]];
        df = toff_[t0 + 1] - toff_[t0];
      }
      roff[q + 1] = roff[q] + df;
    }
    roff_ = roff;
    d_q_.upload(q_);
    d_qoff_.upload(qoff_);
    d_roff_.upload(roff_);
    d_res_.alloc((size_t)roff_.back());
    d_cnt_.alloc(nq_);
  }
  std::pair<int, float> run_hierarchical(int = 0, int = 0, int = 0, int = 0, bool = true) {
    return run(hier_, get_d_hash_ordered_elements());
  }
  std::pair<int, float> run_normal(int = 0, int = 0, int = 0, int = 0, bool = false) {
    return run(norm_, get_d_elements());
  }
  std::vector<int> get_results() const { return d_cnt_.download(); }
  // Survivors of query q, in first-term order.
  std::vector<int> result_list(int q) const {
    std::vector<int> all = d_res_.download(), cnt = d_cnt_.download();
    return std::vector<int>(all.begin() + roff_[q], all.begin() + roff_[q] + cnt[q]);
  }

 private:
  std::pair<int, float> run(reset_table* t, const int* docs) {
    detail::EventTimer tm;
    check(reset_ir(t, get_d_offsets(), docs, d_q_.p, d_qoff_.p, nq_, d_roff_.p, d_res_.p,
                   d_cnt_.p, nullptr));
    float ms = tm.stop();
    check(reset_table_check(t, nullptr));
    long long total = 0;
    for (int c : d_cnt_.download()) total += c;
    return {(int)total, ms};
  }
  std::vector<int> toff_, q_, qoff_;
  std::vector<int64_t> roff_;
  int nq_ = 0;
  DeviceBuffer<int> d_q_, d_qoff_, d_res_, d_cnt_;
  DeviceBuffer<int64_t> d_roff_;
};

// ---- forms with no counterpart in the reference ---------------------------

// Batched pair decisions over one table (reset_batch_*): fill pair_a()/pair_b()
// on the device, run(np), read flags()/inter().
class Batch {
 public:
  Batch(const reset_table* t, const int32_t* d_elems, int64_t capacity, int num = 7,
        int den = 10, bool decisions_only = false, cudaStream_t stream = nullptr) {
    check(reset_batch_create_ex(t, d_elems, capacity, num, den,
                                decisions_only ? RESET_BATCH_DECISIONS_ONLY : 0, &b_,
                                stream));
    check(reset_batch_buffers(b_, &pa_, &pb_, &flags_, &inter_));
  }
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;
  ~Batch() { reset_batch_destroy(b_); }
  int32_t* pair_a() const { return pa_; }
  int32_t* pair_b() const { return pb_; }
  uint8_t* flags() const { return flags_; }
  int32_t* inter() const { return inter_; }
  void run(int64_t np, cudaStream_t stream = nullptr) { check(reset_batch_run(b_, np, stream)); }

 private:
  reset_batch* b_ = nullptr;
  int32_t *pa_ = nullptr, *pb_ = nullptr, *inter_ = nullptr;
  uint8_t* flags_ = nullptr;
};

// A result of the served form, copied out of the server.
struct ServedResult {
  reset_status status = RESET_OK;
  int64_t count = 0;
  std::vector<int32_t> docs;
  std::vector<int64_t> values;
  std::vector<uint8_t> flags;
  double queue_us = 0, service_us = 0, latency_us = 0;
  int32_t batch_size = 0;
};

// The served form (reset_server_*): submit() returns at once, wait() blocks.
class Server {
 public:
  explicit Server(int streams = 4, int max_batch_requests = 1024, int64_t mem_budget = 0) {
    reset_server_config cfg;
    reset_server_config_default(&cfg);
    cfg.streams = streams;
    cfg.max_batch_requests = max_batch_requests;
    cfg.mem_budget_bytes = mem_budget;
    check(reset_server_create(&cfg, &s_));
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  ~Server() { reset_server_destroy(s_); }
  int add_index(const reset_table* t, const int32_t* d_off, const int32_t* d_elems) {
    int32_t ix = 0;
    check(reset_server_add_index(s_, t, d_off, d_elems, &ix));
    return ix;
  }
  uint64_t submit(int kind, int index, const int32_t* args, int64_t nargs,
                  const int32_t* args2 = nullptr, int64_t nargs2 = 0, int num = 7,
                  int den = 10, int64_t arrival_ns = 0) {
    reset_request q = {};
    q.kind = kind;
    q.index = index;
    q.args = args;
    q.nargs = nargs;
    q.args2 = args2;
    q.nargs2 = nargs2;
    q.num = num;
    q.den = den;
    q.arrival_ns = arrival_ns;
    uint64_t t = 0;
    check(reset_server_submit(s_, &q, &t));
    return t;
  }
  ServedResult wait(uint64_t ticket, int timeout_ms = -1) {
    reset_result r;
    check(reset_server_wait(s_, ticket, timeout_ms, &r));
    ServedResult out;
    out.status = r.status;
    out.count = r.count;
    if (r.ndocs) out.docs.assign(r.docs, r.docs + r.ndocs);
    if (r.nvalues) out.values.assign(r.values, r.values + r.nvalues);
    if (r.nvalues && r.flags) out.flags.assign(r.flags, r.flags + r.nvalues);
    out.queue_us = r.queue_us;
    out.service_us = r.service_us;
    out.latency_us = r.latency_us;
    out.batch_size = r.batch_size;
    check(reset_server_release(s_, ticket));
    return out;
  }
  reset_server_counters stats() {
    reset_server_counters c;
    check(reset_server_stats(s_, &c));
    return c;
  }

 private:
  reset_server* s_ = nullptr;
};

}  // namespace reset

#endif  // RESET_HPP
