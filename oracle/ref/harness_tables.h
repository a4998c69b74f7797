// Shared glue of the reference harness drivers (test infrastructure): the
// steps of make_hash_table (triangle-count/hashtable.cu:103-183; the same in
// set-similarity-search/hashtable.cu:100-181 and
// information-retrieval/hashtable.cu:162-249) driven through the reference's
// own kernels, which every app directory defines with these signatures.
// The max-length accumulator is zeroed first (the reference leaves it
// uninitialised) and inputs that would overflow the reference's 32-bit slot
// index are refused before any kernel runs.
#pragma once
#include <cub/cub.cuh>
#include <vector>

#include "harness_io.h"

using std::vector;

__global__ void calculate_hash_length(int* hash_length, int num_nodes,
                                      int* csr_offsets, int* max_length,
                                      float load_factor, int bucket_size);
__global__ void build_hash_table_hierarchical(
    int* hash_table, int* hash_length, long long* hash_tables_offset,
    int num_edges, int bucket_num, int max_length, int* vertexs,
    int* csr_cols, int* conflict_count, int bucket_size);
__global__ void build_hash_table_normal(int* hash_table, int* hash_length,
                                        long long* hash_tables_offset,
                                        int num_edges, int bucket_num,
                                        int* word_id, int* doc_id,
                                        int* conflict_count, int bucket_size);
void gpu_sort_csr_cols(vector<int>& csr_cols, const vector<int>& csr_row,
                       int num_nodes, int max_length);

struct RefTables {
  int n = 0, m = 0, b = 0, max_len = 0;
  long long bucket_num = 0;
  int *d_off = nullptr, *d_len = nullptr, *d_elems = nullptr;
  int *d_tn = nullptr, *d_th = nullptr;
  long long* d_off64 = nullptr;
  vector<int> len;
  vector<long long> off64;
};

inline RefTables ref_build_tables(const vector<int>& off,
                                  const vector<int>& elems, int n, float alpha,
                                  int b, int id_bound) {
  RefTables t;
  t.n = n;
  t.m = (int)elems.size();
  t.b = b;
  if (!(alpha > 0.f && alpha <= 1.f) || b < 1) hio::die("alpha must be in (0,1], bucket >= 1");
  if (n < 1 || (long long)off.size() != (long long)n + 1 || off[0] != 0 || off[n] != t.m)
    hio::die("inconsistent CSR");
  for (int i = 0; i < n; i++)
    if (off[i + 1] < off[i]) hio::die("offsets not monotone");
  for (int x : elems)
    if (x < 0 || x >= id_bound) hio::die("element id out of range");
  int* d_max;
  hio::check(cudaMalloc(&t.d_off, sizeof(int) * (n + 1)), "malloc");
  hio::check(cudaMalloc(&t.d_len, sizeof(int) * n), "malloc");
  hio::check(cudaMalloc(&d_max, sizeof(int)), "malloc");
  hio::check(cudaMalloc(&t.d_off64, sizeof(long long) * (n + 1)), "malloc");
  hio::check(cudaMemcpy(t.d_off, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemset(d_max, 0, sizeof(int)), "memset");
  calculate_hash_length<<<256, 1024>>>(t.d_len, n, t.d_off, d_max, alpha, b);
  hio::check(cudaDeviceSynchronize(), "calculate_hash_length");
  hio::check(cudaMemcpy(&t.max_len, d_max, sizeof(int), cudaMemcpyDeviceToHost), "d2h");
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, t.d_len, t.d_off64, n);
  hio::check(cudaMalloc(&tmp, tmp_bytes), "malloc");
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, t.d_len, t.d_off64, n);
  t.len.resize(n);
  t.off64.resize(n + 1);
  hio::check(cudaMemcpy(t.len.data(), t.d_len, sizeof(int) * n, cudaMemcpyDeviceToHost), "d2h");
  hio::check(cudaMemcpy(t.off64.data(), t.d_off64, sizeof(long long) * n, cudaMemcpyDeviceToHost), "d2h");
  t.bucket_num = t.off64[n - 1] + t.len[n - 1];
  t.off64[n] = t.bucket_num;
  // the reference's kernels index slots as int `bucket + k * bucket_num`
  // (bucket < max_len, k < b; TC.cu:18, hashtable.cu:65): refuse inputs
  // where that overflows, before any kernel runs
  const long long max_index = (long long)(b - 1) * t.bucket_num + t.max_len - 1;
  printf("ref tables: bucket_num=%lld max_len=%d largest int slot index=%lld (limit %lld)\n",
         t.bucket_num, t.max_len, max_index, (1LL << 31) - 1);
  if (max_index >= (1LL << 31)) hio::die("bucket_num too large for the reference's 32-bit slot index");
  hio::check(cudaMemcpy(t.d_off64 + n, &t.bucket_num, sizeof(long long), cudaMemcpyHostToDevice), "h2d");
  size_t tbytes = sizeof(int) * (size_t)t.bucket_num * b;
  hio::check(cudaMalloc(&t.d_tn, tbytes), "malloc");
  hio::check(cudaMalloc(&t.d_th, tbytes), "malloc");
  hio::check(cudaMemset(t.d_tn, -1, tbytes), "memset");
  hio::check(cudaMemset(t.d_th, -1, tbytes), "memset");
  vector<int> owner(t.m);
  for (int i = 0; i < n; i++)
    for (int j = off[i]; j < off[i + 1]; j++) owner[j] = i;
  int *d_owner, *d_conf;
  hio::check(cudaMalloc(&t.d_elems, sizeof(int) * (t.m > 0 ? t.m : 1)), "malloc");
  hio::check(cudaMalloc(&d_owner, sizeof(int) * (t.m > 0 ? t.m : 1)), "malloc");
  hio::check(cudaMalloc(&d_conf, sizeof(int)), "malloc");
  hio::check(cudaMemcpy(t.d_elems, elems.data(), sizeof(int) * t.m, cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_owner, owner.data(), sizeof(int) * t.m, cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemset(d_conf, 0, sizeof(int)), "memset");
  build_hash_table_normal<<<1024, 1024>>>(t.d_tn, t.d_len, t.d_off64, t.m, (int)t.bucket_num, d_owner, t.d_elems, d_conf, b);
  hio::check(cudaDeviceSynchronize(), "build_hash_table_normal");
  build_hash_table_hierarchical<<<1024, 1024>>>(t.d_th, t.d_len, t.d_off64, t.m, (int)t.bucket_num, t.max_len, d_owner, t.d_elems, d_conf, b);
  hio::check(cudaDeviceSynchronize(), "build_hash_table_hierarchical");
  cudaFree(d_owner);
  cudaFree(d_conf);
  cudaFree(d_max);
  cudaFree(tmp);
  return t;
}

inline void ref_dump_tables(const RefTables& t, const std::string& out) {
  size_t cnt = (size_t)t.bucket_num * t.b;
  vector<int> tn(cnt), th(cnt);
  hio::check(cudaMemcpy(tn.data(), t.d_tn, sizeof(int) * cnt, cudaMemcpyDeviceToHost), "d2h");
  hio::check(cudaMemcpy(th.data(), t.d_th, sizeof(int) * cnt, cudaMemcpyDeviceToHost), "d2h");
  hio::write_vec(out + "/len.bin", t.len);
  hio::write_vec(out + "/off64.i64.bin", t.off64);
  hio::write_vec(out + "/table_normal.bin", tn);
  hio::write_vec(out + "/table_hier.bin", th);
}
