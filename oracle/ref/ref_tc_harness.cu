// Reference-side driver for the triangle-count path (test infrastructure).
// Links the reference's own triangle-count/TC.cu and hashtable.cu, compiled
// unchanged for sm_100a, and runs on a folder in the reference's TC input
// format (csr_offsets_tri.bin, csr_cols_tri.bin, num_nodes_tri.bin,
// num_edges_tri.bin; TC.cu:236-245):
//   table build through harness_tables.h,
//   gpu_sort_csr_cols      (triangle-count/TC.cu:107-126),
//   dynamic_triangle_count (triangle-count/TC.cu:128-190) in both hash modes
//   with the launch shape of TC.cu:268-275.
#include "harness_tables.h"

__global__ void dynamic_triangle_count(
    int num_edges, int* vertexs, int* csr_cols, int* csr_offsets,
    int* hash_length, int* hash_table, long long* hash_table_offsets,
    unsigned long long* results, int* G_index, int CHUNK_SIZE, bool opt,
    int max_length, int bucket_num, int bucket_size);

int main(int argc, char** argv) {
  if (argc < 3) hio::die("usage: ref_tc <in_dir> <out_dir> [--alpha=F] [--bucket=N] [--no-dump]");
  std::string in = argv[1], out = argv[2];
  float alpha = 0.2f;
  int b = 5;
  bool no_dump = false;
  hio::parse_params(argc, argv, 3, &alpha, &b, &no_dump);
  vector<int> off = hio::read_arr<int>(in + "/csr_offsets_tri.bin");
  vector<int> cols = hio::read_arr<int>(in + "/csr_cols_tri.bin");
  int n = hio::read_scalar(in + "/num_nodes_tri.bin");
  int m = hio::read_scalar(in + "/num_edges_tri.bin");
  if ((long long)cols.size() != m) hio::die("num_edges mismatch");
  RefTables t = ref_build_tables(off, cols, n, alpha, b, n);
  vector<int> vert(m);
  for (int i = 0; i < n; i++)
    for (int j = off[i]; j < off[i + 1]; j++) vert[j] = i;
  vector<int> cols_h = cols;
  gpu_sort_csr_cols(cols_h, off, n, t.max_len);
  int *d_vert, *d_cols_h, *d_g;
  unsigned long long* d_cnt;
  hio::check(cudaMalloc(&d_vert, sizeof(int) * m), "malloc");
  hio::check(cudaMalloc(&d_cols_h, sizeof(int) * m), "malloc");
  hio::check(cudaMalloc(&d_g, sizeof(int)), "malloc");
  hio::check(cudaMalloc(&d_cnt, sizeof(unsigned long long)), "malloc");
  hio::check(cudaMemcpy(d_vert, vert.data(), sizeof(int) * m, cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_cols_h, cols_h.data(), sizeof(int) * m, cudaMemcpyHostToDevice), "h2d");
  const int grid = 1024, block = 512, chunk = 4;
  int g0 = grid * block / 32 * chunk;
  unsigned long long counts[2];
  float ms[2];
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int opt = 0; opt < 2; opt++) {
    hio::check(cudaMemset(d_cnt, 0, sizeof(unsigned long long)), "memset");
    hio::check(cudaMemcpy(d_g, &g0, sizeof(int), cudaMemcpyHostToDevice), "h2d");
    cudaEventRecord(e0);
    dynamic_triangle_count<<<grid, block>>>(m, d_vert, opt ? d_cols_h : t.d_elems, t.d_off, t.d_len, opt ? t.d_th : t.d_tn, t.d_off64, d_cnt, d_g, chunk, opt != 0, t.max_len, (int)t.bucket_num, b);
    cudaEventRecord(e1);
    hio::check(cudaDeviceSynchronize(), "dynamic_triangle_count");
    cudaEventElapsedTime(&ms[opt], e0, e1);
    hio::check(cudaMemcpy(&counts[opt], d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost), "d2h");
  }
  long long meta[4] = {t.max_len, t.bucket_num, (long long)counts[0], (long long)counts[1]};
  if (!no_dump) {
    hio::write_arr(out + "/meta.i64.bin", meta, 4);
    ref_dump_tables(t, out);
    hio::write_vec(out + "/cols_hier_sorted.bin", cols_h);
  }
  printf("ref_tc n=%d m=%d max_len=%d bucket_num=%lld normal=%llu (%.3f ms) hier=%llu (%.3f ms)\n", n, m, t.max_len, t.bucket_num, counts[0], ms[0], counts[1], ms[1]);
  return 0;
}
