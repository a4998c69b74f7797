// Reference-side driver for set-similarity search (test infrastructure).
// Links the reference's own set-similarity-search/sss.cu and hashtable.cu,
// compiled unchanged for sm_100a, on a folder in the reference's SSS input
// format (csr_offsets.bin, csr_cols.bin, vertexs.bin, num_nodes.bin,
// num_edges.bin; sss.cu:234-244).  Pairs are the CSR entries
// (vertexs[e], csr_cols[e]) as in sss.cu:104-105.  Runs
// set_similarity_search_kernel (sss.cu:93-154) with the launch shape of
// sss.cu:257-260 in both hash modes for a threshold given by --thr=.
#include "harness_tables.h"

__global__ void set_similarity_search_kernel(
    int num_edges, int* vertexs, int* csr_cols, int* csr_offsets,
    int* hash_length, int* hash_table, long long* hash_table_offsets,
    int* results, int* G_index, int CHUNK_SIZE, bool opt, int max_length,
    int bucket_num, float threshold, int bucket_size);

int main(int argc, char** argv) {
  if (argc < 3) hio::die("usage: ref_sss <in_dir> <out_dir> [--thr=F] [--alpha=F] [--bucket=N]");
  std::string in = argv[1], out = argv[2];
  float alpha = 0.2f, thr = 0.25f;
  int b = 5;
  int first = 3;
  if (argc > 3 && std::string(argv[3]).rfind("--thr=", 0) == 0) {
    thr = std::stof(std::string(argv[3]).substr(6));
    first = 4;
  }
  hio::parse_params(argc, argv, first, &alpha, &b);
  vector<int> off = hio::read_arr<int>(in + "/csr_offsets.bin");
  vector<int> cols = hio::read_arr<int>(in + "/csr_cols.bin");
  vector<int> vert = hio::read_arr<int>(in + "/vertexs.bin");
  int n = hio::read_scalar(in + "/num_nodes.bin");
  int m = hio::read_scalar(in + "/num_edges.bin");
  if ((long long)cols.size() != m || (long long)vert.size() != m) hio::die("num_edges mismatch");
  for (int i = 0; i < n; i++)
    for (int j = off[i]; j < off[i + 1]; j++)
      if (vert[j] != i) hio::die("vertexs.bin is not the CSR row expansion");
  RefTables t = ref_build_tables(off, cols, n, alpha, b, n);
  vector<int> cols_h = cols;
  gpu_sort_csr_cols(cols_h, off, n, t.max_len);
  int *d_vert, *d_cols_h, *d_g, *d_res;
  hio::check(cudaMalloc(&d_vert, sizeof(int) * m), "malloc");
  hio::check(cudaMalloc(&d_cols_h, sizeof(int) * m), "malloc");
  hio::check(cudaMalloc(&d_g, sizeof(int)), "malloc");
  hio::check(cudaMalloc(&d_res, sizeof(int) * m), "malloc");
  hio::check(cudaMemcpy(d_vert, vert.data(), sizeof(int) * m, cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_cols_h, cols_h.data(), sizeof(int) * m, cudaMemcpyHostToDevice), "h2d");
  const int grid = 512, block = 1024, chunk = 4;
  int g0 = grid * block / 32 * chunk;
  vector<int> res[2];
  long long sums[2];
  for (int opt = 0; opt < 2; opt++) {
    hio::check(cudaMemset(d_res, 0, sizeof(int) * m), "memset");
    hio::check(cudaMemcpy(d_g, &g0, sizeof(int), cudaMemcpyHostToDevice), "h2d");
    set_similarity_search_kernel<<<grid, block>>>(m, d_vert, opt ? d_cols_h : t.d_elems, t.d_off, t.d_len, opt ? t.d_th : t.d_tn, t.d_off64, d_res, d_g, chunk, opt != 0, t.max_len, (int)t.bucket_num, thr, b);
    hio::check(cudaDeviceSynchronize(), "set_similarity_search_kernel");
    res[opt].resize(m);
    hio::check(cudaMemcpy(res[opt].data(), d_res, sizeof(int) * m, cudaMemcpyDeviceToHost), "d2h");
    sums[opt] = 0;
    for (int x : res[opt]) sums[opt] += x;
  }
  long long meta[4] = {t.max_len, t.bucket_num, sums[0], sums[1]};
  hio::write_arr(out + "/meta.i64.bin", meta, 4);
  ref_dump_tables(t, out);
  hio::write_vec(out + "/results_normal.bin", res[0]);
  hio::write_vec(out + "/results_hier.bin", res[1]);
  hio::write_vec(out + "/cols_hier_sorted.bin", cols_h);
  printf("ref_sss n=%d m=%d thr=%g normal=%lld hier=%lld\n", n, m, thr, sums[0], sums[1]);
  return 0;
}
