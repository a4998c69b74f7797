// Reference-side driver for conjunctive information retrieval (test
// infrastructure).  Links the reference's own information-retrieval/ir.cu
// and hashtable.cu, compiled unchanged for sm_100a, on a folder in the
// reference's IR input format (inverted_index_offsets.bin,
// inverted_index.bin, inverted_index_num.bin, query.bin, query_offsets.bin,
// query_num.bin; ir.cu:254-267).  Result offsets follow ir.cu:324-330 and
// ir_kernel (ir.cu:94-176) runs with the launch shape of ir.cu:305-311 in
// both hash modes.  Empty queries are refused: the reference reads
// query[query_start] for them (ir.cu:119).
#include "harness_tables.h"

__global__ void ir_kernel(int* inverted_index, int* inverted_index_offsets,
                          int* query, int* query_offsets, int query_num,
                          int* result, long long* result_offsets,
                          int* result_count, int* G_index, int CHUNK_SIZE,
                          int max_length, bool opt, int* hashtable,
                          long long* hashtable_offset, int bucket_num,
                          int bucket_size);

int main(int argc, char** argv) {
  if (argc < 3) hio::die("usage: ref_ir <in_dir> <out_dir> [--alpha=F] [--bucket=N]");
  std::string in = argv[1], out = argv[2];
  float alpha = 0.2f;
  int b = 5;
  hio::parse_params(argc, argv, 3, &alpha, &b);
  vector<int> toff = hio::read_arr<int>(in + "/inverted_index_offsets.bin");
  vector<int> docs = hio::read_arr<int>(in + "/inverted_index.bin");
  int nt = hio::read_scalar(in + "/inverted_index_num.bin");
  vector<int> query = hio::read_arr<int>(in + "/query.bin");
  vector<int> qoff = hio::read_arr<int>(in + "/query_offsets.bin");
  int nq = hio::read_scalar(in + "/query_num.bin");
  if ((long long)qoff.size() != (long long)nq + 1 || qoff[0] != 0 || qoff[nq] != (int)query.size()) hio::die("inconsistent queries");
  for (int q = 0; q < nq; q++)
    if (qoff[q + 1] <= qoff[q]) hio::die("empty query");
  for (int t : query)
    if (t < 0 || t >= nt) hio::die("term id out of range");
  RefTables t = ref_build_tables(toff, docs, nt, alpha, b, 1 << 30);
  vector<long long> roff(nq + 1, 0);
  for (int q = 0; q < nq; q++) {
    int t0 = query[qoff[q]];
    roff[q + 1] = roff[q] + toff[t0 + 1] - toff[t0];
  }
  vector<int> docs_h = docs;
  gpu_sort_csr_cols(docs_h, toff, nt, t.max_len);
  int *d_docs_h, *d_q, *d_qoff, *d_res, *d_cnt, *d_g;
  long long* d_roff;
  long long rtot = roff[nq] > 0 ? roff[nq] : 1;
  hio::check(cudaMalloc(&d_docs_h, sizeof(int) * (docs.size() + 1)), "malloc");
  hio::check(cudaMalloc(&d_q, sizeof(int) * query.size()), "malloc");
  hio::check(cudaMalloc(&d_qoff, sizeof(int) * (nq + 1)), "malloc");
  hio::check(cudaMalloc(&d_res, sizeof(int) * rtot), "malloc");
  hio::check(cudaMalloc(&d_cnt, sizeof(int) * nq), "malloc");
  hio::check(cudaMalloc(&d_g, sizeof(int)), "malloc");
  hio::check(cudaMalloc(&d_roff, sizeof(long long) * (nq + 1)), "malloc");
  hio::check(cudaMemcpy(d_docs_h, docs_h.data(), sizeof(int) * docs.size(), cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_q, query.data(), sizeof(int) * query.size(), cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_qoff, qoff.data(), sizeof(int) * (nq + 1), cudaMemcpyHostToDevice), "h2d");
  hio::check(cudaMemcpy(d_roff, roff.data(), sizeof(long long) * (nq + 1), cudaMemcpyHostToDevice), "h2d");
  const int grid = 512, block = 1024, chunk = 2;
  int g0 = grid * block / 32 * chunk;
  for (int opt = 0; opt < 2; opt++) {
    hio::check(cudaMemset(d_res, -1, sizeof(int) * rtot), "memset");
    hio::check(cudaMemset(d_cnt, 0, sizeof(int) * nq), "memset");
    hio::check(cudaMemcpy(d_g, &g0, sizeof(int), cudaMemcpyHostToDevice), "h2d");
    ir_kernel<<<grid, block>>>(opt ? d_docs_h : t.d_elems, t.d_off, d_q, d_qoff, nq, d_res, d_roff, d_cnt, d_g, chunk, t.max_len, opt != 0, opt ? t.d_th : t.d_tn, t.d_off64, (int)t.bucket_num, b);
    hio::check(cudaDeviceSynchronize(), "ir_kernel");
    vector<int> res(roff[nq]), cnt(nq);
    hio::check(cudaMemcpy(res.data(), d_res, sizeof(int) * roff[nq], cudaMemcpyDeviceToHost), "d2h");
    hio::check(cudaMemcpy(cnt.data(), d_cnt, sizeof(int) * nq, cudaMemcpyDeviceToHost), "d2h");
    hio::write_vec(out + (opt ? "/result_hier.bin" : "/result_normal.bin"), res);
    hio::write_vec(out + (opt ? "/count_hier.bin" : "/count_normal.bin"), cnt);
  }
  long long meta[2] = {t.max_len, t.bucket_num};
  hio::write_arr(out + "/meta.i64.bin", meta, 2);
  hio::write_vec(out + "/result_offsets.i64.bin", roff);
  ref_dump_tables(t, out);
  hio::write_vec(out + "/docs_hier_sorted.bin", docs_h);
  printf("ref_ir terms=%d postings=%zu queries=%d\n", nt, docs.size(), nq);
  return 0;
}
