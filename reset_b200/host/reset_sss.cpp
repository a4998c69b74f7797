// reset_sss <folder> [--alpha=F] [--bucket=N] [--thr=F] [--exact=NUM/DEN]
// Drop-in for the reference's set-similarity-search executable
// (set-similarity-search/sss.cu:191-337): same input files (vertexs.bin,
// csr_cols.bin, csr_offsets.bin, num_edges.bin, num_nodes.bin), pairs are
// the CSR entries, threshold 0.25 by default (sss.cu:260), same result lines
// (sss.cu:290-336).  --exact=7/10 switches to the integer rule 10*I >= 7*U.
#include <cstdio>
#include <string>

#include "reset.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "Usage: %s <input_folder>\n", argv[0]);
    return 1;
  }
  float alpha = 0.2f, thr = 0.25f;
  int bucket = 5, num = 0, den = 0;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--alpha=", 0) == 0) alpha = std::stof(a.substr(8));
    else if (a.rfind("--bucket=", 0) == 0) bucket = std::stoi(a.substr(9));
    else if (a.rfind("--thr=", 0) == 0) thr = std::stof(a.substr(6));
    else if (a.rfind("--exact=", 0) == 0) {
      std::string r = a.substr(8);
      size_t s = r.find('/');
      if (s == std::string::npos) { fprintf(stderr, "--exact=NUM/DEN\n"); return 1; }
      num = std::stoi(r.substr(0, s));
      den = std::stoi(r.substr(s + 1));
    } else {
      fprintf(stderr, "Unknown argument: %s\n", a.c_str());
      return 1;
    }
  }
  try {
    std::string d = argv[1];
    reset::CSRGraph g(d + "/csr_offsets.bin", d + "/csr_cols.bin");
    std::vector<int> vert = reset::read_i32_vec(d + "/vertexs.bin");
    int n = reset::read_int_binary(d + "/num_nodes.bin");
    int m = reset::read_int_binary(d + "/num_edges.bin");
    if (n != g.get_num_nodes() || m != g.get_num_elements() || (int)vert.size() != m) {
      fprintf(stderr, "inconsistent counts in %s\n", d.c_str());
      return 1;
    }
    printf("num_nodes: %d, num_edges: %d\n", n, m);
    reset::SSSBaseline s;
    s.build(g, alpha, bucket);
    s.load_vertex_pairs(vert, g.get_host_elements());
    if (den > 0) {
      auto r = s.run_exact(num, den);
      printf("[Target] Exact Kernel execution time: %f seconds\n", r.second / 1e3);
      printf("num of pairs whose similarity is greater than threshold: %d\n", r.first);
      return 0;
    }
    auto r1 = s.run_normal(g, 0, 0, 0, bucket, thr);
    printf("[Target] Normal Kernel execution time: %f seconds\n", r1.second / 1e3);
    auto r2 = s.run_hierarchical(g, 0, 0, 0, bucket, thr);
    printf("[Target] Hierarchical Kernel execution time: %f seconds\n", r2.second / 1e3);
    if (r1.first != r2.first) {
      printf("Wrong Answer!\n");
      printf("sum1: %d, sum2: %d\n", r1.first, r2.first);
      return 2;
    }
    printf("num of pairs whose similarity is greater than threshold: %d\n", r1.first);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
