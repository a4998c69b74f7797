// reset_tc <folder> [--alpha=F] [--bucket=N]
// Drop-in for the reference's triangle-count executable (triangle-count/
// TC.cu:192-347) and baseline/tc/main.cu: same input files
// (csr_offsets_tri.bin, csr_cols_tri.bin, num_nodes_tri.bin,
// num_edges_tri.bin), same flags, and the result lines those programs print
// (TC.cu:310,331; baseline/tc/main.cu:131-144), with times measured by CUDA
// events instead of clock().
#include <cstdio>
#include <string>

#include "reset.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "Usage: %s <input_folder> [--alpha=F] [--bucket=N]\n", argv[0]);
    return 1;
  }
  float alpha = 0.2f;
  int bucket = 5;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--alpha=", 0) == 0) alpha = std::stof(a.substr(8));
    else if (a.rfind("--bucket=", 0) == 0) bucket = std::stoi(a.substr(9));
    else {
      fprintf(stderr, "Unknown argument: %s\n", a.c_str());
      return 1;
    }
  }
  try {
    std::string d = argv[1];
    reset::CSRGraph g(d + "/csr_offsets_tri.bin", d + "/csr_cols_tri.bin");
    int n = reset::read_int_binary(d + "/num_nodes_tri.bin");
    int m = reset::read_int_binary(d + "/num_edges_tri.bin");
    if (n != g.get_num_nodes() || m != g.get_num_elements()) {
      fprintf(stderr, "inconsistent counts in %s\n", d.c_str());
      return 1;
    }
    printf("load_factor:%.2f , bucket_size:%d\n", alpha, bucket);
    printf("Graph loaded: %d nodes, %d edges\n", n, m);
    reset::TCBaseline tc;
    tc.build(g, alpha, bucket);
    printf("Max length: %d\n", tc.get_max_length());
    printf("Total buckets: %lld\n", tc.get_bucket_num());
    auto nr = tc.run_normal(g);
    printf("Normal hash - Triangles: %llu, Time: %.6f sec\n", nr.first, nr.second / 1e3);
    auto hr = tc.run_hierarchical(g);
    printf("Hierarchical hash - Triangles: %llu, Time: %.6f sec\n", hr.first, hr.second / 1e3);
    printf("[Native] 内核执行时间: %.6f 秒\n", nr.second / 1e3);
    printf("三角形数量: %llu\n", nr.first);
    printf("[RESET] 内核执行时间: %.6f 秒\n", hr.second / 1e3);
    printf("三角形数量: %llu\n", hr.first);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
