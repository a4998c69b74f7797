// reset_ir <folder> [--alpha=F] [--bucket=N]
// Drop-in for the reference's information-retrieval executable
// (information-retrieval/ir.cu:213-432): same input files
// (inverted_index_offsets.bin, inverted_index.bin, inverted_index_num.bin,
// query.bin, query_offsets.bin, query_num.bin), same result lines
// (ir.cu:378-430).  Empty queries are answered with 0 results.
#include <cstdio>
#include <string>

#include "reset.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "Usage: %s <input_folder>\n", argv[0]);
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
    reset::InvertedIndex idx(d + "/inverted_index_offsets.bin", d + "/inverted_index.bin");
    int nt = reset::read_int_binary(d + "/inverted_index_num.bin");
    std::vector<int> q = reset::read_i32_vec(d + "/query.bin");
    std::vector<int> qoff = reset::read_i32_vec(d + "/query_offsets.bin");
    int nq = reset::read_int_binary(d + "/query_num.bin");
    if (nt != idx.get_num_nodes() || (int)qoff.size() != nq + 1) {
      fprintf(stderr, "inconsistent counts in %s\n", d.c_str());
      return 1;
    }
    for (int t : q)
      if (t < 0 || t >= nt) {
        fprintf(stderr, "query term out of range\n");
        return 1;
      }
    printf("query_num: %d\n", nq);
    reset::IRBaseline ir;
    ir.build(idx, alpha, bucket);
    ir.load_queries(q, qoff);
    auto r1 = ir.run_normal();
    printf("Noramal Kernel execution time: %f seconds\n", r1.second / 1e3);
    auto r2 = ir.run_hierarchical();
    printf("Hierarchical Kernel execution time: %f seconds\n", r2.second / 1e3);
    if (r1.first != r2.first) {
      printf("Result mismatch between normal and hierarchical!\n");
      return 2;
    }
    printf("Total result count: %d\n", r1.first);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
