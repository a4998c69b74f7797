// reset_smog <graph_folder> <pattern> [process_num] [load_factor] [bucket_size]
//            [block_size] [block_number] [chunk_size]
// Drop-in for SMOG's subgraph-matching executable (SMOG/SMOG_hie/main_hie.cpp,
// SubgraphMatching in subgraph_match_hie.cu:529-794): the same positional
// arguments, the same graph folder files, and its result lines.  The graph
// files are raw int32 arrays without a header, as SMOG reads them
// (common_hie.cu:61-129): begin.bin (row offsets), adjacent.bin (columns),
// vertex.bin (the row of every edge), md.bin (the largest row) for the
// oriented graph of Q0, Q3, Q5, Q7; generic_*.bin of the symmetric graph for
// the other patterns.  The pattern is a name of SMOG's table (Q0..Q8); its
// arrays come from the library instead of a rebuild per pattern.
// process_num, block_size, block_number and chunk_size are accepted and
// ignored: one call counts every start edge on one GPU.  The time is the
// count call's, measured by CUDA events instead of clock().
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "reset.hpp"

namespace {

std::vector<int> read_raw_i32(const std::string& path) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) throw reset::Error(RESET_ERR_ARG, "cannot open file: " + path);
  const std::streamsize bytes = in.tellg();
  if (bytes % (std::streamsize)sizeof(int))
    throw reset::Error(RESET_ERR_ARG, "not an int32 array: " + path);
  std::vector<int> v((size_t)(bytes / (std::streamsize)sizeof(int)));
  in.seekg(0);
  if (!v.empty()) in.read(reinterpret_cast<char*>(v.data()), bytes);
  if (!in) throw reset::Error(RESET_ERR_ARG, "cannot read file: " + path);
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr,
            "Usage: %s <graph_folder> <pattern Q0..Q8> [process_num] [load_factor] "
            "[bucket_size] [block_size] [block_number] [chunk_size]\n",
            argv[0]);
    return 1;
  }
  const std::string folder = argv[1], pattern = argv[2];
  float alpha = 0.2f;
  int bucket = 5;
  try {
    if (argc > 4) alpha = std::stof(argv[4]);
    if (argc > 5) bucket = std::stoi(argv[5]);
  } catch (const std::exception&) {
    fprintf(stderr, "bad load_factor or bucket_size\n");
    return 1;
  }
  reset_pattern p;
  int32_t oriented = 0;
  if (reset_pattern_named(pattern.c_str(), &p, &oriented) != RESET_OK) {
    fprintf(stderr, "unknown pattern %s (SMOG's table has Q0..Q8)\n", pattern.c_str());
    return 1;
  }
  try {
    const std::string pre = folder + (oriented ? "/" : "/generic_");
    std::vector<int> off = read_raw_i32(pre + "begin.bin");
    std::vector<int> cols = read_raw_i32(pre + "adjacent.bin");
    std::vector<int> vtx = read_raw_i32(pre + "vertex.bin");
    std::vector<int> md = read_raw_i32(pre + "md.bin");
    if (off.empty() || (size_t)off.back() != cols.size() || vtx.size() != cols.size() ||
        md.empty())
      throw reset::Error(RESET_ERR_ARG, "inconsistent graph files in " + folder);
    const int n = (int)off.size() - 1;
    for (int u = 0; u < n; u++)
      for (int e = off[u]; e < off[u + 1]; e++)
        if (vtx[e] != u) throw reset::Error(RESET_ERR_ARG, "vertex.bin disagrees with begin.bin");
    printf("graph vertex number is : %d\n", n);
    printf("graph edge number is : %zu\n", cols.size());
    printf("graph bucket size is : %d\n", bucket);
    printf("max degree is : %d\n", md[0]);
    reset::CSRGraph g(std::move(off), std::move(cols));
    reset_params prm;
    reset_params_default(&prm);
    prm.alpha = alpha;
    prm.bucket = bucket;
    reset_table* t = nullptr;
    reset::check(reset_table_build(g.get_device_offsets(), g.get_device_elements(), n,
                                   g.get_num_elements(), &prm, 1, nullptr, &t, nullptr));
    printf("finish make hash table\n");
    reset::DeviceBuffer<uint64_t> d_count(1);
    uint64_t count = 0;
    float ms = 0;
    try {
      printf("start kernel\n");
      reset::detail::EventTimer timer;
      reset::check(reset_pattern_count(t, g.get_device_offsets(), g.get_device_elements(),
                                       g.get_num_elements(), &p, d_count.p, nullptr));
      ms = timer.stop();
      reset::check(reset_table_check(t, nullptr));
      printf("finish kernel\n");
      count = d_count.download()[0];
    } catch (...) {
      reset_table_free(t);
      throw;
    }
    reset_table_free(t);
    printf("Hierarchical time: %g ms\n", ms);
    printf("%s count is %llu\n", pattern.c_str(), (unsigned long long)count);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
