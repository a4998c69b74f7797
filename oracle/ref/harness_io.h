// .bin I/O for the reference harness drivers (test infrastructure only).
// Arrays use the RESET on-disk framing: a u64 element count followed by the
// payload (preprocess/util.py:12-15); int32 scalars are a bare 4-byte value
// (preprocess/util.py:18-20).  64-bit arrays use the same framing with
// 8-byte elements and a ".i64.bin" suffix.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace hio {

inline void die(const std::string& m) {
  fprintf(stderr, "harness: %s\n", m.c_str());
  exit(2);
}

template <typename T>
std::vector<T> read_arr(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) die("cannot open " + path);
  uint64_t n = 0;
  if (fread(&n, 8, 1, f) != 1) die("short read " + path);
  std::vector<T> v(n);
  if (n && fread(v.data(), sizeof(T), n, f) != n) die("short read " + path);
  fclose(f);
  return v;
}

inline int32_t read_scalar(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) die("cannot open " + path);
  int32_t x = 0;
  if (fread(&x, 4, 1, f) != 1) die("short read " + path);
  fclose(f);
  return x;
}

template <typename T>
void write_arr(const std::string& path, const T* p, uint64_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) die("cannot write " + path);
  fwrite(&n, 8, 1, f);
  if (n) fwrite(p, sizeof(T), n, f);
  fclose(f);
}

template <typename T>
void write_vec(const std::string& path, const std::vector<T>& v) {
  write_arr(path, v.data(), v.size());
}

inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "harness: %s: %s\n", what, cudaGetErrorString(e));
    exit(3);
  }
}

inline void parse_params(int argc, char** argv, int first, float* alpha,
                         int* bucket, bool* no_dump = nullptr) {
  for (int i = first; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--alpha=", 0) == 0)
      *alpha = std::stof(a.substr(8));
    else if (a.rfind("--bucket=", 0) == 0)
      *bucket = std::stoi(a.substr(9));
    else if (a == "--no-dump" && no_dump)  // results on stdout only, no table files
      *no_dump = true;
    else
      die("unknown argument " + a);
  }
}

}  // namespace hio
