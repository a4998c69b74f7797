// Reference-side driver for the raw two-set intersection (test
// infrastructure).  Links the reference's own set_size/intersection.cu,
// compiled unchanged for sm_100a, and runs make_hashtable_kernel and
// intersection_kernel (intersection.cu:128-181) on seeded arrays a.bin and
// b.bin instead of the unseeded random arrays of intersection.cu:57-70.
// The table length and the two A orders follow intersection.cu:198-232.
// Sizes are capped: the reference keeps one table replica per warp
// (6912 warps, intersection.cu:16-19,236-241).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "harness_io.h"

using std::vector;

__global__ void make_hashtable_kernel(int* data, int data_size, int* hashtable,
                                      int bucket_num, int hash_length);
__global__ void intersection_kernel(int* a, int a_size, int* hashtable,
                                    int hash_length, int* result_count,
                                    int bucket_num);

int main(int argc, char** argv) {
  if (argc < 3) hio::die("usage: ref_pair <in_dir> <out_dir>");
  std::string in = argv[1], out = argv[2];
  vector<int> a = hio::read_arr<int>(in + "/a.bin");
  vector<int> b = hio::read_arr<int>(in + "/b.bin");
  if (a.size() > b.size()) std::swap(a, b);
  const int kWarps = 216 * 1024 / 32;
  int na = (int)a.size(), nb = (int)b.size();
  if (na < 1 || nb < 16 || nb > 4096) hio::die("sizes must be |A| >= 1, |B| in [16, 4096]");
  for (int x : a) if (x < 0) hio::die("negative key");
  for (int x : b) if (x < 0) hio::die("negative key");
  int max_length = (int)(nb / 0.2 / 5);
  int lg = log2f(max_length);
  max_length = powf(2, lg) == max_length ? max_length : powf(2, lg + 1);
  // The probe loop ends only at an empty slot: require a power-of-two
  // length with room to spare before any kernel runs.
  if (max_length < 8 || (max_length & (max_length - 1)) || max_length * 5 <= nb) hio::die("unexpected table length");
  int bucket_num = max_length * kWarps;
  size_t tbytes = sizeof(int) * (size_t)bucket_num * 5;
  int *d_t, *d_b, *d_a, *d_cnt;
  hio::check(cudaMalloc(&d_t, tbytes), "malloc");
  hio::check(cudaMemset(d_t, -1, tbytes), "memset");
  hio::check(cudaMalloc(&d_b, sizeof(int) * nb), "malloc");
  hio::check(cudaMemcpy(d_b, b.data(), sizeof(int) * nb, cudaMemcpyHostToDevice), "h2d");
  make_hashtable_kernel<<<216, 1024>>>(d_b, nb, d_t, bucket_num, max_length);
  hio::check(cudaDeviceSynchronize(), "make_hashtable_kernel");
  hio::check(cudaMalloc(&d_a, sizeof(int) * (size_t)na * kWarps), "malloc");
  hio::check(cudaMalloc(&d_cnt, sizeof(int)), "malloc");
  long long counts[2];
  for (int opt = 0; opt < 2; opt++) {
    vector<int> s = a;
    if (opt == 0)
      std::sort(s.begin(), s.end());
    else
      std::sort(s.begin(), s.end(), [&](int x, int y) { return x % max_length < y % max_length; });
    vector<int> rep((size_t)na * kWarps);
    for (int w = 0; w < kWarps; w++) std::copy(s.begin(), s.end(), rep.begin() + (size_t)w * na);
    hio::check(cudaMemcpy(d_a, rep.data(), sizeof(int) * rep.size(), cudaMemcpyHostToDevice), "h2d");
    hio::check(cudaMemset(d_cnt, 0, sizeof(int)), "memset");
    intersection_kernel<<<216, 1024>>>(d_a, na, d_t, max_length, d_cnt, bucket_num);
    hio::check(cudaDeviceSynchronize(), "intersection_kernel");
    int c = 0;
    hio::check(cudaMemcpy(&c, d_cnt, sizeof(int), cudaMemcpyDeviceToHost), "d2h");
    counts[opt] = c;
  }
  long long meta[3] = {max_length, counts[0], counts[1]};
  hio::write_arr(out + "/meta.i64.bin", meta, 3);
  printf("ref_pair na=%d nb=%d count=%lld/%lld\n", na, nb, counts[0], counts[1]);
  return 0;
}
