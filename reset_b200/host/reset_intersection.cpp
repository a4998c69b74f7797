// reset_intersection <|A|> <|B|> [--seed=S] | reset_intersection --files <a.bin> <b.bin>
// Drop-in for the reference's set_size/intersection driver
// (set_size/intersection.cu:183-303): two random int arrays in [0, INT_MAX]
// (seeded here; the reference seeds from random_device), the smaller probed
// into the larger one's table, |A ∩ B| counted with A's multiplicity, and
// the same result line (intersection.cu:298).
#include <climits>
#include <cstdio>
#include <random>
#include <string>

#include "reset.hpp"

int main(int argc, char** argv) {
  std::vector<int> a, b;
  try {
    if (argc >= 4 && std::string(argv[1]) == "--files") {
      a = reset::read_i32_vec(argv[2]);
      b = reset::read_i32_vec(argv[3]);
    } else if (argc >= 3) {
      long na = std::atol(argv[1]), nb = std::atol(argv[2]);
      unsigned long long seed = 0x5EEDull;
      for (int i = 3; i < argc; i++) {
        std::string s = argv[i];
        if (s.rfind("--seed=", 0) == 0) seed = std::stoull(s.substr(7));
      }
      std::mt19937 gen((unsigned)seed);
      std::uniform_int_distribution<int> dist(0, INT_MAX);
      a.resize(na);
      b.resize(nb);
      for (auto& x : a) x = dist(gen);
      for (auto& x : b) x = dist(gen);
    } else {
      fprintf(stderr, "Usage: %s <set A size> <set B size> [--seed=S]\n", argv[0]);
      return 1;
    }
    if (a.size() > b.size()) std::swap(a, b);
    reset::DeviceBuffer<int> da, db;
    da.upload(a);
    db.upload(b);
    reset::DeviceBuffer<int64_t> cnt(1);
    reset_params p;
    reset_params_default(&p);
    reset::detail::EventTimer tm;
    reset::check(reset_intersect_count(da.p, (int64_t)a.size(), db.p, (int64_t)b.size(), &p,
                                       cnt.p, nullptr));
    float ms = tm.stop();
    long long c = (long long)cnt.download()[0];
    printf("Intersection Time: %f ms\n", ms);
    printf("Intersection Result Count: %lld\n", c);
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
