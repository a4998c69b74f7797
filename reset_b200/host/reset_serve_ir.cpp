// reset_serve_ir <folder> [--streams=N] [--max-batch=N] [--rate=QPS] [--warmup=N]
//                [--alpha=F] [--bucket=N]
// Serves the queries of a reference information-retrieval folder
// (information-retrieval/ir.cu:213-267 input files: inverted_index_offsets.bin,
// inverted_index.bin, inverted_index_num.bin, query.bin, query_offsets.bin,
// query_num.bin) through the served form: the table stays resident, the
// queries arrive all at once (default) or as a Poisson stream at --rate,
// batches run continuously.  --warmup=N first serves the first N queries
// once, untimed (buffers and memory pools reach their working size).  Prints
// the reference's total line, then throughput and latency percentiles.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "reset.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "Usage: %s <input_folder> [--streams=N] [--max-batch=N] [--rate=QPS]\n",
            argv[0]);
    return 1;
  }
  int streams = 4, max_batch = 1024, bucket = 5, warmup = 0;
  double rate = 0.0;
  float alpha = 0.2f;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--streams=", 0) == 0) streams = std::stoi(a.substr(10));
    else if (a.rfind("--max-batch=", 0) == 0) max_batch = std::stoi(a.substr(12));
    else if (a.rfind("--rate=", 0) == 0) rate = std::stod(a.substr(7));
    else if (a.rfind("--warmup=", 0) == 0) warmup = std::stoi(a.substr(9));
    else if (a.rfind("--alpha=", 0) == 0) alpha = std::stof(a.substr(8));
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
    reset_params p;
    reset_params_default(&p);
    p.alpha = alpha;
    p.bucket = bucket;
    reset_table* t = nullptr;
    reset::check(reset_table_build(idx.get_device_offsets(), idx.get_device_elements(), nt,
                                   idx.get_num_elements(), &p, 1, nullptr, &t, nullptr));
    long long total = 0;
    std::vector<double> lat;
    double wall = 0;
    {
      reset::Server srv(streams, max_batch);
      int ix = srv.add_index(t, idx.get_device_offsets(), idx.get_device_elements());
      {  // untimed warm-up over the first queries
        const int nw = std::min(std::max(warmup, 0), nq);
        std::vector<uint64_t> wt(nw);
        for (int i = 0; i < nw; i++)
          wt[i] = srv.submit(RESET_REQ_IR, ix, q.data() + qoff[i], qoff[i + 1] - qoff[i]);
        for (int i = 0; i < nw; i++) reset::check(srv.wait(wt[i]).status);
      }
      // a waiter thread takes each result (and releases it) as soon as it
      // is done, as a serving client would, while this thread submits
      std::vector<uint64_t> tickets(nq);
      std::atomic<int> submitted{0};
      int bad = 0;
      std::thread waiter([&] {
        for (int i = 0; i < nq; i++) {
          while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
          reset::ServedResult r = srv.wait(tickets[i]);
          if (r.status != RESET_OK) ++bad;
          total += r.count;
          lat.push_back(r.latency_us / 1e3);
        }
      });
      std::mt19937_64 rng(12345);
      std::exponential_distribution<double> gap(rate > 0 ? rate : 1.0);
      const int64_t t0 = reset_now_ns();
      double at = 0;
      for (int i = 0; i < nq; i++) {
        int64_t arrival = 0;
        if (rate > 0) {
          at += gap(rng);
          arrival = t0 + (int64_t)(at * 1e9);
          while (reset_now_ns() < arrival) std::this_thread::yield();
        }
        tickets[i] = srv.submit(RESET_REQ_IR, ix, q.data() + qoff[i], qoff[i + 1] - qoff[i],
                                nullptr, 0, 7, 10, arrival);
        submitted.store(i + 1, std::memory_order_release);
      }
      waiter.join();
      if (bad) throw std::runtime_error("served requests failed");
      wall = (reset_now_ns() - t0) / 1e9;
      reset_server_counters c = srv.stats();
      printf("batches: %lld, mean batch: %.1f\n", (long long)c.batches, c.mean_batch);
    }
    reset_table_free(t);
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double f) { return lat.empty() ? 0.0 : lat[std::min(lat.size() - 1, (size_t)(f * lat.size()))]; };
    printf("query_num: %d\n", nq);
    printf("Total result count: %lld\n", total);
    printf("served: %.1f queries/s, latency p50 %.3f ms, p99 %.3f ms\n", nq / wall, pct(0.5),
           pct(0.99));
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
