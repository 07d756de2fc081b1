// Internal declarations of the CPU oracle (test infrastructure only).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "oracle.h"

struct or_code {
  int64_t n = 0, m = 0, k = 0;
  std::vector<int64_t> row_ptr, row_idx;   // CSR: columns ascending per row
  std::vector<int64_t> col_ptr, col_idx;   // CSC: rows ascending per column
  std::vector<int64_t> col_edge;           // CSC slot -> CSR edge id
  std::vector<int64_t> edge_key;           // per CSR edge: delta order key in a layer
  std::vector<int32_t> slot_order;         // per row: CSR offsets in the library's slot order
  int dvb_q = 0;                           // DVB-T2 step q (0 if not DVB-T2)
  int layers = 0;                          // row groups (QC / DVB-T2), 0 = none
  std::vector<int32_t> check_layer;        // layer of each check
};

void or_set_error(const std::string& s);
int or_threads(int threads);

template <class F>
void or_parallel_frames(int64_t frames, int threads, F&& fn);

#include <atomic>
#include <thread>

template <class F>
void or_parallel_frames(int64_t frames, int threads, F&& fn) {
  int t = or_threads(threads);
  if (t > frames) t = (int)(frames > 0 ? frames : 1);
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      int64_t f = next.fetch_add(1);
      if (f >= frames) break;
      fn(f);
    }
  };
  if (t <= 1) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  for (int i = 0; i < t; i++) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
}
