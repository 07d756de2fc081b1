// CPU oracle: reference-faithful flooding min-sum decoder (test infrastructure
// and the timed CPU baseline).
//
// Restates LdpcDecoder from crates/gf2-coding/src/ldpc/core.rs:
//   new()                      653-697  neighbour lists + per-node message vectors
//   decode_batch()             729-756  one fresh decoder per frame, frames in parallel
//   check_node_update_minsum() 790-814  O(dc^2) gather with find_check_position
//   variable_node_update()     819-838  belief = llr + sum c2v (ascending check), v2c = belief - c2v
//   find_check_position()      841-846  linear search
//   check_to_var_message()     849-856  linear search
//   hard_decode()              859-865  Llr::hard_decision (llr.rs:73-75): value < 0
//   decode_iterative()         889-938
// and the executed min-sum kernel: Llr::boxplus_minsum_n (llr.rs:246-269), which
// copies its inputs into a fresh Vec and calls minsum_avx2_f32
// (crates/gf2-kernels-simd/src/llr.rs:117-180) on AVX2 hosts.
#include <cmath>
#include <cstring>
#include <thread>

#include "oracle_internal.h"

int or_threads(int threads) {
  if (threads > 0) return threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Rust f32::min: IEEE minNum (a NaN operand yields the other operand).
static inline float rust_min(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}

static inline uint32_t bits_of(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return u;
}

static inline float abs_bits(float x) {  // _mm256_andnot_ps(sign_mask, x)
  uint32_t u = bits_of(x) & 0x7fffffffu;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// minsum_avx2_f32: 8-lane chunks (MINPS keeps the second operand when the
// comparison fails; sign bits XOR-accumulated), horizontal reduction, then the
// scalar remainder with `val < 0.0`.
static float minsum_avx2_emulated(const float* in, size_t n) {
  if (n == 0) return 0.0f;
  float lane_min[8];
  uint32_t lane_sign[8];
  for (int l = 0; l < 8; l++) {
    lane_min[l] = INFINITY;
    lane_sign[l] = 0;
  }
  size_t chunks = n / 8;
  for (size_t c = 0; c < chunks; c++)
    for (int l = 0; l < 8; l++) {
      float v = in[c * 8 + l];
      float a = abs_bits(v);
      lane_min[l] = (lane_min[l] < a) ? lane_min[l] : a;
      lane_sign[l] ^= bits_of(v) & 0x80000000u;
    }
  float min_abs = INFINITY;
  for (int l = 0; l < 8; l++) min_abs = rust_min(min_abs, lane_min[l]);
  float sign = 1.0f;
  for (int l = 0; l < 8; l++)
    if (lane_sign[l] & 0x80000000u) sign = -sign;
  for (size_t i = chunks * 8; i < n; i++) {
    float v = in[i];
    min_abs = rust_min(min_abs, std::fabs(v));
    if (v < 0.0f) sign = -sign;
  }
  return sign * min_abs;
}

namespace {

struct FaithfulDecoder {
  const or_code* code;
  int64_t n, m, k;
  std::vector<float> beliefs;
  std::vector<std::vector<float>> c2v, v2c;
  std::vector<std::vector<int64_t>> check_nb, var_nb;
  std::vector<float> temp;
  int64_t last_iterations = 0;

  explicit FaithfulDecoder(const or_code* c) : code(c), n(c->n), m(c->m), k(c->k) {
    check_nb.resize(m);
    size_t max_dc = 0;
    for (int64_t r = 0; r < m; r++) {
      check_nb[r].assign(c->row_idx.begin() + c->row_ptr[r], c->row_idx.begin() + c->row_ptr[r + 1]);
      max_dc = std::max(max_dc, check_nb[r].size());
    }
    var_nb.resize(n);
    for (int64_t v = 0; v < n; v++)
      var_nb[v].assign(c->col_idx.begin() + c->col_ptr[v], c->col_idx.begin() + c->col_ptr[v + 1]);
    c2v.resize(m);
    for (int64_t r = 0; r < m; r++) c2v[r].assign(check_nb[r].size(), 0.0f);
    v2c.resize(n);
    for (int64_t v = 0; v < n; v++) v2c[v].assign(var_nb[v].size(), 0.0f);
    beliefs.assign(n, 0.0f);
    temp.reserve(max_dc);
  }

  size_t find_check_position(int64_t var, int64_t check) const {
    const auto& nb = var_nb[var];
    for (size_t i = 0; i < nb.size(); i++)
      if (nb[i] == check) return i;
    return (size_t)-1;
  }

  float check_to_var_message(int64_t var, size_t pos) const {
    int64_t check = var_nb[var][pos];
    const auto& nb = check_nb[check];
    size_t p = 0;
    while (nb[p] != var) p++;
    return c2v[check][p];
  }

  void check_node_update_minsum() {
    for (int64_t check = 0; check < m; check++) {
      const auto& nb = check_nb[check];
      for (size_t pos = 0; pos < nb.size(); pos++) {
        temp.clear();
        for (size_t other = 0; other < nb.size(); other++) {
          if (other == pos) continue;
          int64_t ov = nb[other];
          temp.push_back(v2c[ov][find_check_position(ov, check)]);
        }
        float msg;
        if (temp.empty()) {
          msg = 0.0f;
        } else {
          std::vector<float> f32_vals(temp.begin(), temp.end());  // llr.rs:261
          msg = minsum_avx2_emulated(f32_vals.data(), f32_vals.size());
        }
        c2v[check][pos] = msg;
      }
    }
  }

  void variable_node_update(const float* llr) {
    for (int64_t var = 0; var < n; var++) {
      const auto& nb = var_nb[var];
      float belief = llr[var];
      for (size_t pos = 0; pos < nb.size(); pos++) belief = belief + check_to_var_message(var, pos);
      beliefs[var] = belief;
      for (size_t pos = 0; pos < nb.size(); pos++) {
        float incoming = check_to_var_message(var, pos);
        v2c[var][pos] = belief - incoming;
      }
    }
  }

  bool is_valid(std::vector<uint8_t>& hard) const {
    for (int64_t v = 0; v < n; v++) hard[v] = beliefs[v] < 0.0f ? 1 : 0;
    for (int64_t r = 0; r < m; r++) {
      uint8_t acc = 0;
      for (int64_t e = code->row_ptr[r]; e < code->row_ptr[r + 1]; e++) acc ^= hard[code->row_idx[e]];
      if (acc) return false;
    }
    return true;
  }

  void decode_iterative(const float* llr, int max_iter, uint8_t* msg, int32_t* iters, uint8_t* conv,
                        uint8_t* synd_ok, float* beliefs_out) {
    for (auto& row : c2v)
      for (auto& x : row) x = 0.0f;
    for (int64_t v = 0; v < n; v++)
      for (auto& x : v2c[v]) x = llr[v];
    std::vector<uint8_t> hard(n);
    int iterations = 0;
    bool converged = false;
    for (int it = 0; it < max_iter; it++) {
      iterations = it + 1;
      check_node_update_minsum();
      variable_node_update(llr);
      if (is_valid(hard)) {
        converged = true;
        break;
      }
    }
    last_iterations = iterations;
    bool passed = is_valid(hard);
    if (msg)
      for (int64_t i = 0; i < k; i++) msg[i] = hard[i];
    if (iters) *iters = iterations;
    if (conv) *conv = converged;
    if (synd_ok) *synd_ok = passed;
    if (beliefs_out) std::memcpy(beliefs_out, beliefs.data(), sizeof(float) * n);
  }
};

}  // namespace

extern "C" int or_decode_minsum_faithful(const or_code* c, const float* llr, int64_t frames,
                                         int max_iter, int threads, uint8_t* msg, int32_t* iters,
                                         uint8_t* conv, uint8_t* synd_ok, float* beliefs) {
  if (!c || frames < 0 || max_iter < 0) {
    or_set_error("invalid arguments");
    return -1;
  }
  or_parallel_frames(frames, threads, [&](int64_t f) {
    // decode_batch: Self::new(code.clone()) per frame (core.rs:740).
    FaithfulDecoder dec(c);
    dec.decode_iterative(llr + f * c->n, max_iter, msg ? msg + f * c->k : nullptr,
                         iters ? iters + f : nullptr, conv ? conv + f : nullptr,
                         synd_ok ? synd_ok + f : nullptr, beliefs ? beliefs + f * c->n : nullptr);
  });
  return 0;
}
