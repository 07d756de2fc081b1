// gf2cuda.hpp -- C++ mirror of the gf2-coding LDPC API over the gf2cuda C ABI.
//
// Names, argument meaning and error behaviour follow erankavija/gf2
// (crates/gf2-coding/src/): LdpcCode (ldpc/core.rs:59-262), QuasiCyclicLdpc
// (ldpc/core.rs:450-606), LdpcDecoder with IterativeSoftDecoder::decode_iterative
// and decode_batch (ldpc/core.rs:632-960, traits.rs:314-347), LdpcEncoder
// (ldpc/core.rs:984-1133), DecoderResult (traits.rs:115-177), Llr (llr.rs:40-119)
// and the BitVec layout of gf2-core (u64 words, LSB first).  Where the reference
// panics (length asserts, invalid shifts) this header throws
// std::invalid_argument; library failures throw gf2::Error.
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gf2cuda.h"

namespace gf2 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error("gf2cuda error " + std::to_string(c) + ": " + m), code(c) {}
};

inline void check(int rc) {
  if (rc == GF2C_OK) return;
  if (rc == GF2C_ERR_INVALID_ARG || rc == GF2C_ERR_RANK) throw std::invalid_argument(gf2c_last_error());
  throw Error(rc, gf2c_last_error());
}

enum class CodeRate { Rate1_2 = 0, Rate3_5 = 1, Rate2_3 = 2, Rate3_4 = 3, Rate4_5 = 4, Rate5_6 = 5 };

// BitVec: u64 words, bit i in word i/64 at position i%64, unused tail bits zero.
class BitVec {
 public:
  BitVec() = default;
  static BitVec zeros(size_t len) {
    BitVec b;
    b.len_ = len;
    b.w_.assign((len + 63) / 64, 0);
    return b;
  }
  size_t len() const { return len_; }
  bool get(size_t i) const { return (w_.at(i / 64) >> (i % 64)) & 1u; }
  void set(size_t i, bool v) {
    if (i >= len_) throw std::out_of_range("bit index");
    if (v) w_[i / 64] |= 1ull << (i % 64);
    else w_[i / 64] &= ~(1ull << (i % 64));
  }
  void push_bit(bool v) {
    if (len_ % 64 == 0) w_.push_back(0);
    ++len_;
    set(len_ - 1, v);
  }
  size_t count_ones() const {
    size_t c = 0;
    for (uint64_t x : w_) c += (size_t)__builtin_popcountll(x);
    return c;
  }
  const std::vector<uint64_t>& words() const { return w_; }
  std::vector<uint64_t>& words() { return w_; }
  bool operator==(const BitVec& o) const { return len_ == o.len_ && w_ == o.w_; }

 private:
  std::vector<uint64_t> w_;
  size_t len_ = 0;
};

class Llr {
 public:
  Llr() = default;
  explicit Llr(float v) : v_(v) {}
  float value() const { return v_; }
  bool hard_decision() const { return v_ < 0.0f; }
  float magnitude() const { return v_ < 0 ? -v_ : v_; }
  Llr saturate(float mx) const { return Llr(v_ > mx ? mx : (v_ < -mx ? -mx : v_)); }

 private:
  float v_ = 0.0f;
};

struct DecoderResult {
  BitVec decoded_bits;
  size_t iterations = 0;
  bool converged = false;
  bool syndrome_check_passed = false;
};

class QuasiCyclicLdpc {
 public:
  QuasiCyclicLdpc(std::vector<std::vector<int32_t>> base, size_t z) : base_(std::move(base)), z_(z) {
    if (base_.empty()) throw std::invalid_argument("Base matrix must have at least one row");
    if (z_ == 0) throw std::invalid_argument("Expansion factor must be positive");
    for (auto& r : base_)
      if (r.size() != base_[0].size()) throw std::invalid_argument("All rows in base matrix must have the same length");
  }
  size_t base_rows() const { return base_.size(); }
  size_t base_cols() const { return base_[0].size(); }
  size_t expansion_factor() const { return z_; }
  const std::vector<std::vector<int32_t>>& base() const { return base_; }

 private:
  std::vector<std::vector<int32_t>> base_;
  size_t z_;
};

class LdpcCode {
 public:
  static LdpcCode dvb_t2_short(CodeRate r) { return make(gf2c_code_create_dvbt2, GF2C_DVBT2_SHORT, (int)r); }
  static LdpcCode dvb_t2_normal(CodeRate r) { return make(gf2c_code_create_dvbt2, GF2C_DVBT2_NORMAL, (int)r); }
  static LdpcCode from_edges(size_t m, size_t n, const std::vector<std::pair<size_t, size_t>>& edges) {
    std::vector<int64_t> p;
    p.reserve(edges.size() * 2);
    for (auto& e : edges) {
      p.push_back((int64_t)e.first);
      p.push_back((int64_t)e.second);
    }
    gf2c_code* c = nullptr;
    check(gf2c_code_create_edges((int64_t)m, (int64_t)n, p.data(), (int64_t)edges.size(), &c));
    return LdpcCode(c);
  }
  static LdpcCode from_quasi_cyclic(const QuasiCyclicLdpc& qc) {
    std::vector<int32_t> flat;
    for (auto& r : qc.base()) flat.insert(flat.end(), r.begin(), r.end());
    gf2c_code* c = nullptr;
    check(gf2c_code_create_qc(flat.data(), (int32_t)qc.base_rows(), (int32_t)qc.base_cols(),
                              (int32_t)qc.expansion_factor(), &c));
    return LdpcCode(c);
  }
  size_t n() const { return (size_t)n_; }
  size_t m() const { return (size_t)m_; }
  size_t k() const { return (size_t)k_; }
  double rate() const { return (double)k_ / (double)n_; }
  gf2c_code* handle() const { return h_.get(); }

  BitVec syndrome(const BitVec& cw) const {
    if (cw.len() != n()) throw std::invalid_argument("Codeword length must equal n");
    BitVec s = BitVec::zeros(m());
    int32_t w = 0;
    check(gf2c_syndrome_batch(handle(), cw.words().data(), 1, s.words().data(), &w, GF2C_MEM_HOST, nullptr));
    return s;
  }
  bool is_valid_codeword(const BitVec& cw) const { return syndrome(cw).count_ones() == 0; }

 private:
  explicit LdpcCode(gf2c_code* c) : h_(c, gf2c_code_destroy) {
    check(gf2c_code_dims(c, &n_, &m_, &k_, nullptr, nullptr));
  }
  template <class F>
  static LdpcCode make(F f, int a, int b) {
    gf2c_code* c = nullptr;
    check(f(a, b, &c));
    return LdpcCode(c);
  }
  std::shared_ptr<gf2c_code> h_;
  int64_t n_ = 0, m_ = 0, k_ = 0;
};

class LdpcDecoder {
 public:
  explicit LdpcDecoder(LdpcCode code, const gf2c_decoder_opts* opts = nullptr) : code_(std::move(code)) {
    gf2c_decoder* d = nullptr;
    check(gf2c_decoder_create(code_.handle(), opts, &d));
    h_.reset(d, gf2c_decoder_destroy);
  }
  size_t k() const { return code_.k(); }
  size_t n() const { return code_.n(); }
  size_t last_iteration_count() const { return last_; }
  void reset() { last_ = 0; }

  // SoftDecoder::decode_soft (core.rs:877-885): hard decisions of the input.
  BitVec decode_soft(const std::vector<Llr>& llrs) const {
    if (llrs.size() != n()) throw std::invalid_argument("LLR length must equal n");
    BitVec b;
    for (auto& l : llrs) b.push_bit(l.hard_decision());
    return b;
  }

  // IterativeSoftDecoder::decode_iterative (core.rs:889-938)
  DecoderResult decode_iterative(const std::vector<Llr>& llrs, size_t max_iterations) {
    auto r = decode_many({llrs}, max_iterations);
    last_ = r[0].iterations;
    return r[0];
  }

  // LdpcDecoder::decode_batch (core.rs:729-756)
  static std::vector<DecoderResult> decode_batch(const LdpcCode& code, const std::vector<std::vector<Llr>>& blocks,
                                                 size_t max_iterations) {
    if (blocks.empty()) return {};
    LdpcDecoder dec(code);
    return dec.decode_many(blocks, max_iterations);
  }

  std::vector<DecoderResult> decode_many(const std::vector<std::vector<Llr>>& blocks, size_t max_iterations) {
    const size_t F = blocks.size(), N = n(), K = k(), W = (K + 63) / 64;
    std::vector<float> llr(F * N);
    for (size_t f = 0; f < F; f++) {
      if (blocks[f].size() != N) throw std::invalid_argument("LLR length must equal n");
      for (size_t i = 0; i < N; i++) llr[f * N + i] = blocks[f][i].value();
    }
    std::vector<uint64_t> msg(F * W);
    std::vector<int32_t> it(F);
    std::vector<uint8_t> cv(F), so(F);
    check(gf2c_decode_batch(h_.get(), llr.data(), (int64_t)F, (int32_t)max_iterations, msg.data(), it.data(),
                            cv.data(), so.data(), nullptr, GF2C_MEM_HOST, nullptr));
    std::vector<DecoderResult> out(F);
    for (size_t f = 0; f < F; f++) {
      BitVec b = BitVec::zeros(K);
      for (size_t w = 0; w < W; w++) b.words()[w] = msg[f * W + w];
      out[f] = DecoderResult{std::move(b), (size_t)it[f], cv[f] != 0, so[f] != 0};
    }
    return out;
  }

 private:
  LdpcCode code_;
  std::shared_ptr<gf2c_decoder> h_;
  size_t last_ = 0;
};

class LdpcEncoder {
 public:
  explicit LdpcEncoder(LdpcCode code) : code_(std::move(code)) {}
  size_t k() const { return code_.k(); }
  size_t n() const { return code_.n(); }
  BitVec encode(const BitVec& msg) const { return encode_batch({msg})[0]; }
  std::vector<BitVec> encode_batch(const std::vector<BitVec>& msgs) const {
    if (msgs.empty()) return {};
    const size_t F = msgs.size(), WK = (k() + 63) / 64, WN = (n() + 63) / 64;
    std::vector<uint64_t> in(F * WK), out(F * WN);
    for (size_t f = 0; f < F; f++) {
      if (msgs[f].len() != k()) throw std::invalid_argument("Message length must be k = " + std::to_string(k()));
      for (size_t w = 0; w < WK; w++) in[f * WK + w] = msgs[f].words()[w];
    }
    check(gf2c_encode_batch(code_.handle(), in.data(), (int64_t)F, out.data(), GF2C_MEM_HOST, nullptr));
    std::vector<BitVec> r(F);
    for (size_t f = 0; f < F; f++) {
      r[f] = BitVec::zeros(n());
      for (size_t w = 0; w < WN; w++) r[f].words()[w] = out[f * WN + w];
    }
    return r;
  }

 private:
  LdpcCode code_;
};

}  // namespace gf2
