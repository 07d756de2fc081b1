// gf2cuda.hpp -- C++ mirror of the gf2-coding LDPC API over the gf2cuda C ABI.
//
// Names, argument meaning and error behaviour follow erankavija/gf2
// (crates/gf2-coding/src/): LdpcCode (ldpc/core.rs:59-262), QuasiCyclicLdpc
// (ldpc/core.rs:450-606), LdpcDecoder with IterativeSoftDecoder::decode_iterative
// and decode_batch (ldpc/core.rs:632-960, traits.rs:314-347), LdpcEncoder
// (ldpc/core.rs:984-1133), DecoderResult (traits.rs:115-177), Llr (llr.rs:40-119)
// and the BitVec layout of gf2-core (u64 words, LSB first); the DVB-T2 outer
// BCH code (bch/core.rs, bch/dvb_t2/); the gf2 file formats (gf2-core/src/io)
// and the LDPC encoder cache (ldpc/encoding/cache.rs).  Where the reference
// panics (length asserts, invalid shifts) this header throws
// std::invalid_argument; library failures throw gf2::Error.
#pragma once
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
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
  // An LdpcCode whose H is an SpBitMatrix / SpBitMatrixDual file (gf2-core/src/io/sparse.rs).
  static LdpcCode from_file(const std::string& path) {
    gf2c_code* c = nullptr;
    check(gf2c_code_create_file(path.c_str(), &c));
    return LdpcCode(c);
  }
  // H as SpBitMatrixDual (dual) or SpBitMatrix; binary (format 0) or text (1).
  void save(const std::string& path, bool dual = true, int format = 0) const {
    check(gf2c_io_write_code(path.c_str(), handle(), dual ? 4 : 3, format));
  }

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
    const size_t F = blocks.size(), K = k(), W = (K + 63) / 64;
    std::vector<float> llr = flatten(blocks);
    std::vector<uint64_t> msg(F * W);
    std::vector<int32_t> it(F);
    std::vector<uint8_t> cv(F), so(F);
    check(gf2c_decode_batch(h_.get(), llr.data(), (int64_t)F, (int32_t)max_iterations, msg.data(), it.data(),
                            cv.data(), so.data(), nullptr, GF2C_MEM_HOST, nullptr));
    return results(F, msg, it, cv, so);
  }

  // This decoder on every frame, then `fallback` (a layered decoder of the
  // same code) on the frames whose syndrome still fails; no counterpart in the
  // reference.  *redecoded (optional): frames the fallback decoded again.
  std::vector<DecoderResult> decode_many_with_fallback(LdpcDecoder& fallback,
                                                       const std::vector<std::vector<Llr>>& blocks,
                                                       size_t max_iterations, size_t fallback_iterations,
                                                       size_t* redecoded = nullptr) {
    const size_t F = blocks.size(), K = k(), W = (K + 63) / 64;
    if (F == 0) return {};
    std::vector<float> llr = flatten(blocks);
    std::vector<uint64_t> msg(F * W);
    std::vector<int32_t> it(F);
    std::vector<uint8_t> cv(F), so(F);
    int64_t count = 0;
    check(gf2c_decode_batch_fallback(h_.get(), fallback.h_.get(), llr.data(), (int64_t)F, (int32_t)max_iterations,
                                     (int32_t)fallback_iterations, msg.data(), it.data(), cv.data(), so.data(), &count,
                                     GF2C_MEM_HOST, nullptr));
    if (redecoded) *redecoded = (size_t)count;
    return results(F, msg, it, cv, so);
  }

 private:
  std::vector<float> flatten(const std::vector<std::vector<Llr>>& blocks) const {
    const size_t F = blocks.size(), N = n();
    std::vector<float> llr(F * N);
    for (size_t f = 0; f < F; f++) {
      if (blocks[f].size() != N) throw std::invalid_argument("LLR length must equal n");
      for (size_t i = 0; i < N; i++) llr[f * N + i] = blocks[f][i].value();
    }
    return llr;
  }
  std::vector<DecoderResult> results(size_t F, const std::vector<uint64_t>& msg, const std::vector<int32_t>& it,
                                     const std::vector<uint8_t>& cv, const std::vector<uint8_t>& so) const {
    const size_t K = k(), W = (K + 63) / 64;
    std::vector<DecoderResult> out(F);
    for (size_t f = 0; f < F; f++) {
      BitVec b = BitVec::zeros(K);
      for (size_t w = 0; w < W; w++) b.words()[w] = msg[f * W + w];
      out[f] = DecoderResult{std::move(b), (size_t)it[f], cv[f] != 0, so[f] != 0};
    }
    return out;
  }
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

// ---------------------------------------------------------------------------
// DVB-T2 outer BCH code (crates/gf2-coding/src/bch)
// ---------------------------------------------------------------------------
class BchCode {
 public:
  // BchCode::dvb_t2 (bch/dvb_t2/mod.rs:62-78): frame 0 normal, 1 short.
  static BchCode dvb_t2(int frame, CodeRate r) {
    gf2c_bch* b = nullptr;
    check(gf2c_bch_create_dvbt2(frame, (int)r, &b));
    return BchCode(b);
  }
  size_t n() const { return (size_t)n_; }
  size_t k() const { return (size_t)k_; }
  size_t t() const { return (size_t)t_; }
  int field_m() const { return m_; }
  size_t designed_distance() const { return 2 * t() + 1; }
  // BchCode::generator: binary coefficients, x^d at [d].
  std::vector<uint8_t> generator() const {
    std::vector<uint8_t> g(n() - k() + 1);
    check(gf2c_bch_generator(handle(), g.data()));
    return g;
  }
  gf2c_bch* handle() const { return h_.get(); }

 private:
  explicit BchCode(gf2c_bch* b) : h_(b, gf2c_bch_destroy) { check(gf2c_bch_dims(b, &n_, &k_, &t_, &m_)); }
  std::shared_ptr<gf2c_bch> h_;
  int64_t n_ = 0, k_ = 0;
  int32_t t_ = 0, m_ = 0;
};

namespace detail {
inline std::vector<uint64_t> pack(const std::vector<BitVec>& v, size_t len) {
  const size_t W = (len + 63) / 64;
  std::vector<uint64_t> out(v.size() * W);
  for (size_t f = 0; f < v.size(); f++) {
    if (v[f].len() != len) throw std::invalid_argument("length must be " + std::to_string(len));
    for (size_t w = 0; w < W; w++) out[f * W + w] = v[f].words()[w];
  }
  return out;
}
inline std::vector<BitVec> unpack(const std::vector<uint64_t>& w, size_t frames, size_t len) {
  const size_t W = (len + 63) / 64;
  std::vector<BitVec> r(frames);
  for (size_t f = 0; f < frames; f++) {
    r[f] = BitVec::zeros(len);
    for (size_t i = 0; i < W; i++) r[f].words()[i] = w[f * W + i];
  }
  return r;
}
}  // namespace detail

// BchEncoder (bch/core.rs:347-480): [message | parity].
class BchEncoder {
 public:
  explicit BchEncoder(BchCode code) : code_(std::move(code)) {}
  size_t k() const { return code_.k(); }
  size_t n() const { return code_.n(); }
  BitVec encode(const BitVec& m) const { return encode_batch({m})[0]; }
  std::vector<BitVec> encode_batch(const std::vector<BitVec>& msgs) const {
    if (msgs.empty()) return {};
    auto in = detail::pack(msgs, k());
    std::vector<uint64_t> out(msgs.size() * ((n() + 63) / 64));
    check(gf2c_bch_encode_batch(code_.handle(), in.data(), (int64_t)msgs.size(), out.data(), GF2C_MEM_HOST, nullptr));
    return detail::unpack(out, msgs.size(), n());
  }

 private:
  BchCode code_;
};

// BchDecoder (bch/core.rs:486-818): syndromes, Berlekamp-Massey, Chien search.
class BchDecoder {
 public:
  explicit BchDecoder(BchCode code) : code_(std::move(code)) {}
  size_t k() const { return code_.k(); }
  size_t n() const { return code_.n(); }
  BitVec decode(const BitVec& r) const { return decode_batch({r})[0]; }
  std::vector<BitVec> decode_batch(const std::vector<BitVec>& received, std::vector<int32_t>* corrected = nullptr) const {
    if (received.empty()) return {};
    auto in = detail::pack(received, n());
    std::vector<uint64_t> out(received.size() * ((k() + 63) / 64));
    std::vector<int32_t> cor(received.size());
    check(gf2c_bch_decode_batch(code_.handle(), in.data(), (int64_t)received.size(), out.data(), cor.data(), nullptr,
                                GF2C_MEM_HOST, nullptr));
    if (corrected) *corrected = cor;
    return detail::unpack(out, received.size(), k());
  }
  // BchDecoder::compute_syndromes: S_1..S_2t.
  std::vector<uint16_t> compute_syndromes(const BitVec& r) const {
    auto in = detail::pack({r}, n());
    std::vector<uint64_t> out((k() + 63) / 64);
    std::vector<uint16_t> syn(2 * code_.t());
    check(gf2c_bch_decode_batch(code_.handle(), in.data(), 1, out.data(), nullptr, syn.data(), GF2C_MEM_HOST, nullptr));
    return syn;
  }

 private:
  BchCode code_;
};

// ---------------------------------------------------------------------------
// gf2 files (gf2-core/src/io): format 0 binary "GF2DATA", 1 text, 2 hex; -1 detect
// ---------------------------------------------------------------------------
namespace io {
inline void save_bitvec(const std::string& path, const BitVec& v, int format = 0) {
  check(gf2c_io_write_bitvec(path.c_str(), v.words().data(), (int64_t)v.len(), format));
}
// BitVec::load_from_file (the format is detected).
inline BitVec load_bitvec(const std::string& path) {
  int64_t len = 0;
  check(gf2c_io_read_bitvec(path.c_str(), nullptr, 0, &len));
  BitVec v = BitVec::zeros((size_t)len);
  check(gf2c_io_read_bitvec(path.c_str(), v.words().data(), (int64_t)v.words().size(), &len));
  return v;
}
// A BitMatrix as row words (rows x ceil(cols/64)).
struct BitMatrix {
  size_t rows = 0, cols = 0;
  std::vector<uint64_t> words;
  size_t stride() const { return cols ? (cols + 63) / 64 : 0; }
  bool get(size_t r, size_t c) const { return (words.at(r * stride() + c / 64) >> (c % 64)) & 1u; }
};
inline void save_bitmatrix(const std::string& path, const BitMatrix& m, int format = 0) {
  check(gf2c_io_write_bitmatrix(path.c_str(), m.words.data(), (int64_t)m.rows, (int64_t)m.cols, format));
}
inline BitMatrix load_bitmatrix(const std::string& path, int format = 0) {
  int64_t r = 0, c = 0;
  check(gf2c_io_read_bitmatrix(path.c_str(), format, nullptr, 0, &r, &c));
  BitMatrix m;
  m.rows = (size_t)r;
  m.cols = (size_t)c;
  m.words.assign(m.rows * m.stride(), 0);
  check(gf2c_io_read_bitmatrix(path.c_str(), format, m.words.data(), (int64_t)m.words.size(), &r, &c));
  return m;
}
}  // namespace io

// Encoding from a dense parity part P (k x r): [message | P^T message] on the GPU.
class DenseEncoder {
 public:
  DenseEncoder(const std::vector<uint64_t>& P, size_t k, size_t n) : k_(k), n_(n) {
    gf2c_dense_encoder* e = nullptr;
    check(gf2c_dense_encoder_create(P.data(), (int64_t)k, (int64_t)n, &e));
    h_.reset(e, gf2c_dense_encoder_destroy);
  }
  size_t k() const { return k_; }
  size_t n() const { return n_; }
  BitVec encode(const BitVec& m) const { return encode_batch({m})[0]; }
  std::vector<BitVec> encode_batch(const std::vector<BitVec>& msgs) const {
    if (msgs.empty()) return {};
    auto in = detail::pack(msgs, k_);
    std::vector<uint64_t> out(msgs.size() * ((n_ + 63) / 64));
    check(gf2c_dense_encode_batch(h_.get(), in.data(), (int64_t)msgs.size(), out.data(), GF2C_MEM_HOST, nullptr));
    return detail::unpack(out, msgs.size(), n_);
  }

 private:
  size_t k_, n_;
  std::shared_ptr<gf2c_dense_encoder> h_;
};

// EncodingCache (ldpc/encoding/cache.rs:141-438): parity parts keyed by
// (n, k, structural hash of H), one "n{n}_k{k}_h{hash:x}.gf2" BitMatrix file each.
class EncodingCache {
 public:
  struct Key {
    size_t n, k;
    uint64_t hash;
    bool operator<(const Key& o) const { return std::tie(n, k, hash) < std::tie(o.n, o.k, o.hash); }
  };
  static Key key(const LdpcCode& code) {
    uint64_t h = 0;
    check(gf2c_code_cache_hash(code.handle(), &h));
    return Key{code.n(), code.k(), h};
  }
  static std::string filename(const Key& k) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "n%zu_k%zu_h%llx.gf2", k.n, k.k, (unsigned long long)k.hash);
    return buf;
  }
  const io::BitMatrix& get_or_compute(const LdpcCode& code) {
    const Key kk = key(code);
    auto it = entries_.find(kk);
    if (it != entries_.end()) return it->second;
    io::BitMatrix P;
    P.rows = code.k();
    P.cols = code.n() - code.k();
    P.words.assign(P.rows * P.stride(), 0);
    check(gf2c_code_parity_part(code.handle(), P.words.data()));
    return entries_.emplace(kk, std::move(P)).first->second;
  }
  // LdpcEncoder::with_cache: an encoder from the cached parity part.
  DenseEncoder encoder(const LdpcCode& code) { return DenseEncoder(get_or_compute(code).words, code.k(), code.n()); }
  size_t size() const { return entries_.size(); }
  void clear() { entries_.clear(); }
  void save_to_directory(const std::string& dir) const {
    std::filesystem::create_directories(dir);
    for (auto& e : entries_) io::save_bitmatrix((std::filesystem::path(dir) / filename(e.first)).string(), e.second);
  }
  static EncodingCache from_directory(const std::string& dir) {
    if (!std::filesystem::is_directory(dir)) throw std::invalid_argument("Directory does not exist: " + dir);
    EncodingCache c;
    for (auto& f : std::filesystem::directory_iterator(dir)) {
      if (f.path().extension() != ".gf2") continue;
      size_t n = 0, k = 0;
      unsigned long long h = 0;
      int used = 0;
      const std::string stem = f.path().stem().string();
      if (std::sscanf(stem.c_str(), "n%zu_k%zu_h%llx%n", &n, &k, &h, &used) != 3 || used != (int)stem.size()) continue;
      io::BitMatrix P = io::load_bitmatrix(f.path().string());
      if (P.rows != k || P.cols != n - k) throw std::invalid_argument(f.path().string() + ": parity part has the wrong shape");
      c.entries_.emplace(Key{n, k, (uint64_t)h}, std::move(P));
    }
    return c;
  }

 private:
  std::map<Key, io::BitMatrix> entries_;
};

}  // namespace gf2
