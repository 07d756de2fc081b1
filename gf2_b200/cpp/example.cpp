// Example / self-check of the C++ API (gf2cuda.hpp).
//   example codes   -- host-only: builds codes, checks dimensions and errors, BCH
//                      parameters, gf2 file roundtrips and the encoder cache
//   example decode  -- GPU: restated decoder tests of crates/gf2-coding/src/ldpc/core.rs,
//                      BCH correction, cached-parity encoding
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <filesystem>

#include "gf2cuda.hpp"

#define EXPECT(c)                                                   \
  do {                                                              \
    if (!(c)) {                                                     \
      std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                                     \
    }                                                               \
  } while (0)

static int codes() {
  auto s = gf2::LdpcCode::dvb_t2_short(gf2::CodeRate::Rate1_2);
  EXPECT(s.n() == 16200 && s.k() == 7200 && s.m() == 9000);
  auto nrm = gf2::LdpcCode::dvb_t2_normal(gf2::CodeRate::Rate3_5);
  EXPECT(nrm.n() == 64800 && nrm.k() == 38880);
  auto q = gf2::LdpcCode::from_quasi_cyclic(gf2::QuasiCyclicLdpc({{0, 1}, {1, 0}}, 3));
  EXPECT(q.m() == 6 && q.n() == 6);
  auto e = gf2::LdpcCode::from_edges(3, 7, {{0, 0}, {0, 1}, {0, 3}, {1, 0}, {1, 2}, {1, 4}, {2, 1}, {2, 2}, {2, 5}});
  EXPECT(e.n() == 7 && e.m() == 3 && e.k() == 4);
  bool threw = false;
  try {
    gf2::LdpcCode::from_quasi_cyclic(gf2::QuasiCyclicLdpc({{5}}, 3));
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  EXPECT(threw);
  // BCH parameters (bch/dvb_t2/params.rs tests): generator degree t m
  auto bch = gf2::BchCode::dvb_t2(0, gf2::CodeRate::Rate2_3);
  EXPECT(bch.n() == 43200 && bch.k() == 43040 && bch.t() == 10 && bch.field_m() == 16);
  EXPECT(bch.generator().size() == 161 && bch.generator()[160] == 1);
  EXPECT(gf2::BchCode::dvb_t2(1, gf2::CodeRate::Rate1_2).generator().size() == 169);
  // gf2 files: roundtrips and the cache file name
  const std::string dir = std::filesystem::temp_directory_path() / ("gf2cpp_" + std::to_string(::getpid()));
  std::filesystem::create_directories(dir);
  gf2::BitVec v = gf2::BitVec::zeros(100);
  v.set(3, true);
  v.set(99, true);
  for (int fmt = 0; fmt < 3; fmt++) {
    gf2::io::save_bitvec(dir + "/v", v, fmt);
    EXPECT(gf2::io::load_bitvec(dir + "/v") == v);
  }
  s.save(dir + "/h.gf2");
  auto s2 = gf2::LdpcCode::from_file(dir + "/h.gf2");
  EXPECT(s2.n() == s.n() && s2.k() == s.k());
  gf2::EncodingCache cache;
  const auto& P = cache.get_or_compute(s);
  EXPECT(P.rows == 7200 && P.cols == 9000);
  gf2::BitVec cw = gf2::BitVec::zeros(s.n());
  cw.set(17, true);
  for (size_t j = 0; j < P.cols; j++) cw.set(7200 + j, P.get(17, j));
  {  // H cw = 0 on the host, from the CSR
    std::vector<int64_t> ptr(s.m() + 1);
    int64_t nnz = 0;
    gf2::check(gf2c_code_dims(s.handle(), nullptr, nullptr, nullptr, &nnz, nullptr));
    std::vector<int64_t> idx((size_t)nnz);
    gf2::check(gf2c_code_csr(s.handle(), ptr.data(), idx.data()));
    for (size_t r = 0; r < s.m(); r++) {
      bool par = false;
      for (int64_t e = ptr[r]; e < ptr[r + 1]; e++) par ^= cw.get((size_t)idx[e]);
      EXPECT(!par);
    }
  }
  cache.save_to_directory(dir + "/cache");
  auto loaded = gf2::EncodingCache::from_directory(dir + "/cache");
  EXPECT(loaded.size() == 1);
  const auto name = gf2::EncodingCache::filename(gf2::EncodingCache::key(s));
  EXPECT(name.rfind("n16200_k7200_h", 0) == 0 && std::filesystem::exists(dir + "/cache/" + name));
  std::filesystem::remove_all(dir);
  std::printf("codes ok\n");
  return 0;
}

static int decode() {
  using gf2::Llr;
  auto spc = gf2::LdpcCode::from_edges(1, 3, {{0, 0}, {0, 1}, {0, 2}});
  gf2::LdpcDecoder dec(spc);
  auto r = dec.decode_iterative({Llr(10), Llr(10), Llr(10)}, 10);
  EXPECT(r.converged && r.syndrome_check_passed && r.decoded_bits.count_ones() == 0 && r.iterations <= 2);
  r = dec.decode_iterative({Llr(-5), Llr(-5), Llr(2)}, 20);
  EXPECT(r.converged && r.decoded_bits.count_ones() == 2);
  auto rs = gf2::LdpcDecoder::decode_batch(spc, {{Llr(10), Llr(10), Llr(10)}, {Llr(-10), Llr(-10), Llr(10)}}, 10);
  EXPECT(rs.size() == 2 && rs[0].decoded_bits.count_ones() == 0 && rs[1].decoded_bits.count_ones() == 2);
  gf2::LdpcEncoder enc(spc);
  gf2::BitVec m = gf2::BitVec::zeros(2);
  m.set(0, true);
  auto cw = enc.encode(m);
  EXPECT(cw.len() == 3 && cw.get(0) && !cw.get(1) && cw.get(2));
  EXPECT(spc.is_valid_codeword(cw));
  auto s = gf2::LdpcCode::dvb_t2_short(gf2::CodeRate::Rate1_2);
  gf2::LdpcDecoder ds(s);
  r = ds.decode_iterative(std::vector<Llr>(s.n(), Llr(5.0f)), 10);
  EXPECT(r.converged && r.decoded_bits.count_ones() == 0);
  gf2::BitVec msg = gf2::BitVec::zeros(s.k());
  for (size_t i = 0; i < s.k(); i += 3) msg.set(i, true);
  auto c = gf2::LdpcEncoder(s).encode(msg);
  EXPECT(s.is_valid_codeword(c));
  std::vector<Llr> l(s.n());
  for (size_t i = 0; i < s.n(); i++) l[i] = Llr(c.get(i) ? -4.0f : 4.0f);
  r = ds.decode_iterative(l, 20);
  EXPECT(r.converged && r.decoded_bits == msg);
  // a decoder with a layered fallback: one primary iteration leaves the noisy
  // frame failing, the fallback finishes it; the clean frame stays with the
  // primary decoder
  {
    gf2c_decoder_opts lo;
    gf2c_decoder_opts_default(&lo);
    lo.schedule = GF2C_SCHED_LAYERED;
    gf2::LdpcDecoder prim(s, &lo), fb(s, &lo);
    std::vector<Llr> noisy = l;
    for (size_t i = 0; i < s.n(); i += 7) noisy[i] = Llr(-0.25f * noisy[i].value());
    size_t redecoded = 0;
    auto rf = prim.decode_many_with_fallback(fb, {l, noisy}, 1, 30, &redecoded);
    EXPECT(rf.size() == 2 && rf[0].decoded_bits == msg && rf[0].iterations == 1);
    EXPECT(redecoded == 1 && rf[1].syndrome_check_passed && rf[1].decoded_bits == msg && rf[1].iterations > 1);
  }
  // outer BCH: t errors corrected (bch/dvb_t2/mod.rs roundtrip tests)
  auto bch = gf2::BchCode::dvb_t2(1, gf2::CodeRate::Rate1_2);
  gf2::BitVec bm = gf2::BitVec::zeros(bch.k());
  for (size_t i = 0; i < bch.k(); i += 5) bm.set(i, true);
  auto bc = gf2::BchEncoder(bch).encode(bm);
  EXPECT(bc.len() == bch.n());
  for (size_t e = 0; e < bch.t(); e++) bc.set(97 * e + 11, !bc.get(97 * e + 11));
  std::vector<int32_t> corrected;
  auto bd = gf2::BchDecoder(bch).decode_batch({bc}, &corrected);
  EXPECT(bd[0] == bm && corrected[0] == (int32_t)bch.t());
  // encoding from the cached parity part equals the encoder's codeword
  gf2::EncodingCache cache;
  EXPECT(cache.encoder(s).encode(msg) == c);
  std::printf("decode ok\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 1 && std::strcmp(argv[1], "decode") == 0) return decode();
  return codes();
}
