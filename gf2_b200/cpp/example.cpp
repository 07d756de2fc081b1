// Example / self-check of the C++ API (gf2cuda.hpp).
//   example codes   -- host-only: builds codes, checks dimensions and errors
//   example decode  -- GPU: restated decoder tests of crates/gf2-coding/src/ldpc/core.rs
#include <cstdio>
#include <cstring>

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
  std::printf("decode ok\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 1 && std::strcmp(argv[1], "decode") == 0) return decode();
  return codes();
}
