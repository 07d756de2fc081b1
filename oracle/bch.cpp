// CPU oracle (test infrastructure): restatement of the reference's DVB-T2 BCH
// outer code.
//
//   DvbBchParams::for_code (n = k_ldpc, k = Kbch, t, GF(2^m), primitive poly)
//                                            bch/dvb_t2/params.rs:56-85
//   g(x) = g_1(x) ... g_t(x), binary tables    bch/dvb_t2/generators.rs:14-62
//   BchCode::dvb_t2                            bch/dvb_t2/mod.rs:62-78
//   BchEncoder::encode: [message | parity], bit i at degree n-1-i,
//     parity = x^r m(x) mod g(x)               bch/core.rs:421-480
//   BchDecoder::compute_syndromes: S_j = r(alpha^j), j = 1..2t
//                                            bch/core.rs:562-617
//   BchDecoder::decode: all-zero syndromes -> message as received, else
//     Berlekamp-Massey, Chien search over alpha^-i, flip bit n-1-i for every
//     root i (no check of the root count), first k bits
//                                            bch/core.rs:620-665, 695-818
//   Gf2mField::primitive_element = exp[1] = x  gf2-core/src/gf2m/field.rs:340-351
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "oracle.h"

namespace {

// ETSI EN 302 755 generator factors g_1..g_12 (exponent lists; standard data,
// the same numbers as the reference's tables).
const std::vector<std::vector<int>> kShortGen = {
    {0, 1, 3, 5, 14},          {0, 6, 8, 11, 14},         {0, 1, 2, 6, 9, 10, 14},
    {0, 4, 7, 8, 10, 12, 14},  {0, 2, 4, 6, 8, 9, 11, 13, 14}, {0, 3, 7, 8, 9, 13, 14},
    {0, 2, 5, 6, 7, 10, 11, 13, 14}, {0, 5, 8, 9, 10, 11, 14}, {0, 1, 2, 3, 9, 10, 14},
    {0, 3, 6, 9, 11, 12, 14},  {0, 4, 11, 12, 14},        {0, 1, 2, 3, 5, 6, 7, 8, 10, 13, 14}};
const std::vector<std::vector<int>> kNormalGen = {
    {0, 2, 3, 5, 16},
    {0, 1, 4, 5, 6, 8, 16},
    {0, 2, 3, 4, 5, 7, 8, 9, 10, 11, 16},
    {0, 2, 4, 6, 9, 11, 12, 14, 16},
    {0, 1, 2, 3, 5, 8, 9, 10, 11, 12, 16},
    {0, 2, 4, 5, 7, 8, 9, 10, 12, 13, 14, 15, 16},
    {0, 2, 5, 6, 8, 9, 10, 11, 13, 15, 16},
    {0, 1, 2, 5, 6, 8, 9, 12, 13, 14, 16},
    {0, 5, 7, 9, 10, 11, 16},
    {0, 1, 2, 5, 7, 8, 10, 12, 13, 14, 16},
    {0, 2, 3, 5, 9, 11, 12, 13, 16},
    {0, 1, 5, 6, 7, 9, 11, 12, 16}};

}  // namespace

struct or_bch {
  int n = 0, k = 0, t = 0, mf = 0;
  int N = 0;                       // 2^m - 1
  std::vector<uint16_t> exp, log;  // exp[0..2N), log[0..2^m)
  std::vector<uint8_t> g;          // generator coefficients, g[d] of x^d

  uint16_t mul(uint16_t a, uint16_t b) const {
    if (!a || !b) return 0;
    return exp[log[a] + log[b]];
  }
  uint16_t inv(uint16_t a) const { return exp[(N - log[a]) % N]; }
  uint16_t alpha_pow(long long e) const {  // alpha^e, any integer e
    long long r = e % N;
    if (r < 0) r += N;
    return exp[r];
  }
};

namespace {

int degree_of(const std::vector<uint16_t>& p) {
  for (int d = (int)p.size() - 1; d >= 0; d--)
    if (p[d]) return d;
  return -1;  // zero polynomial
}

void encode_one(const or_bch& B, const uint8_t* msg, uint8_t* cw) {
  const int r = B.n - B.k;
  std::vector<uint8_t> reg(r, 0);  // remainder of x^r m(x) mod g, reg[d] of x^d
  for (int i = 0; i < B.k; i++) {   // message bit i = coefficient of degree k-1-i (highest first)
    const uint8_t fb = (uint8_t)((msg[i] & 1) ^ reg[r - 1]);
    for (int d = r - 1; d > 0; d--) reg[d] = reg[d - 1] ^ (fb & B.g[d]);
    reg[0] = fb & B.g[0];
  }
  for (int i = 0; i < B.k; i++) cw[i] = msg[i] & 1;
  for (int q = 0; q < r; q++) cw[B.k + q] = reg[r - 1 - q];  // parity degree r-1-q
}

void syndromes_one(const or_bch& B, const uint8_t* cw, uint16_t* S) {
  for (int j = 1; j <= 2 * B.t; j++) {
    uint16_t s = 0;
    for (int i = 0; i < B.n; i++)
      if (cw[i] & 1) s ^= B.alpha_pow((long long)j * (B.n - 1 - i));
    S[j - 1] = s;
  }
}

// BchDecoder::berlekamp_massey, step for step
std::vector<uint16_t> berlekamp_massey(const or_bch& B, const uint16_t* S) {
  std::vector<uint16_t> lambda{1}, b{1};
  int l = 0, m = 1;
  for (int n = 0; n < 2 * B.t; n++) {
    uint16_t delta = S[n];
    const int dl = std::max(degree_of(lambda), 0);
    for (int i = 1; i <= l; i++)
      if (i <= dl && n >= i) delta ^= B.mul(lambda[i], S[n - i]);
    if (delta == 0) {
      m += 1;
    } else {
      const std::vector<uint16_t> t = lambda;
      const int db = std::max(degree_of(b), 0);
      std::vector<uint16_t> term(m + db + 1, 0);
      for (int i = 0; i <= db; i++) term[m + i] = B.mul(delta, b[i]);
      if (lambda.size() < term.size()) lambda.resize(term.size(), 0);
      for (size_t i = 0; i < term.size(); i++) lambda[i] ^= term[i];
      if (2 * l <= n) {
        l = n + 1 - l;
        const uint16_t di = B.inv(delta);
        const int dt = std::max(degree_of(t), 0);
        b.assign(dt + 1, 0);
        for (int i = 0; i <= dt; i++) b[i] = B.mul(t[i], di);
        m = 1;
      } else {
        m += 1;
      }
    }
  }
  lambda.resize(std::max(degree_of(lambda), 0) + 1);
  return lambda;
}

// BchDecoder::chien_search: degrees i in [0, n) with lambda(alpha^-i) = 0
std::vector<int> chien_search(const or_bch& B, const std::vector<uint16_t>& lambda) {
  std::vector<int> pos;
  const int deg = std::max(degree_of(lambda), 0);
  if (deg == 0) return pos;
  std::vector<uint16_t> step(deg + 1), c(lambda.begin(), lambda.begin() + deg + 1);
  for (int j = 0; j <= deg; j++) step[j] = B.alpha_pow(-(long long)j);
  for (int i = 0; i < B.n; i++) {
    uint16_t e = 0;
    for (int j = 0; j <= deg; j++) e ^= c[j];
    if (e == 0) pos.push_back(i);
    for (int j = 0; j <= deg; j++) c[j] = B.mul(c[j], step[j]);
  }
  return pos;
}

}  // namespace

extern "C" {

or_bch* or_bch_dvbt2(int frame, int rate) {
  static const int kShortN[6] = {7200, 9720, 10800, 11880, 12600, 13320};
  static const int kShortK[6] = {7032, 9552, 10632, 11712, 12432, 13152};
  static const int kNormalN[6] = {32400, 38880, 43200, 48600, 51840, 54000};
  static const int kNormalK[6] = {32208, 38688, 43040, 48408, 51648, 53840};
  static const int kNormalT[6] = {12, 12, 10, 12, 12, 10};
  if (frame < 0 || frame > 1 || rate < 0 || rate > 5) return nullptr;
  or_bch* B = new or_bch();
  const bool shortf = frame == 1;
  B->n = shortf ? kShortN[rate] : kNormalN[rate];
  B->k = shortf ? kShortK[rate] : kNormalK[rate];
  B->t = shortf ? 12 : kNormalT[rate];
  B->mf = shortf ? 14 : 16;
  const uint32_t prim = shortf ? 0b100000000101011u : 0b10000000000101101u;
  const int q = 1 << B->mf;
  B->N = q - 1;
  B->exp.assign(2 * B->N, 0);
  B->log.assign(q, 0);
  uint32_t x = 1;
  for (int e = 0; e < B->N; e++) {
    B->exp[e] = (uint16_t)x;
    B->log[x] = (uint16_t)e;
    x <<= 1;
    if (x & (uint32_t)q) x ^= prim;
  }
  for (int e = B->N; e < 2 * B->N; e++) B->exp[e] = B->exp[e - B->N];
  const auto& gens = shortf ? kShortGen : kNormalGen;
  std::vector<uint8_t> g{1};
  for (int i = 0; i < B->t; i++) {
    std::vector<uint8_t> f(B->mf + 1, 0);
    for (int e : gens[i]) f[e] = 1;
    std::vector<uint8_t> p(g.size() + f.size() - 1, 0);
    for (size_t a = 0; a < g.size(); a++)
      if (g[a])
        for (size_t b = 0; b < f.size(); b++) p[a + b] ^= f[b];
    g = p;
  }
  B->g = g;
  return B;
}

void or_bch_free(or_bch* B) { delete B; }

void or_bch_dims(const or_bch* B, int64_t* out5) {
  out5[0] = B->n;
  out5[1] = B->k;
  out5[2] = B->t;
  out5[3] = B->mf;
  out5[4] = (int64_t)B->g.size() - 1;
}

void or_bch_generator(const or_bch* B, uint8_t* coeffs) {
  std::memcpy(coeffs, B->g.data(), B->g.size());
}

void or_bch_encode(const or_bch* B, const uint8_t* msg, int64_t frames, uint8_t* cw) {
  for (int64_t f = 0; f < frames; f++) encode_one(*B, msg + f * B->k, cw + f * B->n);
}

void or_bch_syndromes(const or_bch* B, const uint8_t* cw, int64_t frames, uint16_t* synd) {
  for (int64_t f = 0; f < frames; f++) syndromes_one(*B, cw + f * B->n, synd + f * 2 * B->t);
}

int or_bch_berlekamp_massey(const or_bch* B, const uint16_t* synd, uint16_t* lambda) {
  const std::vector<uint16_t> L = berlekamp_massey(*B, synd);
  for (int i = 0; i <= 2 * B->t; i++) lambda[i] = i < (int)L.size() ? L[i] : 0;
  return (int)L.size() - 1;
}

void or_bch_decode(const or_bch* B, const uint8_t* cw, int64_t frames, uint8_t* msg, int32_t* nflips) {
  std::vector<uint16_t> S(2 * B->t);
  std::vector<uint8_t> c(B->n);
  for (int64_t f = 0; f < frames; f++) {
    const uint8_t* r = cw + f * B->n;
    syndromes_one(*B, r, S.data());
    for (int i = 0; i < B->n; i++) c[i] = r[i] & 1;
    int flips = 0;
    if (std::any_of(S.begin(), S.end(), [](uint16_t s) { return s != 0; })) {
      const std::vector<int> pos = chien_search(*B, berlekamp_massey(*B, S.data()));
      for (int i : pos) c[B->n - 1 - i] ^= 1;
      flips = (int)pos.size();
    }
    std::memcpy(msg + f * B->k, c.data(), B->k);
    if (nflips) nflips[f] = flips;
  }
}

}  // extern "C"
