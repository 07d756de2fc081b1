// CPU oracle: systematic encoder and seeded AWGN channel (test infrastructure).
//
// Encoder semantics: LdpcEncoder::encode (crates/gf2-coding/src/ldpc/core.rs:1106-1132)
// -> RuEncodingMatrices::{compute_generator_matrix, encode}
// (crates/gf2-coding/src/ldpc/encoding/richardson_urbanke.rs:158-289): parity
// columns are the pivots of an RREF that searches columns right to left
// (crates/gf2-core/src/alg/rref.rs:67-130), message bits go to the remaining
// columns in ascending order, and the codeword is the unique one with those
// message bits.  For DVB-T2 codes the pivots are exactly the staircase columns
// k..n-1, so the unique codeword is produced by the accumulator
// p[0] = s[0], p[i] = s[i] ^ p[i-1] with s = H_info u (builder.rs:94-115).
//
// Channel: BpskModulator / AwgnChannel (crates/gf2-coding/src/channel.rs:51-218):
// bit 0 -> +1, bit 1 -> -1, sigma^2 = 1 / (2 R 10^(EbN0/10)) with R = k/n,
// y = s + sigma z, LLR = (2 y / sigma^2) as f32.  The reference draws z from
// rand_distr::Normal (unpinned); here z comes from Philox4x32-10 (Salmon et
// al., SC'11) and the Box-Muller transform with the own_math.h functions.
#include <cmath>
#include <cstring>

#include "oracle_internal.h"
#include "own_math.h"

extern "C" void or_philox4x32(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

extern "C" double or_sigma2(double ebn0_db, double rate) {
  double lin = std::pow(10.0, ebn0_db / 10.0);
  return 1.0 / (2.0 * rate * lin);
}

extern "C" double or_own_log(double x) { return ownm::log_d(x); }
extern "C" void or_own_sincos2pi(double u, double* s, double* c) { ownm::sincos_2pi_d(u, s, c); }

// ---------------- encoder ----------------
namespace {
struct Pivots {
  std::vector<int64_t> msg_cols, par_cols;
  std::vector<std::vector<uint64_t>> rows;  // reduced H, bit-packed rows
  std::vector<int64_t> pivot_row;           // row of each parity column (same order as par_cols)
  bool ok = false;
};

Pivots right_greedy(const or_code* c) {
  Pivots P;
  const int64_t m = c->m, n = c->n, W = (n + 63) / 64;
  P.rows.assign(m, std::vector<uint64_t>(W, 0));
  for (int64_t r = 0; r < m; r++)
    for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++)
      P.rows[r][c->row_idx[e] >> 6] |= 1ull << (c->row_idx[e] & 63);
  std::vector<char> used(m, 0), is_piv(n, 0);
  int64_t cur = 0;
  for (int64_t col = n - 1; col >= 0 && cur < m; col--) {
    int64_t pr = -1;
    for (int64_t r = 0; r < m; r++)
      if (!used[r] && ((P.rows[r][col >> 6] >> (col & 63)) & 1)) {
        pr = r;
        break;
      }
    if (pr < 0) continue;
    used[pr] = 1;
    for (int64_t r = 0; r < m; r++)
      if (r != pr && ((P.rows[r][col >> 6] >> (col & 63)) & 1))
        for (int64_t w = 0; w < W; w++) P.rows[r][w] ^= P.rows[pr][w];
    P.par_cols.push_back(col);
    P.pivot_row.push_back(pr);
    is_piv[col] = 1;
    cur++;
  }
  if (cur != m) return P;
  for (int64_t col = 0; col < n; col++)
    if (!is_piv[col]) P.msg_cols.push_back(col);
  P.ok = true;
  return P;
}
}  // namespace

extern "C" int or_encoder_columns(const or_code* c, int64_t* msg_cols, int64_t* par_cols) {
  Pivots P = right_greedy(c);
  if (!P.ok) {
    or_set_error("parity-check matrix is rank deficient");
    return -1;
  }
  std::memcpy(msg_cols, P.msg_cols.data(), sizeof(int64_t) * P.msg_cols.size());
  std::memcpy(par_cols, P.par_cols.data(), sizeof(int64_t) * P.par_cols.size());
  return 0;
}

static void encode_dvb(const or_code* c, const uint8_t* u, uint8_t* cw) {
  const int64_t k = c->k, m = c->m;
  std::memcpy(cw, u, (size_t)k);
  uint8_t prev = 0;
  for (int64_t p = 0; p < m; p++) {
    uint8_t s = 0;
    for (int64_t e = c->row_ptr[p]; e < c->row_ptr[p + 1]; e++) {
      int64_t v = c->row_idx[e];
      if (v < k) s ^= u[v];
    }
    prev = s ^ prev;
    cw[k + p] = prev;
  }
}

extern "C" int or_encode(const or_code* c, const uint8_t* msg, int64_t frames, uint8_t* cw) {
  if (c->dvb_q > 0) {
    for (int64_t f = 0; f < frames; f++) encode_dvb(c, msg + f * c->k, cw + f * c->n);
    return 0;
  }
  if (c->m >= c->n || c->m == 0) {
    or_set_error("invalid dimensions for encoding");
    return -1;
  }
  Pivots P = right_greedy(c);
  if (!P.ok) {
    or_set_error("parity-check matrix is rank deficient");
    return -1;
  }
  const int64_t n = c->n, k = c->k;
  for (int64_t f = 0; f < frames; f++) {
    const uint8_t* u = msg + f * k;
    uint8_t* x = cw + f * n;
    std::memset(x, 0, (size_t)n);
    for (int64_t i = 0; i < k; i++) x[P.msg_cols[i]] = u[i] & 1;
    for (size_t j = 0; j < P.par_cols.size(); j++) {
      const auto& row = P.rows[P.pivot_row[j]];
      uint8_t acc = 0;
      for (int64_t i = 0; i < k; i++) {
        int64_t col = P.msg_cols[i];
        if ((row[col >> 6] >> (col & 63)) & 1) acc ^= x[col];
      }
      x[P.par_cols[j]] = acc;
    }
  }
  return 0;
}

// ---------------- channel ----------------
extern "C" int or_channel_frames(const or_code* c, uint64_t seed, uint64_t frame0, int64_t frames,
                                 const double* ebn0_db, uint8_t* info, uint8_t* cw, float* llr) {
  const int64_t n = c->n, k = c->k;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const double rate = (double)k / (double)n;
  std::vector<uint8_t> u(k), x(n);
  for (int64_t f = 0; f < frames; f++) {
    uint32_t fr = (uint32_t)(frame0 + f);
    for (int64_t blk = 0; blk * 128 < k; blk++) {
      uint32_t ctr[4] = {(uint32_t)blk, fr, 1u, 0u}, out[4];
      or_philox4x32(ctr, key, out);
      for (int b = 0; b < 128 && blk * 128 + b < k; b++) u[blk * 128 + b] = (out[b >> 5] >> (b & 31)) & 1u;
    }
    if (or_encode(c, u.data(), 1, x.data()) != 0) return -1;
    double s2 = or_sigma2(ebn0_db[f], rate);
    double sigma = std::sqrt(s2);
    for (int64_t pair = 0; 2 * pair < n; pair++) {
      uint32_t ctr[4] = {(uint32_t)pair, fr, 2u, 0u}, out[4];
      or_philox4x32(ctr, key, out);
      uint64_t a = ((((uint64_t)out[0]) << 32) | out[1]) >> 11;
      uint64_t b = ((((uint64_t)out[2]) << 32) | out[3]) >> 11;
      double u1 = (double)(a + 1) * 1.1102230246251565404e-16;  // 2^-53
      double u2 = (double)b * 1.1102230246251565404e-16;
      double rad = std::sqrt(-2.0 * ownm::log_d(u1));
      double sn, cs;
      ownm::sincos_2pi_d(u2, &sn, &cs);
      double z[2] = {rad * cs, rad * sn};
      for (int h = 0; h < 2; h++) {
        int64_t i = 2 * pair + h;
        if (i >= n) break;
        double sym = x[i] ? -1.0 : 1.0;
        double y = sym + sigma * z[h];
        if (llr) llr[f * n + i] = (float)((2.0 * y) / s2);
      }
    }
    if (info) std::memcpy(info + f * k, u.data(), (size_t)k);
    if (cw) std::memcpy(cw + f * n, x.data(), (size_t)n);
  }
  return 0;
}

// AwgnChannel::shannon_capacity / shannon_limit (channel.rs:245-330)
static double capacity_numerical(double snr) {
  double sq = std::sqrt(snr);
  int npts = 1000;
  double ymax = sq + 6.0;
  double dy = 2.0 * ymax / npts;
  double s2pi = std::sqrt(2.0 * M_PI);
  double integral = 0.0;
  for (int i = 0; i <= npts; i++) {
    double y = -ymax + i * dy;
    double fy = std::exp(-((y - sq) * (y - sq)) / 2.0) / s2pi;
    double arg = -2.0 * sq * y;
    double lt;
    if (arg > 20.0) lt = arg / M_LN2;
    else if (arg < -20.0) lt = 0.0;
    else lt = std::log2(1.0 + std::exp(arg));
    double w = (i == 0 || i == npts) ? 0.5 : 1.0;
    integral += w * fy * lt;
  }
  double cap = 1.0 - integral * dy;
  return cap < 0 ? 0 : (cap > 1 ? 1 : cap);
}

extern "C" double or_shannon_limit(double rate) {
  double lo = -10.0, hi = 25.0;
  for (int i = 0; i < 60; i++) {
    double mid = (lo + hi) / 2.0;
    double cap = capacity_numerical(std::pow(10.0, mid / 10.0));
    if (std::fabs(cap - rate) < 1e-6) return mid;
    if (cap > rate) hi = mid;
    else lo = mid;
  }
  return (lo + hi) / 2.0;
}
