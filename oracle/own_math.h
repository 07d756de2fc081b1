// CPU oracle: the numeric specification of the library's FP32 sum-product
// check node and of its FP64 channel transcendental functions (test
// infrastructure only).
//
// These are written from textbook methods so that the CPU and the GPU evaluate
// the same sequence of correctly-rounded IEEE operations (add, sub, mul, div,
// sqrt; no fused multiply-add) and agree bit for bit:
//   * exp / expm1: Cody & Waite range reduction x = k ln2 + r with ln2 split
//     into a short high part and a low part, then the Taylor series of
//     expm1(r) in Horner form.
//   * log / log1p: x = 2^e f with f in [sqrt(1/2), sqrt(2)), then
//     log f = 2 atanh(s), s = (f-1)/(f+1), by its odd power series
//     (Abramowitz & Stegun 4.1.27).
//   * sin / cos of 2*pi*u: exact quadrant split of 4u, reflection to
//     [0, pi/4], Taylor series.
// The oracle is compiled with -ffp-contract=off.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace ownm {

// ---------------- FP32: sum-product check node ----------------
// tanh(a/2) for a >= 0, via expm1(-a): tanh(a/2) = -em1 / (2 + em1).
static inline float expm1_neg_f(float a) {  // expm1(-a), a >= 0
  if (a > 30.0f) return -1.0f;
  const float inv_ln2 = 1.44269504088896341f;
  const float ln2_hi = 0.693145751953125f;      // 12 significant bits
  const float ln2_lo = 1.42860682030941723e-06f;
  float x = -a;
  float kf = std::nearbyint(x * inv_ln2);       // round half to even
  float r = (x - kf * ln2_hi) - kf * ln2_lo;
  // expm1(r), |r| <= 0.35: Taylor to r^8
  float p = 1.0f / 40320.0f;
  p = p * r + 1.0f / 5040.0f;
  p = p * r + 1.0f / 720.0f;
  p = p * r + 1.0f / 120.0f;
  p = p * r + 1.0f / 24.0f;
  p = p * r + 1.0f / 6.0f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  float em1r = p * r;
  int k = (int)kf;
  if (k == 0) return em1r;
  float two_k = std::ldexp(1.0f, k);
  return two_k * em1r + (two_k - 1.0f);
}

static inline float tanh_half_f(float x) {  // tanh(x/2), signed
  float a = std::fabs(x);
  float em1 = expm1_neg_f(a);
  float t = -em1 / (2.0f + em1);
  return (x < 0.0f) ? -t : t;
}

// log(u) for u > 0 finite
static inline float log_f(float u) {
  int e;
  float f = std::frexp(u, &e);  // u = f 2^e, f in [0.5, 1)
  if (f < 0.70710678118654752f) {
    f = f * 2.0f;
    e -= 1;
  }
  float s = (f - 1.0f) / (f + 1.0f);
  float s2 = s * s;
  float p = 1.0f / 11.0f;
  p = p * s2 + 1.0f / 9.0f;
  p = p * s2 + 1.0f / 7.0f;
  p = p * s2 + 1.0f / 5.0f;
  p = p * s2 + 1.0f / 3.0f;
  p = p * s2 + 1.0f;
  float logf_ = 2.0f * (s * p);
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.42860682030941723e-06f;
  float ef = (float)e;
  return (ef * ln2_hi + logf_) + ef * ln2_lo;
}

// log1p(y) for y >= 0: log(u) * y / (u - 1) with u = 1 + y (Goldberg's trick)
static inline float log1p_f(float y) {
  float u = 1.0f + y;
  if (u == 1.0f) return y;
  return log_f(u) * (y / (u - 1.0f));
}

// 2 atanh(p) for |p| < 1: sign(p) log1p(2|p| / (1 - |p|))
static inline float two_atanh_f(float p) {
  float a = std::fabs(p);
  float r = log1p_f((2.0f * a) / (1.0f - a));
  return (p < 0.0f) ? -r : r;
}

// clamp of the extrinsic tanh product: |P| <= 1 - 2^-23, |c2v| <= 16.64
static const float kSpaPMax = 0.99999988079071045f;

// ---------------- FP64: channel ----------------
static inline double log_d(double u) {  // u > 0 finite
  int e;
  double f = std::frexp(u, &e);
  if (f < 0.70710678118654752440) {
    f = f * 2.0;
    e -= 1;
  }
  double s = (f - 1.0) / (f + 1.0);
  double s2 = s * s;
  // 2 atanh(s) = 2 sum s^(2j+1)/(2j+1), |s| <= 0.1716, thirteen terms
  static const double inv_odd[13] = {1.0, 1.0 / 3.0, 1.0 / 5.0, 1.0 / 7.0, 1.0 / 9.0,
                                     1.0 / 11.0, 1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0,
                                     1.0 / 19.0, 1.0 / 21.0, 1.0 / 23.0, 1.0 / 25.0};
  double p = inv_odd[12];
  for (int j = 11; j >= 0; j--) p = p * s2 + inv_odd[j];
  double lf = 2.0 * (s * p);
  const double ln2_hi = 6.93147180369123816490e-01;  // 32 significant bits
  const double ln2_lo = 1.90821492927058770002e-10;
  double ed = (double)e;
  return (ed * ln2_hi + lf) + ed * ln2_lo;
}

// sin(2 pi u), cos(2 pi u) for u in [0, 1)
static inline void sincos_2pi_d(double u, double* s_out, double* c_out) {
  const double half_pi = 1.57079632679489661923;
  double t4 = u * 4.0;        // exact
  double qd = std::floor(t4);
  double r = t4 - qd;         // exact, in [0, 1)
  int q = (int)qd & 3;
  bool refl = r > 0.5;
  double rr = refl ? (1.0 - r) : r;  // exact
  double a = rr * half_pi;           // in [0, pi/4]
  double a2 = a * a;
  // Taylor series: sin a = sum (-1)^j a^(2j+1)/(2j+1)!, cos a = sum (-1)^j a^(2j)/(2j)!,
  // |a| <= pi/4, ten terms each; Horner in a^2 with the exact reciprocal factorials.
  static const double inv_fact[22] = {
      1.0, 1.0, 1.0 / 2.0, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0,
      1.0 / 40320.0, 1.0 / 362880.0, 1.0 / 3628800.0, 1.0 / 39916800.0, 1.0 / 479001600.0,
      1.0 / 6227020800.0, 1.0 / 87178291200.0, 1.0 / 1307674368000.0,
      1.0 / 20922789888000.0, 1.0 / 355687428096000.0, 1.0 / 6402373705728000.0,
      1.0 / 121645100408832000.0, 1.0 / 2432902008176640000.0,
      1.0 / 51090942171709440000.0};
  double ss = 0.0, cc = 0.0;
  for (int j = 10; j >= 0; j--) {
    ss = ss * a2 + ((j & 1) ? -inv_fact[2 * j + 1] : inv_fact[2 * j + 1]);
    cc = cc * a2 + ((j & 1) ? -inv_fact[2 * j] : inv_fact[2 * j]);
  }
  double sn = a * ss;
  double cs = cc;
  double s0 = refl ? cs : sn;   // sin(r pi/2)
  double c0 = refl ? sn : cs;   // cos(r pi/2)
  switch (q) {
    case 0: *s_out = s0; *c_out = c0; break;
    case 1: *s_out = c0; *c_out = -s0; break;
    case 2: *s_out = -s0; *c_out = -c0; break;
    default: *s_out = -c0; *c_out = s0; break;
  }
}

}  // namespace ownm
