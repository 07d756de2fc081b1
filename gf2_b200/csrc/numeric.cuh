// Device numeric helpers of gf2cuda.
//
// The FP32 sum-product check node and the FP64 Box-Muller channel use
// transcendental functions written here from textbook methods, using only
// correctly rounded IEEE operations (explicit _rn intrinsics: no contraction to
// fused multiply-add), so that their results are reproducible bit for bit by a
// plain C++ implementation of the same steps:
//   * expm1: Cody & Waite reduction x = k ln2 + r (ln2 split in a 12-bit high
//     part and a low part), Taylor series of expm1(r) to r^8 in Horner form;
//     tanh(a/2) = -expm1(-a) / (2 + expm1(-a)).
//   * log: x = 2^e f, f in [sqrt(1/2), sqrt(2)), log f = 2 atanh(s) with
//     s = (f - 1)/(f + 1) by its odd power series (Abramowitz & Stegun 4.1.27);
//     log1p(y) = log(1 + y) * y / ((1 + y) - 1) (Goldberg 1991).
//   * sin/cos(2 pi u): exact quadrant split of 4u, reflection to [0, pi/4],
//     Taylor series with exactly rounded reciprocal factorials.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

namespace gf2c {

// ---------------------------- FP32 ----------------------------
__device__ __forceinline__ float frexp_pos(float u, int* e) {
  // u > 0, normal
  uint32_t b = __float_as_uint(u);
  *e = (int)((b >> 23) & 0xff) - 126;
  return __uint_as_float((b & 0x807fffffu) | (126u << 23));
}

__device__ __forceinline__ float expm1_neg_f(float a) {  // expm1(-a), a >= 0
  if (a > 30.0f) return -1.0f;
  const float inv_ln2 = 1.44269504088896341f;
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.42860682030941723e-06f;
  float x = -a;
  float kf = rintf(__fmul_rn(x, inv_ln2));
  float r = __fsub_rn(__fsub_rn(x, __fmul_rn(kf, ln2_hi)), __fmul_rn(kf, ln2_lo));
  float p = 1.0f / 40320.0f;
  p = __fadd_rn(__fmul_rn(p, r), 1.0f / 5040.0f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f / 720.0f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f / 120.0f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f / 24.0f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f / 6.0f);
  p = __fadd_rn(__fmul_rn(p, r), 0.5f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f);
  float em1r = __fmul_rn(p, r);
  int k = (int)kf;
  if (k == 0) return em1r;
  float two_k = __uint_as_float((uint32_t)(k + 127) << 23);  // k in [-44, 0]
  return __fadd_rn(__fmul_rn(two_k, em1r), __fsub_rn(two_k, 1.0f));
}

__device__ __forceinline__ float tanh_half_f(float x) {  // tanh(x/2)
  float a = fabsf(x);
  float em1 = expm1_neg_f(a);
  float t = __fdiv_rn(-em1, __fadd_rn(2.0f, em1));
  return (x < 0.0f) ? -t : t;
}

__device__ __forceinline__ float log_f(float u) {  // u >= 1, finite
  int e;
  float f = frexp_pos(u, &e);
  if (f < 0.70710678118654752f) {
    f = __fmul_rn(f, 2.0f);
    e -= 1;
  }
  float s = __fdiv_rn(__fsub_rn(f, 1.0f), __fadd_rn(f, 1.0f));
  float s2 = __fmul_rn(s, s);
  float p = 1.0f / 11.0f;
  p = __fadd_rn(__fmul_rn(p, s2), 1.0f / 9.0f);
  p = __fadd_rn(__fmul_rn(p, s2), 1.0f / 7.0f);
  p = __fadd_rn(__fmul_rn(p, s2), 1.0f / 5.0f);
  p = __fadd_rn(__fmul_rn(p, s2), 1.0f / 3.0f);
  p = __fadd_rn(__fmul_rn(p, s2), 1.0f);
  float lf = __fmul_rn(2.0f, __fmul_rn(s, p));
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.42860682030941723e-06f;
  float ef = (float)e;
  return __fadd_rn(__fadd_rn(__fmul_rn(ef, ln2_hi), lf), __fmul_rn(ef, ln2_lo));
}

__device__ __forceinline__ float log1p_f(float y) {  // y >= 0
  float u = __fadd_rn(1.0f, y);
  if (u == 1.0f) return y;
  return __fmul_rn(log_f(u), __fdiv_rn(y, __fsub_rn(u, 1.0f)));
}

__device__ __forceinline__ float two_atanh_f(float p) {  // |p| < 1
  float a = fabsf(p);
  float r = log1p_f(__fdiv_rn(__fmul_rn(2.0f, a), __fsub_rn(1.0f, a)));
  return (p < 0.0f) ? -r : r;
}

// |extrinsic tanh product| <= 1 - 2^-23, so |c2v| <= 16.64
#define GF2C_SPA_PMAX 0.99999988079071045f

// ---------------------------- FP64 ----------------------------
__device__ __forceinline__ double frexp_pos_d(double u, int* e) {  // u > 0 normal
  unsigned long long b = (unsigned long long)__double_as_longlong(u);
  *e = (int)((b >> 52) & 0x7ff) - 1022;
  return __longlong_as_double((long long)((b & 0x800fffffffffffffull) | (1022ull << 52)));
}

__device__ __forceinline__ double log_d(double u) {  // u in (0, 1], normal
  int e;
  double f = frexp_pos_d(u, &e);
  if (f < 0.70710678118654752440) {
    f = __dmul_rn(f, 2.0);
    e -= 1;
  }
  double s = __ddiv_rn(__dsub_rn(f, 1.0), __dadd_rn(f, 1.0));
  double s2 = __dmul_rn(s, s);
  const double inv_odd[13] = {1.0, 1.0 / 3.0, 1.0 / 5.0, 1.0 / 7.0, 1.0 / 9.0,
                              1.0 / 11.0, 1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0,
                              1.0 / 19.0, 1.0 / 21.0, 1.0 / 23.0, 1.0 / 25.0};
  double p = inv_odd[12];
#pragma unroll
  for (int j = 11; j >= 0; j--) p = __dadd_rn(__dmul_rn(p, s2), inv_odd[j]);
  double lf = __dmul_rn(2.0, __dmul_rn(s, p));
  const double ln2_hi = 6.93147180369123816490e-01;
  const double ln2_lo = 1.90821492927058770002e-10;
  double ed = (double)e;
  return __dadd_rn(__dadd_rn(__dmul_rn(ed, ln2_hi), lf), __dmul_rn(ed, ln2_lo));
}

__device__ __forceinline__ void sincos_2pi_d(double u, double* s_out, double* c_out) {
  const double half_pi = 1.57079632679489661923;
  double t4 = __dmul_rn(u, 4.0);
  double qd = floor(t4);
  double r = __dsub_rn(t4, qd);
  int q = (int)qd & 3;
  bool refl = r > 0.5;
  double rr = refl ? __dsub_rn(1.0, r) : r;
  double a = __dmul_rn(rr, half_pi);
  double a2 = __dmul_rn(a, a);
  const double inv_fact[22] = {
      1.0, 1.0, 1.0 / 2.0, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0,
      1.0 / 40320.0, 1.0 / 362880.0, 1.0 / 3628800.0, 1.0 / 39916800.0, 1.0 / 479001600.0,
      1.0 / 6227020800.0, 1.0 / 87178291200.0, 1.0 / 1307674368000.0,
      1.0 / 20922789888000.0, 1.0 / 355687428096000.0, 1.0 / 6402373705728000.0,
      1.0 / 121645100408832000.0, 1.0 / 2432902008176640000.0,
      1.0 / 51090942171709440000.0};
  double ss = 0.0, cc = 0.0;
#pragma unroll
  for (int j = 10; j >= 0; j--) {
    ss = __dadd_rn(__dmul_rn(ss, a2), (j & 1) ? -inv_fact[2 * j + 1] : inv_fact[2 * j + 1]);
    cc = __dadd_rn(__dmul_rn(cc, a2), (j & 1) ? -inv_fact[2 * j] : inv_fact[2 * j]);
  }
  double sn = __dmul_rn(a, ss);
  double cs = cc;
  double s0 = refl ? cs : sn;
  double c0 = refl ? sn : cs;
  switch (q) {
    case 0: *s_out = s0; *c_out = c0; break;
    case 1: *s_out = c0; *c_out = -s0; break;
    case 2: *s_out = -s0; *c_out = -c0; break;
    default: *s_out = -c0; *c_out = s0; break;
  }
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

// ---------------------------- message storage ----------------------------
template <int MSG16>
struct MsgIO;

template <>
struct MsgIO<0> {
  typedef float T;
  static __device__ __forceinline__ float ld(const float* p, int s) { return p[s]; }
  static __device__ __forceinline__ void st(float* p, int s, float v) { p[s] = v; }
  static __device__ __forceinline__ float rt(float v) { return v; }
};

template <>
struct MsgIO<1> {
  typedef __half T;
  static __device__ __forceinline__ float clampv(float v) {
    return v > 65504.0f ? 65504.0f : (v < -65504.0f ? -65504.0f : v);
  }
  static __device__ __forceinline__ float ld(const __half* p, int s) { return __half2float(p[s]); }
  static __device__ __forceinline__ void st(__half* p, int s, float v) {
    p[s] = __float2half_rn(clampv(v));
  }
  static __device__ __forceinline__ float rt(float v) { return __half2float(__float2half_rn(clampv(v))); }
};

}  // namespace gf2c
