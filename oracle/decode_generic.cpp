// CPU oracle: edge-indexed flooding and layered decoders (test infrastructure).
//
// One loop, several check-node rules, written as the numeric specification the
// GPU library follows:
//   algo 0  min-sum as executed by the reference (Llr::boxplus_minsum_n,
//           crates/gf2-coding/src/llr.rs:246-284): sign = parity of (x < 0),
//           magnitude = min |x| over the other edges (NaN-ignoring like f32::min)
//   algo 1  sum-product, FP32 (the semantics of the reference's unused
//           check_node_update_spa + Llr::boxplus_n, core.rs:762-787 and
//           llr.rs:210-215: 2 atanh(prod tanh(x/2)) over the other edges),
//           evaluated with the own_math.h functions, extrinsic product by
//           prefix/suffix products, clamp |P| <= 1 - 2^-23
//   algo 2  sum-product, FP64 (libm tanh/atanh, clamp |P| <= 1 - 2^-50): judge
//   algo 3  normalised + offset min-sum (Llr::boxplus_normalized_minsum_n and
//           boxplus_offset_minsum_n, llr.rs:352-399) with per-(iteration, layer)
//           weights: sign * alpha * max(min - beta, 0)
// Flooding follows LdpcDecoder::decode_iterative (core.rs:889-938) with
// v2c = belief - c2v formed inside the check node (bit-identical to the
// reference's stored v2c).  Layered (no reference counterpart): per row group,
// v2c = APP - c2v_old from the pre-layer APP, APP += (c2v_new - c2v_old), a
// variable with several edges in one layer adding its deltas in ascending
// circulant-shift order.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "oracle_internal.h"
#include "own_math.h"

extern "C" uint16_t or_f32_to_f16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
  int e = (int)(ax >> 23) - 127 + 15;
  uint32_t mant = ax & 0x7fffffu;
  if (e >= 31) return (uint16_t)(sign | 0x7c00u);
  if (e >= 1) {
    uint32_t res = ((uint32_t)e << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (res & 1u))) res++;
    return (uint16_t)(sign | res);  // a carry into the exponent is the correct rounding
  }
  // subnormal half: round((mant | 2^23) * 2^(exp - 126 - 23 + 24)) -> shift
  uint32_t mm = mant | 0x800000u;
  int shift = 14 - e;  // e <= 0 -> shift >= 14
  if (ax == 0) return (uint16_t)sign;
  if (shift > 24) return (uint16_t)sign;
  uint32_t res = mm >> shift;
  uint32_t rem = mm & ((1u << shift) - 1u);
  uint32_t half = 1u << (shift - 1);
  if (rem > half || (rem == half && (res & 1u))) res++;
  return (uint16_t)(sign | res);
}

extern "C" float or_f16_to_f32(uint16_t h) {
  uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1fu;
  uint32_t mant = h & 0x3ffu;
  uint32_t out;
  if (e == 0) {
    if (mant == 0) {
      out = sign;
    } else {  // subnormal: mant * 2^-24
      float v = (float)mant * 5.9604644775390625e-08f;
      std::memcpy(&out, &v, 4);
      out |= sign;
    }
  } else if (e == 31) {
    out = sign | 0x7f800000u | (mant << 13);
  } else {
    out = sign | ((e - 15 + 127) << 23) | (mant << 13);
  }
  float r;
  std::memcpy(&r, &out, 4);
  return r;
}

namespace {

template <class Real>
struct Store32 {
  typedef Real T;
  static T st(Real x) { return x; }
  static Real ld(T x) { return x; }
};

struct Store16 {
  typedef uint16_t T;
  static T st(float x) {
    const float lim = 65504.0f;
    if (x > lim) x = lim;
    if (x < -lim) x = -lim;
    return or_f32_to_f16(x);
  }
  static float ld(T h) { return or_f16_to_f32(h); }
};

struct Params {
  int algo;
  const float* alpha;
  const float* beta;
  int n_wt_iters;
  int L;
};

// Check-node rule: x[0..d) -> out[0..d)
template <class Real>
void check_node(const Params& P, int it, int layer, const Real* x, Real* out, int d,
                std::vector<Real>& scratch) {
  if (d == 1) {
    out[0] = (Real)0;
    return;
  }
  if (P.algo == 0 || P.algo == 3) {
    Real m1 = (Real)INFINITY, m2 = (Real)INFINITY;
    int i1 = -1;
    int neg = 0;
    for (int j = 0; j < d; j++) {
      Real a = std::fabs(x[j]);
      if (a < m1) {
        m2 = m1;
        m1 = a;
        i1 = j;
      } else if (a < m2) {
        m2 = a;
      }
      neg ^= (x[j] < (Real)0) ? 1 : 0;
    }
    float al = 1.0f, be = 0.0f;
    if (P.algo == 3) {
      int t = it < P.n_wt_iters ? it : P.n_wt_iters - 1;
      al = P.alpha[t * P.L + layer];
      be = P.beta[t * P.L + layer];
    }
    for (int j = 0; j < d; j++) {
      Real mag = (j == i1) ? m2 : m1;
      if (P.algo == 3) {
        Real dd = mag - (Real)be;
        dd = dd > (Real)0 ? dd : (Real)0;
        mag = (Real)al * dd;
      }
      int s = neg ^ ((x[j] < (Real)0) ? 1 : 0);
      out[j] = s ? -mag : mag;
    }
    return;
  }
  // sum-product: extrinsic tanh products by prefix/suffix products
  scratch.resize(3 * (size_t)d);
  Real* t = scratch.data();
  Real* pre = t + d;
  Real* suf = pre + d;
  for (int j = 0; j < d; j++) {
    if (P.algo == 1) t[j] = (Real)ownm::tanh_half_f((float)x[j]);
    else t[j] = (Real)std::tanh((double)x[j] / 2.0);
  }
  pre[0] = t[0];
  for (int j = 1; j < d; j++) pre[j] = pre[j - 1] * t[j];
  suf[d - 1] = t[d - 1];
  for (int j = d - 2; j >= 0; j--) suf[j] = t[j] * suf[j + 1];
  const Real pmax = (P.algo == 1) ? (Real)ownm::kSpaPMax : (Real)(1.0 - std::ldexp(1.0, -50));
  for (int j = 0; j < d; j++) {
    Real p;
    if (j == 0) p = suf[1];
    else if (j == d - 1) p = pre[d - 2];
    else p = pre[j - 1] * suf[j + 1];
    if (p > pmax) p = pmax;
    if (p < -pmax) p = -pmax;
    if (P.algo == 1) out[j] = (Real)ownm::two_atanh_f((float)p);
    else out[j] = (Real)(2.0 * std::atanh((double)p));
  }
}

template <class Real, class S>
void decode_frame(const or_code* c, const Params& P, int sched, const float* llr, int max_iter,
                  uint8_t* msg, int32_t* iters, uint8_t* conv, uint8_t* synd_ok, Real* beliefs_out,
                  const std::vector<std::vector<int64_t>>& layer_checks,
                  const std::vector<std::vector<int64_t>>& layer_edges_by_key) {
  const int64_t n = c->n, m = c->m, E = (int64_t)c->row_idx.size();
  std::vector<Real> belief(n, (Real)0);
  std::vector<uint8_t> hard(n, 0);
  auto syndrome_zero = [&]() {
    for (int64_t v = 0; v < n; v++) hard[v] = belief[v] < (Real)0 ? 1 : 0;
    for (int64_t r = 0; r < m; r++) {
      uint8_t acc = 0;
      for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) acc ^= hard[c->row_idx[e]];
      if (acc) return false;
    }
    return true;
  };
  int iterations = 0;
  bool converged = false;
  if (max_iter > 0) {
    std::vector<typename S::T> c2v(E, S::st((Real)0));
    for (int64_t v = 0; v < n; v++) belief[v] = (Real)llr[v];
    std::vector<Real> x, out, scratch;
    std::vector<Real> newv(E);
    for (int it = 0; it < max_iter; it++) {
      iterations = it + 1;
      if (sched == 0) {
        for (int64_t r = 0; r < m; r++) {
          int64_t b = c->row_ptr[r];
          int d = (int)(c->row_ptr[r + 1] - b);
          if (d == 0) continue;
          x.resize(d);
          out.resize(d);
          const int32_t* so = &c->slot_order[b];
          for (int j = 0; j < d; j++) x[j] = belief[c->row_idx[b + so[j]]] - (Real)S::ld(c2v[b + so[j]]);
          int layer = c->layers ? c->check_layer[r] : 0;
          check_node<Real>(P, it, layer, x.data(), out.data(), d, scratch);
          for (int j = 0; j < d; j++) c2v[b + so[j]] = S::st(out[j]);
        }
        for (int64_t v = 0; v < n; v++) {
          Real acc = (Real)llr[v];
          for (int64_t s = c->col_ptr[v]; s < c->col_ptr[v + 1]; s++)
            acc = acc + (Real)S::ld(c2v[c->col_edge[s]]);
          belief[v] = acc;
        }
      } else {
        for (int l = 0; l < (int)layer_checks.size(); l++) {
          for (int64_t r : layer_checks[l]) {
            int64_t b = c->row_ptr[r];
            int d = (int)(c->row_ptr[r + 1] - b);
            if (d == 0) continue;
            x.resize(d);
            out.resize(d);
            const int32_t* so = &c->slot_order[b];
            for (int j = 0; j < d; j++) x[j] = belief[c->row_idx[b + so[j]]] - (Real)S::ld(c2v[b + so[j]]);
            check_node<Real>(P, it, l, x.data(), out.data(), d, scratch);
            for (int j = 0; j < d; j++) newv[b + so[j]] = out[j];
          }
          for (int64_t e : layer_edges_by_key[l]) {
            typename S::T stn = S::st(newv[e]);
            Real delta = (Real)S::ld(stn) - (Real)S::ld(c2v[e]);
            int64_t v = c->row_idx[e];
            belief[v] = belief[v] + delta;
            c2v[e] = stn;
          }
        }
      }
      if (syndrome_zero()) {
        converged = true;
        break;
      }
    }
  }
  bool passed = syndrome_zero();
  if (msg)
    for (int64_t i = 0; i < c->k; i++) msg[i] = hard[i];
  if (iters) *iters = iterations;
  if (conv) *conv = converged;
  if (synd_ok) *synd_ok = passed;
  if (beliefs_out)
    for (int64_t v = 0; v < n; v++) beliefs_out[v] = belief[v];
}

void build_layers(const or_code* c, std::vector<std::vector<int64_t>>& lc,
                  std::vector<std::vector<int64_t>>& le) {
  lc.assign(c->layers, {});
  le.assign(c->layers, {});
  for (int64_t r = 0; r < c->m; r++) lc[c->check_layer[r]].push_back(r);
  for (int l = 0; l < c->layers; l++) {
    std::vector<int64_t>& v = le[l];
    for (int64_t r : lc[l])
      for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) v.push_back(e);
    std::stable_sort(v.begin(), v.end(),
                     [&](int64_t a, int64_t b) { return c->edge_key[a] < c->edge_key[b]; });
  }
}

template <class Real, class S>
int run(const or_code* c, const Params& P, int sched, const float* llr, int64_t frames,
        int max_iter, int threads, uint8_t* msg, int32_t* iters, uint8_t* conv,
        uint8_t* synd_ok, Real* beliefs) {
  std::vector<std::vector<int64_t>> lc, le;
  if (sched == 1) build_layers(c, lc, le);
  or_parallel_frames(frames, threads, [&](int64_t f) {
    decode_frame<Real, S>(c, P, sched, llr + f * c->n, max_iter, msg ? msg + f * c->k : nullptr,
                          iters ? iters + f : nullptr, conv ? conv + f : nullptr,
                          synd_ok ? synd_ok + f : nullptr, beliefs ? beliefs + f * c->n : nullptr,
                          lc, le);
  });
  return 0;
}

}  // namespace

extern "C" int or_decode(const or_code* c, const float* llr, int64_t frames, int max_iter, int algo,
                         int sched, int msg16, const float* alpha, const float* beta,
                         int n_wt_iters, int threads, uint8_t* msg, int32_t* iters, uint8_t* conv,
                         uint8_t* synd_ok, float* beliefs) {
  if (!c || frames < 0 || max_iter < 0 || algo < 0 || algo > 3 || sched < 0 || sched > 1) {
    or_set_error("invalid arguments");
    return -1;
  }
  if (sched == 1 && c->layers == 0) {
    or_set_error("layered schedule needs a QC / DVB-T2 code");
    return -1;
  }
  if (algo == 3 && (!alpha || !beta || n_wt_iters <= 0)) {
    or_set_error("algo 3 needs weights");
    return -1;
  }
  Params P{algo, alpha, beta, n_wt_iters, c->layers ? c->layers : 1};
  if (algo == 2) {
    std::vector<double> b64(beliefs ? (size_t)(frames * c->n) : 0);
    run<double, Store32<double>>(c, P, sched, llr, frames, max_iter, threads, msg, iters, conv,
                                 synd_ok, beliefs ? b64.data() : nullptr);
    if (beliefs)
      for (size_t i = 0; i < b64.size(); i++) beliefs[i] = (float)b64[i];
    return 0;
  }
  if (msg16)
    return run<float, Store16>(c, P, sched, llr, frames, max_iter, threads, msg, iters, conv,
                               synd_ok, beliefs);
  return run<float, Store32<float>>(c, P, sched, llr, frames, max_iter, threads, msg, iters, conv,
                                    synd_ok, beliefs);
}

extern "C" int or_decode_spa64(const or_code* c, const float* llr, int64_t frames, int max_iter,
                               int sched, int threads, uint8_t* msg, int32_t* iters, uint8_t* conv,
                               uint8_t* synd_ok, double* beliefs) {
  if (!c || frames < 0 || max_iter < 0 || (sched == 1 && c->layers == 0)) {
    or_set_error("invalid arguments");
    return -1;
  }
  Params P{2, nullptr, nullptr, 0, c->layers ? c->layers : 1};
  return run<double, Store32<double>>(c, P, sched, llr, frames, max_iter, threads, msg, iters,
                                      conv, synd_ok, beliefs);
}
