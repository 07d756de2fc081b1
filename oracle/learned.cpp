// CPU oracle: learned normalised/offset min-sum, forward and backward in FP64
// (test infrastructure: the gradient judge of the GPU training kernels).
//
// The check-node rule is the reference's normalised and offset min-sum
// (Llr::boxplus_normalized_minsum_n / boxplus_offset_minsum_n,
// crates/gf2-coding/src/llr.rs:352-399) combined, with one (alpha, beta) pair
// per unrolled iteration t and per row group l:
//     c_e = s_e * alpha[t,l] * max(m_e - beta[t,l], 0)
//     m_e = min over the other edges j of |x_j|,  s_e = prod over the others of sgn(x_j)
// with the flooding schedule of LdpcDecoder::decode_iterative (core.rs:889-938):
//     x^0 = llr, b^t = llr + sum c^t, x^{t+1}_e = b^t[v_e] - c^t_e.
// Loss: mean over frames and all n codeword bits of softplus(-(1 - 2 c_v) b^{T-1}_v),
// the binary cross-entropy of sigmoid(b) against the transmitted bit.
// Subgradients: the min routes to the first index attaining it among the
// others; d|x|/dx = -1 if x < 0 else +1; d max(u,0)/du = [u > 0].
#include <cmath>
#include <cstring>

#include "oracle_internal.h"

extern "C" double or_nms_loss_grad(const or_code* c, const float* llr, const uint8_t* cw,
                                   int64_t frames, int T, const double* alpha, const double* beta,
                                   double* grad_alpha, double* grad_beta, double* out_llr) {
  const int64_t n = c->n, m = c->m, E = (int64_t)c->row_idx.size();
  const int L = c->layers ? c->layers : 1;
  std::vector<double> ga(T * L, 0.0), gbeta(T * L, 0.0);
  double loss = 0.0;
  const double scale = 1.0 / ((double)frames * (double)n);
  for (int64_t f = 0; f < frames; f++) {
    const float* lf = llr + f * n;
    std::vector<std::vector<double>> X(T, std::vector<double>(E));
    std::vector<std::vector<double>> Cm(T, std::vector<double>(E));
    std::vector<double> b(n);
    std::vector<double> x(E);
    for (int64_t e = 0; e < E; e++) x[e] = lf[c->row_idx[e]];
    for (int t = 0; t < T; t++) {
      X[t] = x;
      for (int64_t r = 0; r < m; r++) {
        int l = c->layers ? c->check_layer[r] : 0;
        double al = alpha[t * L + l], be = beta[t * L + l];
        int64_t e0 = c->row_ptr[r], e1 = c->row_ptr[r + 1];
        for (int64_t e = e0; e < e1; e++) {
          double mn = INFINITY;
          int neg = 0;
          for (int64_t j = e0; j < e1; j++) {
            if (j == e) continue;
            double a = std::fabs(x[j]);
            if (a < mn) mn = a;
            neg ^= x[j] < 0 ? 1 : 0;
          }
          if (e1 - e0 == 1) mn = 0.0;
          double mag = al * std::max(mn - be, 0.0);
          Cm[t][e] = neg ? -mag : mag;
        }
      }
      for (int64_t v = 0; v < n; v++) {
        double acc = lf[v];
        for (int64_t s = c->col_ptr[v]; s < c->col_ptr[v + 1]; s++) acc += Cm[t][c->col_edge[s]];
        b[v] = acc;
      }
      for (int64_t e = 0; e < E; e++) x[e] = b[c->row_idx[e]] - Cm[t][e];
    }
    // loss and dL/db^{T-1}
    std::vector<double> gb(n), gc(E, 0.0), gx(E);
    for (int64_t v = 0; v < n; v++) {
      double sv = cw[f * n + v] ? -1.0 : 1.0;
      double z = -sv * b[v];
      double sp = z > 0 ? z + std::log1p(std::exp(-z)) : std::log1p(std::exp(z));
      loss += sp * scale;
      double sig = 1.0 / (1.0 + std::exp(-z));
      gb[v] = scale * sig * (-sv);
      if (out_llr) out_llr[f * n + v] = b[v];
    }
    for (int t = T - 1; t >= 0; t--) {
      // b^t = llr + sum c^t  ->  gc += gb[v_e]
      for (int64_t e = 0; e < E; e++) gc[e] += gb[c->row_idx[e]];
      std::fill(gx.begin(), gx.end(), 0.0);
      const std::vector<double>& xt = X[t];
      for (int64_t r = 0; r < m; r++) {
        int l = c->layers ? c->check_layer[r] : 0;
        double al = alpha[t * L + l], be = beta[t * L + l];
        int64_t e0 = c->row_ptr[r], e1 = c->row_ptr[r + 1];
        if (e1 - e0 == 1) continue;
        for (int64_t e = e0; e < e1; e++) {
          double mn = INFINITY;
          int64_t arg = -1;
          int neg = 0;
          for (int64_t j = e0; j < e1; j++) {
            if (j == e) continue;
            double a = std::fabs(xt[j]);
            if (a < mn) {
              mn = a;
              arg = j;
            }
            neg ^= xt[j] < 0 ? 1 : 0;
          }
          double s = neg ? -1.0 : 1.0;
          double u = mn - be;
          bool act = u > 0;
          ga[t * L + l] += gc[e] * s * (act ? u : 0.0);
          if (act) {
            gbeta[t * L + l] += -gc[e] * s * al;
            double gm = gc[e] * s * al;
            gx[arg] += gm * (xt[arg] < 0 ? -1.0 : 1.0);
          }
        }
      }
      if (t == 0) break;
      // x^t = b^{t-1}[v_e] - c^{t-1}_e
      std::fill(gb.begin(), gb.end(), 0.0);
      for (int64_t e = 0; e < E; e++) {
        gb[c->row_idx[e]] += gx[e];
        gc[e] = -gx[e];
      }
    }
  }
  if (grad_alpha) std::memcpy(grad_alpha, ga.data(), sizeof(double) * ga.size());
  if (grad_beta) std::memcpy(grad_beta, gbeta.data(), sizeof(double) * gbeta.size());
  return loss;
}

// Layered schedule (row groups of the QC structure in order; no reference
// counterpart -- the reference decoder is flooding only):
//     per row group l of iteration t, for its edges e:
//       x_e = A[v_e] - c_e        (A = the posterior before the row group, c_e = the
//                                  edge's message of iteration t-1, 0 at t = 0)
//       c'_e = s_e * alpha[t,l] * max(m_e - beta[t,l], 0)
//       A[v] += sum over the row group's edges of v of (c'_e - c_e)
// Loss as above on the posterior after T iterations.  Backward, row groups in
// reverse order with G = dL/dA after the row group and P_e = dL/dc'_e from
// iteration t+1:
//       dL/dc'_e = G[v_e] + P_e  -> check-node backward -> dL/dx_e
//       P_e <- -G[v_e] - dL/dx_e  (the gradient on c_e, used by iteration t-1)
//       G[v_e] += dL/dx_e         (the gradient on A before the row group)
extern "C" double or_nms_layered_loss_grad(const or_code* c, const float* llr, const uint8_t* cw,
                                           int64_t frames, int T, const double* alpha,
                                           const double* beta, double* grad_alpha, double* grad_beta,
                                           double* out_llr) {
  if (!c || c->layers == 0) {
    or_set_error("layered schedule needs a QC / DVB-T2 code");
    return NAN;
  }
  const int64_t n = c->n, m = c->m, E = (int64_t)c->row_idx.size();
  const int L = c->layers;
  std::vector<std::vector<int64_t>> lc(L);
  for (int64_t r = 0; r < m; r++) lc[c->check_layer[r]].push_back(r);
  std::vector<double> ga(T * L, 0.0), gbeta(T * L, 0.0);
  double loss = 0.0;
  const double scale = 1.0 / ((double)frames * (double)n);
  // extrinsic min / sign of edge e of row [e0, e1) over x: (mn, arg, sign)
  auto extrinsic = [](const std::vector<double>& x, int64_t e0, int64_t e1, int64_t e, double& mn,
                      int64_t& arg, double& s) {
    mn = INFINITY;
    arg = -1;
    int neg = 0;
    for (int64_t j = e0; j < e1; j++) {
      if (j == e) continue;
      double a = std::fabs(x[j]);
      if (a < mn) {
        mn = a;
        arg = j;
      }
      neg ^= x[j] < 0 ? 1 : 0;
    }
    if (e1 - e0 == 1) mn = 0.0;
    s = neg ? -1.0 : 1.0;
  };
  for (int64_t f = 0; f < frames; f++) {
    const float* lf = llr + f * n;
    std::vector<std::vector<double>> X(T, std::vector<double>(E, 0.0));
    std::vector<double> A(n), C(E, 0.0), Cn(E, 0.0);
    for (int64_t v = 0; v < n; v++) A[v] = lf[v];
    for (int t = 0; t < T; t++) {
      std::vector<double>& x = X[t];
      for (int l = 0; l < L; l++) {
        const double al = alpha[t * L + l], be = beta[t * L + l];
        for (int64_t r : lc[l])
          for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) x[e] = A[c->row_idx[e]] - C[e];
        for (int64_t r : lc[l]) {
          const int64_t e0 = c->row_ptr[r], e1 = c->row_ptr[r + 1];
          for (int64_t e = e0; e < e1; e++) {
            double mn, s;
            int64_t arg;
            extrinsic(x, e0, e1, e, mn, arg, s);
            Cn[e] = s * al * std::max(mn - be, 0.0);
          }
        }
        for (int64_t r : lc[l])
          for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) {
            A[c->row_idx[e]] += Cn[e] - C[e];
            C[e] = Cn[e];
          }
      }
    }
    std::vector<double> G(n), P(E, 0.0), dx(E, 0.0);
    for (int64_t v = 0; v < n; v++) {
      double sv = cw[f * n + v] ? -1.0 : 1.0;
      double z = -sv * A[v];
      double sp = z > 0 ? z + std::log1p(std::exp(-z)) : std::log1p(std::exp(z));
      loss += sp * scale;
      double sig = 1.0 / (1.0 + std::exp(-z));
      G[v] = scale * sig * (-sv);
      if (out_llr) out_llr[f * n + v] = A[v];
    }
    for (int t = T - 1; t >= 0; t--) {
      const std::vector<double>& x = X[t];
      for (int l = L - 1; l >= 0; l--) {
        const double al = alpha[t * L + l], be = beta[t * L + l];
        for (int64_t r : lc[l])
          for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) dx[e] = 0.0;
        for (int64_t r : lc[l]) {
          const int64_t e0 = c->row_ptr[r], e1 = c->row_ptr[r + 1];
          if (e1 - e0 == 1) continue;
          for (int64_t e = e0; e < e1; e++) {
            const double gc = G[c->row_idx[e]] + P[e];
            double mn, s;
            int64_t arg;
            extrinsic(x, e0, e1, e, mn, arg, s);
            const double u = mn - be;
            if (u > 0) {
              ga[t * L + l] += gc * s * u;
              gbeta[t * L + l] += -gc * s * al;
              dx[arg] += gc * s * al * (x[arg] < 0 ? -1.0 : 1.0);
            }
          }
        }
        for (int64_t r : lc[l])
          for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) P[e] = -G[c->row_idx[e]] - dx[e];
        for (int64_t r : lc[l])
          for (int64_t e = c->row_ptr[r]; e < c->row_ptr[r + 1]; e++) G[c->row_idx[e]] += dx[e];
      }
    }
  }
  if (grad_alpha) std::memcpy(grad_alpha, ga.data(), sizeof(double) * ga.size());
  if (grad_beta) std::memcpy(grad_beta, gbeta.data(), sizeof(double) * gbeta.size());
  return loss;
}
