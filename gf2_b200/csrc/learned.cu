// gf2cuda learned normalised / offset min-sum: training kernels (sm_100a).
//
// Check-node rule (the reference's Llr::boxplus_normalized_minsum_n and
// Llr::boxplus_offset_minsum_n, crates/gf2-coding/src/llr.rs:352-399, combined,
// with one (alpha, beta) pair per unrolled iteration t and row group l):
//     c_e = s_e * alpha[t,l] * max(m_e - beta[t,l], 0)
//     m_e = min_{j != e} |x_j|,  s_e = prod_{j != e} sgn(x_j)
// Flooding schedule of LdpcDecoder::decode_iterative (ldpc/core.rs:889-938):
//     x^0 = llr, b^t = llr + sum_e c^t_e, x^{t+1}_e = b^t[v_e] - c^t_e.
// Loss: mean over frames and the n codeword bits of softplus(-(1 - 2 c_v) b^{T-1}_v).
//
// nms_forward_kernel: one CTA per frame, T iterations without early stop,
//   saving x^t of every edge slot (the only activations the backward needs).
// nms_backward_kernel: one CTA per frame, t = T-1 .. 0.  The min routes the
//   gradient to the first index attaining it among the other edges, so inside
//   a check only the two smallest-magnitude slots receive gradient; d|x|/dx =
//   -1 if x < 0 else +1; d max(u, 0)/du = [u > 0].
// Reductions are deterministic (no floating-point atomics): each check
// writes its weight-gradient terms to the CTA workspace, one warp per row
// group sums them in a fixed order, each frame's gradients and loss go to its
// own row of a per-frame buffer, and nms_reduce_kernel sums the frames in
// order.  Training is therefore bit-reproducible.
// adam_kernel: Adam (Kingma & Ba 2015) with bias correction.
#include <algorithm>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

static constexpr int kLearnThreads = 512;
static constexpr int kLearnDcMax = 32;

struct LearnCtx {
  int n, m, ncg, vgs, L;
  const int4* cg;
  const int* slot_var;
  const uint16_t* chk_cg;
  const int2* vg;
  const int* vg_slot;
};

__device__ __forceinline__ LearnCtx make_ctx(const DevCode& C, int L) {
  return LearnCtx{C.n, C.m, C.ncg, C.vgs, L, C.cg, C.slot_var, C.chk_cg, C.vg, C.vg_slot};
}

// Sum over a warp in a fixed order (butterfly), every lane gets the total.
__device__ __forceinline__ float warp_sum_fixed(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = __fadd_rn(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// belief[v] = llr[v] + sum_e c2v[e] (ascending original check index)
__device__ __forceinline__ float var_sum(const LearnCtx& F, int v, float base, const float* __restrict__ msg) {
  const int h = v / F.vgs, j = v - h * F.vgs;
  const int2 V = F.vg[h];
  const int* sl = F.vg_slot + V.y + j;
  float b = base;
  for (int i = 0; i < V.x; i++) {
    const int s = __ldg(&sl[i * F.vgs]);
    if (s < 0) break;
    b = __fadd_rn(b, msg[s]);
  }
  return b;
}

__global__ void __launch_bounds__(kLearnThreads) nms_forward_kernel(
    const DevCode* __restrict__ Cp, int T, int L, const float* __restrict__ llr, const uint64_t* __restrict__ cw,
    long long frames, const float* __restrict__ alpha, const float* __restrict__ beta, float* __restrict__ X,
    float* __restrict__ Bout, char* __restrict__ work, long long work_stride, float* __restrict__ pf) {
  __shared__ float s_part[kLearnThreads / 32];
  const DevCode C = *Cp;
  const LearnCtx F = make_ctx(C, L);
  const int n = F.n, E = C.e_slots;
  float* c2v = (float*)(work + (long long)blockIdx.x * work_stride);
  float* app = c2v + ((E + 63) & ~63);
  const float scale = 1.0f / ((float)frames * (float)n);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const float* lf = llr + f * (long long)n;
    for (int v = threadIdx.x; v < n; v += blockDim.x) app[v] = lf[v];
    __syncthreads();
    for (int t = 0; t < T; t++) {
      float* Xt = X + (f * T + t) * (long long)E;
      for (int cc = threadIdx.x; cc < F.m; cc += blockDim.x) {
        const int g = F.chk_cg[cc];
        const int4 G = F.cg[g];
        const int tt = cc - G.x, d = G.z, s0 = G.w + tt;
        const int lay = (L == F.ncg) ? g : 0;
        const float al = __ldg(&alpha[t * L + lay]), be = __ldg(&beta[t * L + lay]);
        float m1 = __int_as_float(0x7f800000), m2 = m1;
        int i1 = -1, nreal = 0;
        uint32_t neg = 0;
        for (int i = 0; i < d; i++) {
          const int s = s0 + i * G.y;
          const int v = __ldg(&F.slot_var[s]);
          if (v < 0) continue;
          const float x = (t == 0) ? app[v] : __fsub_rn(app[v], c2v[s]);
          Xt[s] = x;
          const float ax = fabsf(x);
          if (ax < m1) {
            m2 = m1;
            m1 = ax;
            i1 = i;
          } else if (ax < m2) {
            m2 = ax;
          }
          neg ^= (x < 0.0f) ? 1u : 0u;
          nreal++;
        }
        for (int i = 0; i < d; i++) {
          const int s = s0 + i * G.y;
          const int v = __ldg(&F.slot_var[s]);
          if (v < 0) continue;
          const float x = Xt[s];
          float mag = (nreal == 1) ? 0.0f : ((i == i1) ? m2 : m1);
          const float u = __fsub_rn(mag, be);
          mag = __fmul_rn(al, u > 0.0f ? u : 0.0f);
          const uint32_t sg = neg ^ ((x < 0.0f) ? 1u : 0u);
          c2v[s] = sg ? -mag : mag;
        }
      }
      __syncthreads();
      for (int v = threadIdx.x; v < n; v += blockDim.x) app[v] = var_sum(F, v, lf[v], c2v);
      __syncthreads();
    }
    // loss and final soft output
    float part = 0.0f;
    const uint64_t* cf = cw + f * (long long)C.words_n;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
      const float b = app[v];
      Bout[f * (long long)n + v] = b;
      const float s = ((cf[v >> 6] >> (v & 63)) & 1ull) ? -1.0f : 1.0f;
      const float z = -s * b;
      part += (z > 0.0f ? z + log1pf(expf(-z)) : log1pf(expf(z))) * scale;
    }
    part = warp_sum_fixed(part);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      float sum = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum = __fadd_rn(sum, s_part[w]);
      pf[f * (2LL * T * L + 1) + 2 * T * L] = sum;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kLearnThreads) nms_backward_kernel(
    const DevCode* __restrict__ Cp, int T, int L, const float* __restrict__ llr, const uint64_t* __restrict__ cw,
    long long frames, const float* __restrict__ alpha, const float* __restrict__ beta,
    const float* __restrict__ X, const float* __restrict__ Bin, char* __restrict__ work, long long work_stride,
    float* __restrict__ pf) {
  const DevCode C = *Cp;
  const LearnCtx F = make_ctx(C, L);
  const int n = F.n, E = C.e_slots;
  float* gx = (float*)(work + (long long)blockIdx.x * work_stride);
  float* gb = gx + ((E + 63) & ~63);
  float* gchk = gb + ((n + 63) & ~63);  // [2][m]: per-check alpha / beta gradient terms
  const float scale = 1.0f / ((float)frames * (float)n);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const uint64_t* cf = cw + f * (long long)C.words_n;
    // dL/db^{T-1}
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
      const float b = Bin[f * (long long)n + v];
      const float s = ((cf[v >> 6] >> (v & 63)) & 1ull) ? -1.0f : 1.0f;
      const float z = -s * b;
      const float sig = 1.0f / (1.0f + expf(-z));
      gb[v] = scale * sig * (-s);
    }
    __syncthreads();
    for (int t = T - 1; t >= 0; t--) {
      const float* Xt = X + (f * T + t) * (long long)E;
      for (int cc = threadIdx.x; cc < F.m; cc += blockDim.x) {
        const int g = F.chk_cg[cc];
        const int4 G = F.cg[g];
        const int tt = cc - G.x, d = G.z, s0 = G.w + tt;
        const int lay = (L == F.ncg) ? g : 0;
        const float al = __ldg(&alpha[t * L + lay]), be = __ldg(&beta[t * L + lay]);
        float m1 = __int_as_float(0x7f800000), m2 = m1;
        int i1 = -1, i2 = -1, nreal = 0;
        uint32_t neg = 0;
        float gcv[kLearnDcMax];
        for (int i = 0; i < d; i++) {
          const int s = s0 + i * G.y;
          const int v = __ldg(&F.slot_var[s]);
          gcv[i] = 0.0f;
          if (v < 0) continue;
          // gradient reaching c^t_e: from b^t (gb) and, for t < T-1, from x^{t+1}_e = b^t - c^t (-gx)
          gcv[i] = (t == T - 1) ? gb[v] : __fsub_rn(gb[v], gx[s]);
          const float x = Xt[s];
          const float ax = fabsf(x);
          if (ax < m1) {
            m2 = m1;
            i2 = i1;
            m1 = ax;
            i1 = i;
          } else if (ax < m2) {
            m2 = ax;
            i2 = i;
          }
          neg ^= (x < 0.0f) ? 1u : 0u;
          nreal++;
        }
        float gA = 0.0f, gB = 0.0f, g1 = 0.0f, g2 = 0.0f;
        if (nreal > 1) {
          for (int i = 0; i < d; i++) {
            const int s = s0 + i * G.y;
            if (__ldg(&F.slot_var[s]) < 0) continue;
            const float x = Xt[s];
            const float sg = ((neg ^ ((x < 0.0f) ? 1u : 0u)) ? -1.0f : 1.0f);
            const float mag = (i == i1) ? m2 : m1;
            const float u = mag - be;
            if (u > 0.0f) {
              gA += gcv[i] * sg * u;
              gB -= gcv[i] * sg * al;
              const float gm = gcv[i] * sg * al;
              if (i == i1) g2 += gm;  // min over the others is slot i2
              else g1 += gm;          // min over the others is slot i1
            }
          }
        }
        // gx for this check's slots: only i1 and i2 are nonzero
        for (int i = 0; i < d; i++) {
          const int s = s0 + i * G.y;
          float gxi = 0.0f;
          if (i == i1) gxi = g1 * (Xt[s] < 0.0f ? -1.0f : 1.0f);
          else if (i == i2) gxi = g2 * (Xt[s] < 0.0f ? -1.0f : 1.0f);
          gx[s] = gxi;
        }
        gchk[cc] = gA;
        gchk[F.m + cc] = gB;
      }
      __syncthreads();
      // per row group sums in a fixed order: warp w takes layers w, w + nwarps, ...
      for (int lay = threadIdx.x >> 5; lay < L; lay += blockDim.x >> 5) {
        const int c0 = (L == F.ncg) ? F.cg[lay].x : 0, c1 = (L == F.ncg) ? c0 + F.cg[lay].y : F.m;
        float sa = 0.0f, sb = 0.0f;
        for (int cc = c0 + (threadIdx.x & 31); cc < c1; cc += 32) {
          sa = __fadd_rn(sa, gchk[cc]);
          sb = __fadd_rn(sb, gchk[F.m + cc]);
        }
        sa = warp_sum_fixed(sa);
        sb = warp_sum_fixed(sb);
        if ((threadIdx.x & 31) == 0) {
          float* row = pf + f * (2LL * T * L + 1);
          row[t * L + lay] = sa;
          row[T * L + t * L + lay] = sb;
        }
      }
      if (t > 0)
        for (int v = threadIdx.x; v < n; v += blockDim.x) gb[v] = var_sum(F, v, 0.0f, gx);  // dL/db^{t-1}
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Layered schedule (no reference counterpart; the reference decoder floods).
// Row groups g = 0 .. ncg-1 of iteration t, each check t' of g:
//     x_e = A[v_e] - c_e,  c'_e = s_e * alpha[t,g] * max(m_e - beta[t,g], 0),
//     A[v_e] += c'_e - c_e
// with v2c formed from the posterior before the row group and the deltas of a
// variable with several edges in one row group added in slot order (ascending
// circulant shift) -- the arithmetic and the order of the layered inference
// kernel (bp_layered_kernel, GF2C_ALGO_NMS, FP32 messages), so the training
// forward and the inference decoder give the same posteriors bit for bit.
// Backward, row groups in reverse order, with G = dL/dA after the row group and
// P_e = dL/dc'_e from iteration t+1:
//     dL/dc'_e = G[v_e] + P_e -> check-node backward (min routed to the first
//     index attaining it) -> dL/dx_e;  P_e <- -G[v_e] - dL/dx_e;  G[v_e] += dL/dx_e
// One CTA per frame, one thread per check of a row group (blockDim >= the
// largest row group).  Weight gradients: per-check terms in shared memory,
// summed per row group by warp 0 in a fixed order -- deterministic.
// ---------------------------------------------------------------------------
static constexpr int kLayThreadsMax = 1024;

__global__ void __launch_bounds__(kLayThreadsMax) nms_layered_forward_kernel(
    const DevCode* __restrict__ Cp, int T, int L, const float* __restrict__ llr, const uint64_t* __restrict__ cw,
    long long frames, const float* __restrict__ alpha, const float* __restrict__ beta, float* __restrict__ X,
    float* __restrict__ Bout, char* __restrict__ work, long long work_stride, float* __restrict__ pf) {
  __shared__ float s_part[kLayThreadsMax / 32];
  const DevCode& C = *Cp;
  const int n = C.n, E = C.e_slots, ncg = C.ncg, tid = threadIdx.x;
  const int* __restrict__ slot_var = C.slot_var;
  float* c2v = (float*)(work + (long long)blockIdx.x * work_stride);
  float* app = c2v + ((E + 63) & ~63);
  const float scale = 1.0f / ((float)frames * (float)n);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const float* lf = llr + f * (long long)n;
    for (int v = tid; v < n; v += blockDim.x) app[v] = lf[v];
    __syncthreads();
    for (int t = 0; t < T; t++) {
      float* Xt = X + (f * T + t) * (long long)E;
      for (int g = 0; g < ncg; g++) {
        const int4 G = C.cg[g];
        const uint32_t sync = C.cg_sync[g];
        const int nchk = G.y, d = G.z;
        const bool act = tid < nchk;
        const int lay = (L == ncg) ? g : 0;
        const float al = __ldg(&alpha[t * L + lay]), be = __ldg(&beta[t * L + lay]);
        int vv[kLearnDcMax];
        float dl[kLearnDcMax];
        if (act) {
          float ap[kLearnDcMax], o[kLearnDcMax];
          float m1 = __int_as_float(0x7f800000), m2 = m1;
          int i1 = -1, nreal = 0;
          uint32_t neg = 0, negall = 0;
          for (int i = 0; i < d; i++) {
            const int s = G.w + i * nchk + tid;
            const int v = __ldg(&slot_var[s]);
            vv[i] = v;
            if (v < 0) continue;
            ap[i] = app[v];
            o[i] = (t == 0) ? 0.0f : c2v[s];
            const float x = __fsub_rn(ap[i], o[i]);
            Xt[s] = x;
            const float ax = fabsf(x);
            if (ax < m1) {
              m2 = m1;
              m1 = ax;
              i1 = i;
            } else if (ax < m2) {
              m2 = ax;
            }
            const uint32_t ng = (x < 0.0f) ? 1u : 0u;
            neg |= ng << i;
            negall ^= ng;
            nreal++;
          }
          float mag1 = (nreal == 1) ? 0.0f : m1, mag2 = (nreal == 1) ? 0.0f : m2;
          const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
          mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
          mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
          for (int i = 0; i < d; i++) {
            if (vv[i] < 0) continue;
            const int s = G.w + i * nchk + tid;
            const float mag = (i == i1) ? mag2 : mag1;
            const float out = (negall ^ ((neg >> i) & 1u)) ? -mag : mag;
            c2v[s] = out;
            dl[i] = __fsub_rn(out, o[i]);
            if (sync == 0) app[vv[i]] = __fadd_rn(ap[i], dl[i]);
          }
        }
        if (sync != 0) {
          __syncthreads();  // every pre-row-group posterior read
          for (int i = 0; i < d; i++) {
            if (act && vv[i] >= 0) app[vv[i]] = __fadd_rn(app[vv[i]], dl[i]);
            if ((sync >> i) & 1u) __syncthreads();  // the next slot may hold the same variable
          }
        }
        __syncthreads();
      }
    }
    float part = 0.0f;
    const uint64_t* cf = cw + f * (long long)C.words_n;
    for (int v = tid; v < n; v += blockDim.x) {
      const float b = app[v];
      Bout[f * (long long)n + v] = b;
      const float sv = ((cf[v >> 6] >> (v & 63)) & 1ull) ? -1.0f : 1.0f;
      const float z = -sv * b;
      part += (z > 0.0f ? z + log1pf(expf(-z)) : log1pf(expf(z))) * scale;
    }
    part = warp_sum_fixed(part);
    if ((tid & 31) == 0) s_part[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      float sum = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum = __fadd_rn(sum, s_part[w]);
      pf[f * (2LL * T * L + 1) + 2 * T * L] = sum;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kLayThreadsMax) nms_layered_backward_kernel(
    const DevCode* __restrict__ Cp, int T, int L, const uint64_t* __restrict__ cw, long long frames,
    const float* __restrict__ alpha, const float* __restrict__ beta, const float* __restrict__ X,
    const float* __restrict__ Bin, char* __restrict__ work, long long work_stride, float* __restrict__ pf) {
  __shared__ float s_ga[kLayThreadsMax], s_gb[kLayThreadsMax];
  const DevCode& C = *Cp;
  const int n = C.n, E = C.e_slots, ncg = C.ncg, tid = threadIdx.x;
  const int* __restrict__ slot_var = C.slot_var;
  float* Gv = (float*)(work + (long long)blockIdx.x * work_stride);  // dL/dA, natural order
  float* P = Gv + ((n + 63) & ~63);                                  // dL/dc from iteration t+1
  const float scale = 1.0f / ((float)frames * (float)n);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const uint64_t* cf = cw + f * (long long)C.words_n;
    for (int v = tid; v < n; v += blockDim.x) {
      const float b = Bin[f * (long long)n + v];
      const float sv = ((cf[v >> 6] >> (v & 63)) & 1ull) ? -1.0f : 1.0f;
      const float z = -sv * b;
      Gv[v] = scale * (1.0f / (1.0f + expf(-z))) * (-sv);
    }
    for (int s = tid; s < E; s += blockDim.x) P[s] = 0.0f;
    __syncthreads();
    float* row = pf + f * (2LL * T * L + 1);
    for (int t = T - 1; t >= 0; t--) {
      const float* Xt = X + (f * T + t) * (long long)E;
      for (int g = ncg - 1; g >= 0; g--) {
        const int4 G = C.cg[g];
        const uint32_t sync = C.cg_sync[g];
        const int nchk = G.y, d = G.z;
        const bool act = tid < nchk;
        const int lay = (L == ncg) ? g : 0;
        const float al = __ldg(&alpha[t * L + lay]), be = __ldg(&beta[t * L + lay]);
        int vv[kLearnDcMax];
        float dx[kLearnDcMax];
        if (act) {
          float x[kLearnDcMax], gc[kLearnDcMax];
          float m1 = __int_as_float(0x7f800000), m2 = m1;
          int i1 = -1, i2 = -1, nreal = 0;
          uint32_t neg = 0;
          for (int i = 0; i < d; i++) {
            const int s = G.w + i * nchk + tid;
            const int v = __ldg(&slot_var[s]);
            vv[i] = v;
            dx[i] = 0.0f;
            if (v < 0) continue;
            gc[i] = __fadd_rn(Gv[v], P[s]);
            x[i] = Xt[s];
            const float ax = fabsf(x[i]);
            if (ax < m1) {
              m2 = m1;
              i2 = i1;
              m1 = ax;
              i1 = i;
            } else if (ax < m2) {
              m2 = ax;
              i2 = i;
            }
            neg ^= (x[i] < 0.0f) ? 1u : 0u;
            nreal++;
          }
          float gA = 0.0f, gB = 0.0f, g1 = 0.0f, g2 = 0.0f;
          if (nreal > 1) {
            for (int i = 0; i < d; i++) {
              if (vv[i] < 0) continue;
              const float sg = ((neg ^ ((x[i] < 0.0f) ? 1u : 0u)) ? -1.0f : 1.0f);
              const float u = ((i == i1) ? m2 : m1) - be;
              if (u > 0.0f) {
                gA += gc[i] * sg * u;
                gB -= gc[i] * sg * al;
                const float gm = gc[i] * sg * al;
                if (i == i1) g2 += gm;  // the min over the others is slot i2
                else g1 += gm;          // the min over the others is slot i1
              }
            }
            if (i1 >= 0) dx[i1] = g1 * (x[i1] < 0.0f ? -1.0f : 1.0f);
            if (i2 >= 0) dx[i2] = g2 * (x[i2] < 0.0f ? -1.0f : 1.0f);
          }
          for (int i = 0; i < d; i++) {
            if (vv[i] < 0) continue;
            P[G.w + i * nchk + tid] = -Gv[vv[i]] - dx[i];  // dL/dc of iteration t-1
          }
          s_ga[tid] = gA;
          s_gb[tid] = gB;
        }
        __syncthreads();  // every read of G after the row group done
        if (sync == 0) {
          if (act)
            for (int i = 0; i < d; i++)
              if (vv[i] >= 0 && dx[i] != 0.0f) Gv[vv[i]] = __fadd_rn(Gv[vv[i]], dx[i]);
        } else {
          for (int i = 0; i < d; i++) {
            if (act && vv[i] >= 0 && dx[i] != 0.0f) Gv[vv[i]] = __fadd_rn(Gv[vv[i]], dx[i]);
            if ((sync >> i) & 1u) __syncthreads();
          }
        }
        if (tid < 32) {
          float sa = 0.0f, sb = 0.0f;
          for (int c = tid; c < nchk; c += 32) {
            sa = __fadd_rn(sa, s_ga[c]);
            sb = __fadd_rn(sb, s_gb[c]);
          }
          sa = warp_sum_fixed(sa);
          sb = warp_sum_fixed(sb);
          if (tid == 0) {
            if (L == ncg) {
              row[t * L + lay] = sa;
              row[T * L + t * L + lay] = sb;
            } else {  // one weight pair per iteration: row groups summed in descending order
              row[t * L] = (g == ncg - 1) ? sa : __fadd_rn(row[t * L], sa);
              row[T * L + t * L] = (g == ncg - 1) ? sb : __fadd_rn(row[T * L + t * L], sb);
            }
          }
        }
        __syncthreads();
      }
    }
  }
}

// out[i] = sum over frames f (ascending) of pf[f][i], i < 2 T L + 1; warp per i.
__global__ void nms_reduce_kernel(const float* __restrict__ pf, long long frames, int TL,
                                  float* __restrict__ grad_alpha, float* __restrict__ grad_beta,
                                  float* __restrict__ loss) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i > 2 * TL) return;
  float s = 0.0f;
  for (long long f = threadIdx.x & 31; f < frames; f += 32) s = __fadd_rn(s, pf[f * (2LL * TL + 1) + i]);
  s = warp_sum_fixed(s);
  if ((threadIdx.x & 31) == 0) {
    if (i < TL) grad_alpha[i] = s;
    else if (i < 2 * TL) grad_beta[i - TL] = s;
    else *loss = s;
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int count, float lr, float b1, float b2, float eps, float c1,
                            float c2, float lo, float hi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  float x = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
  p[i] = fminf(fmaxf(x, lo), hi);
}

int launch_nms_forward(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                       long long frames, const float* alpha, const float* beta, float* X, float* B, char* work,
                       long long work_stride, int grid, float* pf, cudaStream_t st) {
  if (h.max_dc > kLearnDcMax) return set_error(GF2C_ERR_UNSUPPORTED, "learned decoder: check degree above 32");
  nms_forward_kernel<<<grid, kLearnThreads, 0, st>>>(dcode, T, L, llr, cw, frames, alpha, beta, X, B, work,
                                                     work_stride, pf);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_nms_backward(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                        long long frames, const float* alpha, const float* beta, const float* X, const float* B,
                        char* work, long long work_stride, int grid, float* pf, float* ga, float* gb,
                        float* loss, cudaStream_t st) {
  nms_backward_kernel<<<grid, kLearnThreads, 0, st>>>(dcode, T, L, llr, cw, frames, alpha, beta, X, B, work,
                                                      work_stride, pf);
  GF2C_CUDA(cudaGetLastError());
  const int outs = 2 * T * L + 1, warps = 8;
  nms_reduce_kernel<<<(outs + warps - 1) / warps, warps * 32, 0, st>>>(pf, frames, T * L, ga, gb, loss);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_nms_layered(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                       long long frames, const float* alpha, const float* beta, float* X, float* B, char* work,
                       long long work_stride, int grid, float* pf, float* ga, float* gb, float* loss,
                       cudaStream_t st) {
  if (h.max_dc > kLearnDcMax) return set_error(GF2C_ERR_UNSUPPORTED, "learned decoder: check degree above 32");
  if (!h.layered_ok || h.max_nchk > kLayThreadsMax)
    return set_error(GF2C_ERR_UNSUPPORTED, "layered training needs row groups of at most 1024 checks");
  const int threads = std::max(32, (h.max_nchk + 31) / 32 * 32);
  nms_layered_forward_kernel<<<grid, threads, 0, st>>>(dcode, T, L, llr, cw, frames, alpha, beta, X, B, work,
                                                        work_stride, pf);
  GF2C_CUDA(cudaGetLastError());
  nms_layered_backward_kernel<<<grid, threads, 0, st>>>(dcode, T, L, cw, frames, alpha, beta, X, B, work,
                                                         work_stride, pf);
  GF2C_CUDA(cudaGetLastError());
  const int outs = 2 * T * L + 1, warps = 8;
  nms_reduce_kernel<<<(outs + warps - 1) / warps, warps * 32, 0, st>>>(pf, frames, T * L, ga, gb, loss);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2, float eps,
                int step, float lo, float hi, cudaStream_t st) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<(count + 255) / 256, 256, 0, st>>>(p, g, m1, m2, count, lr, b1, b2, eps, c1, c2, lo, hi);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

}  // namespace gf2c
