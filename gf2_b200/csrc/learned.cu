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
//   -1 if x < 0 else +1; d max(u, 0)/du = [u > 0].  Weight gradients are
//   summed per (t, row group) in shared memory and added to the global
//   gradient with one atomic per CTA.
// adam_kernel: Adam (Kingma & Ba 2015) with bias correction.
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
    float* __restrict__ Bout, char* __restrict__ work, long long work_stride, float* __restrict__ loss) {
  __shared__ float s_loss;
  const DevCode C = *Cp;
  const LearnCtx F = make_ctx(C, L);
  const int n = F.n, E = C.e_slots;
  float* c2v = (float*)(work + (long long)blockIdx.x * work_stride);
  float* app = c2v + ((E + 63) & ~63);
  const float scale = 1.0f / ((float)frames * (float)n);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const float* lf = llr + f * (long long)n;
    for (int v = threadIdx.x; v < n; v += blockDim.x) app[v] = lf[v];
    if (threadIdx.x == 0) s_loss = 0.0f;
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
    atomicAdd(&s_loss, part);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(loss, s_loss);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kLearnThreads) nms_backward_kernel(
    const DevCode* __restrict__ Cp, int T, int L, const float* __restrict__ llr, const uint64_t* __restrict__ cw,
    long long frames, const float* __restrict__ alpha, const float* __restrict__ beta,
    const float* __restrict__ X, const float* __restrict__ Bin, char* __restrict__ work, long long work_stride,
    float* __restrict__ grad_alpha, float* __restrict__ grad_beta) {
  extern __shared__ float s_g[];  // [2 * L]: alpha then beta gradients of the current t
  const DevCode C = *Cp;
  const LearnCtx F = make_ctx(C, L);
  const int n = F.n, E = C.e_slots;
  float* gx = (float*)(work + (long long)blockIdx.x * work_stride);
  float* gb = gx + ((E + 63) & ~63);
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
      for (int i = threadIdx.x; i < 2 * L; i += blockDim.x) s_g[i] = 0.0f;
      __syncthreads();
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
        if (gA != 0.0f) atomicAdd(&s_g[lay], gA);
        if (gB != 0.0f) atomicAdd(&s_g[L + lay], gB);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < L; i += blockDim.x) {
        if (s_g[i] != 0.0f) atomicAdd(&grad_alpha[t * L + i], s_g[i]);
        if (s_g[L + i] != 0.0f) atomicAdd(&grad_beta[t * L + i], s_g[L + i]);
      }
      if (t > 0)
        for (int v = threadIdx.x; v < n; v += blockDim.x) gb[v] = var_sum(F, v, 0.0f, gx);  // dL/db^{t-1}
      __syncthreads();
    }
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
                       long long work_stride, int grid, float* loss, cudaStream_t st) {
  if (h.max_dc > kLearnDcMax) return set_error(GF2C_ERR_UNSUPPORTED, "learned decoder: check degree above 32");
  nms_forward_kernel<<<grid, kLearnThreads, 0, st>>>(dcode, T, L, llr, cw, frames, alpha, beta, X, B, work,
                                                     work_stride, loss);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_nms_backward(const DevCode* dcode, const DevCode& h, int T, int L, const float* llr, const uint64_t* cw,
                        long long frames, const float* alpha, const float* beta, const float* X, const float* B,
                        char* work, long long work_stride, int grid, float* ga, float* gb, cudaStream_t st) {
  nms_backward_kernel<<<grid, kLearnThreads, 2 * L * sizeof(float), st>>>(dcode, T, L, llr, cw, frames, alpha, beta,
                                                                          X, B, work, work_stride, ga, gb);
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
