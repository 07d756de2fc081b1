// gf2cuda flooding min-sum decoder with the whole frame in shared memory (sm_100a).
//
// For min-sum the messages leaving a check are determined by five numbers:
// the smallest and second-smallest |v2c| (min1, min2), the slot of min1, the
// sign bits of the v2c and their parity -- slot i receives
//     sign_i * (i == argmin ? min2 : min1),  sign_i = negp ^ neg_i
// (Llr::boxplus_minsum_n, crates/gf2-coding/src/llr.rs:246-284, over the other
// edges).  Storing that 16-byte check state instead of the dc messages
// reproduces every message bit for bit, and for the DVB-T2 short codes the
// check states (m x 16 B) plus the posteriors (n x 4 B) fit in one SM's shared
// memory (short 1/2: 144 KB + 65 KB).  One CTA of 1024 threads decodes one frame
// at a time from shared memory only; global memory is read for the channel LLRs
// and the code tables and written for the results.
//
// The schedule and arithmetic are those of decode.cu (the reference's flooding
// loop, ldpc/core.rs:889-938): v2c = belief - c2v, belief = llr + sum of c2v in
// ascending original check index, syndrome of iteration t evaluated in the
// check-node pass of iteration t+1.  Normalised / offset min-sum stores the
// transformed magnitudes; FP16 message storage stores them rounded to binary16
// (rounding is odd-symmetric, so the stored messages are those of the
// full-message kernels).
#include <cuda_fp16.h>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

static constexpr int kSmemThreads = 1024;

__device__ __forceinline__ int sf_desc_var(uint32_t D, int t, int Z, int g) {
  const int base = (int)(D & 0xFFFFFu), sh = (int)((D >> 20) & 1023u), type = (int)(D >> 30);
  if (type == 0) {
    const int c = t + sh;
    return base + (c >= Z ? c - Z : c);
  }
  const int v = base + sh * t;
  if (type == 1) return (g == 0 && t == 0) ? -1 : v - 1;
  return v;
}

// c2v of slot i from a check state {mag1, mag2, negmask, argmin | negp << 8}
__device__ __forceinline__ float state_msg(const uint4 s, int i) {
  const int i1 = (int)(s.w & 0xffu);
  const uint32_t sg = ((s.w >> 8) ^ (s.z >> i)) & 1u;
  const float mag = __uint_as_float(i == i1 ? s.y : s.x);
  return sg ? -mag : mag;
}

template <int ALGO, int MSG16, int DCMAX>
__global__ void __launch_bounds__(kSmemThreads, 1) bp_smem_flood_kernel(const DecodeArgs a) {
  typedef MsgIO<MSG16> IO;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_frame;
  __shared__ DevCode C;
  const int tid = threadIdx.x, NT = blockDim.x;
  for (;;) {
    if (tid == 0) s_frame = (long long)atomicAdd(a.queue, 1ull);
    __syncthreads();
    const long long f = s_frame;
    if (f >= a.frames) break;
    const int cid = a.code_id ? a.code_id[f] : 0;
    if (cid < 0 || cid >= a.ncodes) {
      if (tid == 0) {
        atomicExch(a.status, 1);
        if (a.iters) a.iters[f] = -1;
      }
      __syncthreads();
      continue;
    }
    if (tid == 0) C = a.codes[cid];
    __syncthreads();
    const int n = C.n, m = C.m, vgs = C.vgs, ncg = C.ncg;
    // shared memory: check states (m x 16 B), posteriors (n x 4 B), hard decisions
    uint4* st = (uint4*)smem_raw;
    float* app = (float*)(smem_raw + (size_t)m * 16);
    uint32_t* bitmap = (uint32_t*)(app + ((n + 3) & ~3));
    const int4* __restrict__ cgp = C.cg;
    const uint16_t* __restrict__ chk_cg = C.chk_cg;
    const int* __restrict__ slot_var = C.slot_var;
    const uint32_t* __restrict__ sdesc = C.slot_desc;
    const int2* __restrict__ vg = C.vg;
    const int* __restrict__ vg_ci = C.vg_ci;
    const float* __restrict__ llr = a.llr + (a.llr_off ? a.llr_off[f] : f * (long long)n);
    const int maxit = a.max_iter_arr ? a.max_iter_arr[f] : a.max_iter;
    const int wn = (n + 31) >> 5;
    uint64_t* mo = a.msg ? a.msg + (a.msg_off ? a.msg_off[f] : f * (long long)C.words_k) : nullptr;
    float* bo = a.beliefs ? a.beliefs + (a.llr_off ? a.llr_off[f] : f * (long long)n) : nullptr;

    if (maxit <= 0) {
      if (mo)
        for (int w = tid; w < C.words_k; w += NT) mo[w] = 0ull;
      if (bo)
        for (int v = tid; v < n; v += NT) bo[v] = 0.0f;
      if (tid == 0) {
        if (a.iters) a.iters[f] = 0;
        if (a.conv) a.conv[f] = 0;
        if (a.synd_ok) a.synd_ok[f] = 1;
      }
      __syncthreads();
      continue;
    }
    for (int base = 0; base < n; base += NT) {
      const int v = base + tid;
      float x = 0.0f;
      if (v < n) {
        x = llr[v];
        app[v] = x;
      }
      const unsigned b = __ballot_sync(0xffffffffu, v < n && x < 0.0f);
      if ((tid & 31) == 0 && v < n) bitmap[v >> 5] = b;
    }
    __syncthreads();

    int it = 0, converged = 0, synd = 1;
    for (;;) {
      const int tw = (a.nms_iters > 0) ? min(it, a.nms_iters - 1) : 0;
      const bool first = it == 0;
      int par = 0;
      for (int cc = tid; cc < m; cc += NT) {
        const int g = chk_cg[cc];
        const int4 G = cgp[g];
        const int t = cc - G.x, nchk = G.y, d = G.z;
        int vv[DCMAX];
        if (sdesc) {
          const uint32_t* sd = sdesc + G.w / nchk;
#pragma unroll
          for (int i = 0; i < DCMAX; i++) vv[i] = (i < d) ? sf_desc_var(__ldg(&sd[i]), t, nchk, g) : -1;
        } else {
#pragma unroll
          for (int i = 0; i < DCMAX; i++) vv[i] = (i < d) ? __ldg(&slot_var[G.w + i * nchk + t]) : -1;
        }
        const uint4 so = first ? make_uint4(0u, 0u, 0u, 0u) : st[cc];
        float m1 = __int_as_float(0x7f800000), m2 = m1;
        int i1 = -1;
        uint32_t neg = 0, real = 0;
#pragma unroll
        for (int i = 0; i < DCMAX; i++) {
          if (vv[i] >= 0) {
            const float ap = app[vv[i]];
            par ^= (int)(ap < 0.0f);
            const float x = __fsub_rn(ap, state_msg(so, i));
            const float ax = fabsf(x);
            if (ax < m1) {
              m2 = m1;
              m1 = ax;
              i1 = i;
            } else if (ax < m2) {
              m2 = ax;
            }
            neg |= (uint32_t)(x < 0.0f) << i;
            real |= 1u << i;
          }
        }
        const bool single = __popc(real) == 1;
        float mag1 = single ? 0.0f : m1, mag2 = single ? 0.0f : m2;
        if (ALGO == 2) {  // normalised / offset
          const int lay = (a.nms_L == ncg) ? g : 0;
          const float al = __ldg(&a.alpha[tw * a.nms_L + lay]), be = __ldg(&a.beta[tw * a.nms_L + lay]);
          const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
          mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
          mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
        }
        mag1 = IO::rt(mag1);
        mag2 = IO::rt(mag2);
        const uint32_t negp = __popc(neg) & 1u;
        st[cc] = make_uint4(__float_as_uint(mag1), __float_as_uint(mag2), neg, (uint32_t)(i1 & 0xff) | (negp << 8));
      }
      par = __syncthreads_or(par);
      if (it > 0 && a.early_stop && !par) {
        converged = 1;
        synd = 0;
        break;
      }
      // variable nodes: belief = llr + sum of c2v in ascending original check index
      for (int base = 0; base < n; base += NT) {
        const int v = base + tid;
        float b = 0.0f;
        if (v < n) {
          const int h = v / vgs, j = v - h * vgs;
          const int2 V = vg[h];
          const int* ci = vg_ci + V.y + j;
          b = llr[v];
          int e[4];
          for (int i0 = 0; i0 < V.x; i0 += 4) {
#pragma unroll
            for (int q = 0; q < 4; q++) e[q] = (i0 + q < V.x) ? __ldg(&ci[(i0 + q) * vgs]) : -1;
#pragma unroll
            for (int q = 0; q < 4; q++)
              if (e[q] >= 0) b = __fadd_rn(b, state_msg(st[e[q] & 0xffffff], e[q] >> 24));
          }
          app[v] = b;
        }
        const unsigned bits = __ballot_sync(0xffffffffu, v < n && b < 0.0f);
        if ((tid & 31) == 0 && v < n) bitmap[v >> 5] = bits;
      }
      __syncthreads();
      ++it;
      if (it >= maxit) break;
    }
    if (!converged) {
      // syndrome of the final hard decisions
      int p = 0;
      for (int cc = tid; cc < m; cc += NT) {
        const int g = chk_cg[cc];
        const int4 G = cgp[g];
        const int t = cc - G.x;
        int q = 0;
        for (int i = 0; i < G.z; i++) {
          const int v = __ldg(&slot_var[G.w + i * G.y + t]);
          if (v >= 0) q ^= (bitmap[v >> 5] >> (v & 31)) & 1;
        }
        p |= q;
      }
      synd = __syncthreads_or(p);
      converged = !synd;
    }
    if (mo) {
      for (int w = tid; w < C.words_k; w += NT) {
        const uint32_t lo = bitmap[2 * w];
        const uint32_t hi = (2 * w + 1 < wn) ? bitmap[2 * w + 1] : 0u;
        unsigned long long word = (unsigned long long)lo | ((unsigned long long)hi << 32);
        const int rem = C.k - 64 * w;
        if (rem < 64) word &= (1ull << rem) - 1ull;
        mo[w] = word;
      }
    }
    if (bo)
      for (int v = tid; v < n; v += NT) bo[v] = app[v];
    if (tid == 0) {
      if (a.iters) a.iters[f] = it;
      if (a.conv) a.conv[f] = (uint8_t)converged;
      if (a.synd_ok) a.synd_ok[f] = (uint8_t)(!synd);
    }
    __syncthreads();
  }
}

// Shared memory of the kernel for codes up to (n, m).
size_t smem_flood_bytes(int n, int m) {
  return (size_t)m * 16 + (size_t)((n + 3) & ~3) * 4 + (size_t)((n + 31) / 32) * 4;
}

template <int ALGO, int MSG16>
static const void* sf_dc(int dcmax) {
  switch (dcmax) {
    case 8: return (const void*)bp_smem_flood_kernel<ALGO, MSG16, 8>;
    case 16: return (const void*)bp_smem_flood_kernel<ALGO, MSG16, 16>;
    case 24: return (const void*)bp_smem_flood_kernel<ALGO, MSG16, 24>;
    case 32: return (const void*)bp_smem_flood_kernel<ALGO, MSG16, 32>;
  }
  return nullptr;
}

// Kernel for min-sum (algo 0) / normalised-offset min-sum (algo 2), or nullptr.
const void* smem_flood_kernel_ptr(int algo, int msg16, int dcmax) {
  if (algo == 0) return msg16 ? sf_dc<0, 1>(dcmax) : sf_dc<0, 0>(dcmax);
  if (algo == 2) return msg16 ? sf_dc<2, 1>(dcmax) : sf_dc<2, 0>(dcmax);
  return nullptr;
}

}  // namespace gf2c
