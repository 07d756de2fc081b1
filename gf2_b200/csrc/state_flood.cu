// gf2cuda flooding min-sum decoder on compressed check states (sm_100a).
//
// For min-sum every message leaving a check is determined by four numbers: the
// smallest and second-smallest |v2c| (min1, min2), the slot of min1 and the
// final sign of each slot's message (the parity of the other inputs' signs):
//     c2v_i = sign_i * (i == argmin ? min2 : min1)
// (Llr::boxplus_minsum_n, crates/gf2-coding/src/llr.rs:246-284, over the other
// edges of the check).  A 16-byte state {min1, min2, sign bits, argmin} per
// check therefore reproduces every message bit for bit while moving 16 B per
// check instead of 4 B per edge, and the check-node pass writes nothing per
// edge.
//
// Schedule and arithmetic are the reference's flooding loop
// (ldpc/core.rs:889-938): v2c = belief - c2v (formed in the check node, the
// same IEEE subtraction), belief = llr + sum of c2v in ascending original check
// index, the syndrome of the hard decisions of iteration t evaluated in the
// check-node pass of iteration t + 1.  Normalised / offset min-sum transforms
// the two magnitudes; FP16 message storage rounds them to binary16 (the
// rounding is odd-symmetric, so the messages equal those of a decoder that
// stores each message in binary16).
//
// Work decomposition.  One CTA of 1024 threads decodes one frame at a time
// (persistent, frames from an atomic queue).  Each warp takes chunks of 32
// consecutive checks of one row group (check pass) or 32 consecutive
// variables of one variable group (variable pass), so the degree, the slot
// descriptors and the loop trip counts are warp-uniform.  The posteriors are
// kept in "u order" (DVB-T2 parity bit k + a + q t at k + a Z + t), in which
// every slot of every row group reads a contiguous, rotated run of Z
// posteriors and every variable group reads contiguous check states.
//
// Placement.  The check states (m x 16 B) and the posteriors (n x 4 B) live in
// shared memory when they fit together (DVB-T2 short frames); otherwise each
// lives in the CTA's global workspace slice, which stays in the 126 MB L2 for
// the frames in flight.  The u-order copy of the channel LLRs (read once per
// iteration) is always in the workspace.
#include <cuda_fp16.h>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

static constexpr int kStateThreads = 1024;

// c2v of slot i from a check state {min1, min2, sign bits, argmin}
__device__ __forceinline__ float state_c2v(const uint4 s, int i) {
  const uint32_t mag = (i == (int)s.w) ? s.y : s.x;
  return __uint_as_float(mag | ((s.z >> i) << 31));
}

__device__ __forceinline__ float round_mag16(float v) {
  return __half2float(__float2half_rn(v > 65504.0f ? 65504.0f : v));
}

// u-order variable of slot descriptor D for check t of a row group of Z checks
__device__ __forceinline__ int state_desc_var(uint32_t D, int t, int Z) {
  const int base = (int)(D & 0xFFFFFu), sh = (int)((D >> 20) & 1023u);
  const int c = t + sh;
  const int u = base + (c >= Z ? c - Z : c);
  return ((D >> 31) && t == 0) ? -1 : u;
}

// Posteriors of the slots of check t of row group G (slot i in ap[i]); returns
// the mask of the slots that hold an edge.
template <int DCMAX>
__device__ __forceinline__ uint32_t load_slots(const DevCode& C, const int4 G, int t, const float* app,
                                               float (&ap)[DCMAX]) {
  uint32_t real = 0;
  if (C.sp_desc) {
    const uint32_t* __restrict__ sd = C.sp_desc + G.w;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if (i < G.z) {
        const int u = state_desc_var(__ldg(&sd[i]), t, G.y);
        real |= (uint32_t)(u >= 0) << i;
        ap[i] = app[u < 0 ? 0 : u];
      }
    }
  } else {
    const int* __restrict__ sv = C.slot_var + G.w + t;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if (i < G.z) {
        const int u = __ldg(&sv[i * G.y]);
        real |= (uint32_t)(u >= 0) << i;
        ap[i] = app[u < 0 ? 0 : u];
      }
    }
  }
  return real;
}

template <int DCMAX, bool ALL_SMEM>
__global__ void __launch_bounds__(kStateThreads, 1) bp_state_flood_kernel(const DecodeArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_frame;
  __shared__ DevCode C;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = NT >> 5;
  char* work = a.work + (long long)blockIdx.x * a.work_stride;
  const bool msg16 = a.sf_msg16 != 0;  // magnitudes rounded to binary16
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
    const int n = C.n, m = C.m, k = C.k, vgs = C.vgs;
    uint4* st;
    float* app;
    if (ALL_SMEM) {
      st = (uint4*)smem_raw;
      app = (float*)(smem_raw + (size_t)m * 16);
    } else {
      st = a.sf_st_smem ? (uint4*)smem_raw : (uint4*)(work + a.sf_st_off);
      app = a.sf_app_smem ? (float*)(smem_raw + (a.sf_st_smem ? (size_t)m * 16 : 0)) : (float*)(work + a.sf_app_off);
    }
    const float* __restrict__ llr = a.llr + (a.llr_off ? a.llr_off[f] : f * (long long)n);
    const int* __restrict__ u2v = C.sp_u2v;
    float* llr_u = (float*)(work + a.sf_llr_off);
    const float* __restrict__ lu = u2v ? llr_u : llr;
    const int maxit = a.max_iter_arr ? a.max_iter_arr[f] : a.max_iter;
    uint64_t* mo = a.msg ? a.msg + (a.msg_off ? a.msg_off[f] : f * (long long)C.words_k) : nullptr;
    float* bo = a.beliefs ? a.beliefs + (a.llr_off ? a.llr_off[f] : f * (long long)n) : nullptr;

    if (maxit <= 0) {  // a fresh reference decoder: all-zero beliefs, valid word
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
    for (int u = tid; u < n; u += NT) {
      const float x = u2v ? llr[__ldg(&u2v[u])] : llr[u];
      if (u2v) llr_u[u] = x;
      app[u] = x;
    }
    __syncthreads();

    const int4* __restrict__ spcg = C.sp_cg;
    const int2* __restrict__ cch = C.sp_cchunk;
    const int2* __restrict__ vch = C.sp_vchunk;
    const int2* __restrict__ svg = C.sp_vg;
    const int* __restrict__ sci = C.sp_ci;
    const int ncc = C.sp_ncchunk, nvc = C.sp_nvchunk;
    int it = 0, converged = 0, synd = 1;
    for (;;) {
      const bool first = it == 0;
      const int tw = (a.nms_iters > 0) ? min(it, a.nms_iters - 1) : 0;
      int par = 0;
      // check nodes: new state from the posteriors and the old state
      for (int ch = warp; ch < ncc; ch += nwarps) {
        const int2 CH = cch[ch];
        const int4 G = spcg[CH.x];
        const int t = CH.y + lane;
        if (t >= G.y) continue;
        const int cc = G.x + t;
        float ap[DCMAX];
        const uint32_t real = load_slots<DCMAX>(C, G, t, app, ap);
        const uint4 so = first ? make_uint4(0u, 0u, 0u, 0xffu) : st[cc];
        float m1 = __int_as_float(0x7f800000), m2 = m1;
        uint32_t i1 = 0xffu, neg = 0u;
        int hp = 0;
#pragma unroll
        for (int i = 0; i < DCMAX; i++) {
          if (i < G.z && ((real >> i) & 1u)) {
            hp ^= (int)(ap[i] < 0.0f);
            const float x = __fsub_rn(ap[i], state_c2v(so, i));
            const float ax = fabsf(x);
            const bool lt1 = ax < m1, lt2 = ax < m2;
            m2 = lt1 ? m1 : (lt2 ? ax : m2);
            m1 = lt1 ? ax : m1;
            i1 = lt1 ? (uint32_t)i : i1;
            neg |= (uint32_t)(x < 0.0f) << i;
          }
        }
        par |= hp;
        const bool single = __popc(real) == 1;
        float mag1 = single ? 0.0f : m1, mag2 = single ? 0.0f : m2;
        if (a.nms_iters > 0) {  // normalised / offset min-sum
          const int lay = (a.nms_L == C.ncg) ? CH.x : 0;
          const float al = __ldg(&a.alpha[tw * a.nms_L + lay]), be = __ldg(&a.beta[tw * a.nms_L + lay]);
          const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
          mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
          mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
        }
        if (msg16) {
          mag1 = round_mag16(mag1);
          mag2 = round_mag16(mag2);
        }
        const uint32_t sgn = (__popc(neg) & 1) ? ~neg : neg;
        st[cc] = make_uint4(__float_as_uint(mag1), __float_as_uint(mag2), sgn, i1);
      }
      par = __syncthreads_or(par);
      if (it > 0 && a.early_stop && !par) {
        converged = 1;
        synd = 0;
        break;
      }
      // variable nodes: belief = llr + sum of c2v in ascending original check index
      for (int ch = warp; ch < nvc; ch += nwarps) {
        const int2 CH = vch[ch];
        const int2 V = svg[CH.x];
        const int j = CH.y + lane;
        const int u = CH.x * vgs + j;
        if (j >= vgs || u >= n) continue;
        const int* __restrict__ ci = sci + V.y + j;
        float b = lu[u];
        int i = 0;
        for (; i + 4 <= V.x; i += 4) {
          int e[4];
          uint4 s[4];
#pragma unroll
          for (int q = 0; q < 4; q++) e[q] = __ldg(&ci[(i + q) * vgs]);
#pragma unroll
          for (int q = 0; q < 4; q++) s[q] = st[e[q] < 0 ? 0 : (e[q] & 0xffffff)];
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (e[q] >= 0) b = __fadd_rn(b, state_c2v(s[q], e[q] >> 24));
        }
        if (V.x - i >= 2) {
          const int e0 = __ldg(&ci[i * vgs]), e1 = __ldg(&ci[(i + 1) * vgs]);
          const uint4 s0 = st[e0 < 0 ? 0 : (e0 & 0xffffff)], s1 = st[e1 < 0 ? 0 : (e1 & 0xffffff)];
          if (e0 >= 0) b = __fadd_rn(b, state_c2v(s0, e0 >> 24));
          if (e1 >= 0) b = __fadd_rn(b, state_c2v(s1, e1 >> 24));
          i += 2;
        }
        if (i < V.x) {
          const int e0 = __ldg(&ci[i * vgs]);
          if (e0 >= 0) b = __fadd_rn(b, state_c2v(st[e0 & 0xffffff], e0 >> 24));
        }
        app[u] = b;
      }
      __syncthreads();
      ++it;
      if (it >= maxit) break;
    }
    if (!converged) {
      // syndrome of the final hard decisions
      int p = 0;
      for (int ch = warp; ch < ncc; ch += nwarps) {
        const int2 CH = cch[ch];
        const int4 G = spcg[CH.x];
        const int t = CH.y + lane;
        if (t >= G.y) continue;
        float ap[DCMAX];
        const uint32_t real = load_slots<DCMAX>(C, G, t, app, ap);
#pragma unroll
        for (int i = 0; i < DCMAX; i++)
          if (i < G.z && ((real >> i) & 1u)) p ^= (int)(ap[i] < 0.0f);
      }
      synd = __syncthreads_or(p);
      converged = !synd;
    }
    if (mo) {  // message bits: the first k variables (identical in u order)
      uint32_t* mo32 = (uint32_t*)mo;
      for (int base = 0; base < 64 * C.words_k; base += NT) {
        const int u = base + tid;
        const unsigned bits = __ballot_sync(0xffffffffu, u < k && app[u < n ? u : 0] < 0.0f);
        if (lane == 0 && u < 64 * C.words_k) mo32[u >> 5] = bits;
      }
    }
    if (bo)
      for (int u = tid; u < n; u += NT) bo[u2v ? __ldg(&u2v[u]) : u] = app[u];
    if (tid == 0) {
      if (a.iters) a.iters[f] = it;
      if (a.conv) a.conv[f] = (uint8_t)converged;
      if (a.synd_ok) a.synd_ok[f] = (uint8_t)(!synd);
    }
    __syncthreads();
  }
}

int state_dcmax_bucket(int max_dc) {
  static const int buckets[] = {7, 9, 10, 11, 13, 14, 18, 19, 22, 26, 32};
  for (int b : buckets)
    if (max_dc <= b) return b;
  return -1;
}

template <bool ALL_SMEM>
static const void* state_kernel(int dcmax) {
  switch (dcmax) {
    case 7: return (const void*)bp_state_flood_kernel<7, ALL_SMEM>;
    case 9: return (const void*)bp_state_flood_kernel<9, ALL_SMEM>;
    case 10: return (const void*)bp_state_flood_kernel<10, ALL_SMEM>;
    case 11: return (const void*)bp_state_flood_kernel<11, ALL_SMEM>;
    case 13: return (const void*)bp_state_flood_kernel<13, ALL_SMEM>;
    case 14: return (const void*)bp_state_flood_kernel<14, ALL_SMEM>;
    case 18: return (const void*)bp_state_flood_kernel<18, ALL_SMEM>;
    case 19: return (const void*)bp_state_flood_kernel<19, ALL_SMEM>;
    case 22: return (const void*)bp_state_flood_kernel<22, ALL_SMEM>;
    case 26: return (const void*)bp_state_flood_kernel<26, ALL_SMEM>;
    case 32: return (const void*)bp_state_flood_kernel<32, ALL_SMEM>;
  }
  return nullptr;
}

const void* state_flood_kernel_ptr(int dcmax, bool all_smem) {
  return all_smem ? state_kernel<true>(dcmax) : state_kernel<false>(dcmax);
}

}  // namespace gf2c
