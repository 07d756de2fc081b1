// gf2cuda flooding-schedule decoder (sm_100a).
//
// One persistent kernel decodes a batch: each CTA takes the next frame from an
// atomic queue, decodes it to completion (per-frame early stop, no wasted
// iterations on converged frames), writes its results and takes another.  The
// frame's posterior LLRs (APP) live in shared memory when they fit (short
// frames) and otherwise in the CTA's slice of a global workspace, which stays
// resident in the 126 MB L2 for the frames in flight.  The c2v messages live in
// the same workspace, laid out check-group-major so that consecutive threads
// (consecutive checks of a circulant) touch consecutive addresses.
//
// Schedule: LdpcDecoder::decode_iterative (crates/gf2-coding/src/ldpc/core.rs:889-938).
// The reference stores v2c and c2v; here only c2v and the belief are stored and
// v2c = belief - c2v is formed inside the check node, which is the same IEEE
// subtraction the reference performs (core.rs:831-836), so messages and beliefs
// agree bit for bit.  The belief sum runs over the variable's checks in
// ascending original check index (core.rs:824-827, the CSC order of
// gf2-core/src/sparse.rs:297-328).  The syndrome of iteration t is evaluated
// while the check nodes of iteration t+1 read the beliefs.
//
// Every check node first computes the variables of all its slots, then issues
// all loads from always-valid addresses, then does the arithmetic, so the
// loads of one check are in flight together.
#include <cuda_fp16.h>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

enum { ALGO_MS = 0, ALGO_SPA = 1, ALGO_NMS = 2, ALGO_SPA_FAST = 3 };

__device__ __forceinline__ float sfu_ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sfu_lg2(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sfu_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <int DCMAX>
struct MaskOf {
  typedef uint32_t T;
  static __device__ __forceinline__ int popc(T x) { return __popc(x); }
};
template <>
struct MaskOf<64> {
  typedef unsigned long long T;
  static __device__ __forceinline__ int popc(T x) { return __popcll(x); }
};

struct FrameCtx {
  int n, m, k, ncg, vgs;
  const int4* cg;
  const int* slot_var;
  const uint32_t* slot_desc;
  const uint16_t* chk_cg;
  const int2* vg;
  const int* vg_slot;
};

__device__ __forceinline__ int desc_var(uint32_t D, int t, int Z, int g) {
  const int base = (int)(D & 0xFFFFFu), sh = (int)((D >> 20) & 1023u), type = (int)(D >> 30);
  if (type == 0) {
    const int c = t + sh;
    return base + (c >= Z ? c - Z : c);
  }
  const int v = base + sh * t;
  if (type == 1) return (g == 0 && t == 0) ? -1 : v - 1;
  return v;
}

// Check-node update of flattened check cc: reads the APP and the old c2v,
// writes the new c2v.  Returns the parity of the hard decisions of the APP over
// the check (the syndrome bit of the previous iteration).
template <int ALGO, int MSG16, int DCMAX>
__device__ __forceinline__ int check_update(const FrameCtx& F, int cc, const float* __restrict__ app,
                                            typename MsgIO<MSG16>::T* __restrict__ c2v, bool first, float al,
                                            float be) {
  typedef MsgIO<MSG16> IO;
  typedef typename MaskOf<DCMAX>::T MaskT;
  const int g = F.chk_cg[cc];
  const int4 G = F.cg[g];
  const int t = cc - G.x, nchk = G.y, d = G.z, s0 = G.w + t;
  int vv[DCMAX];
  float ap[DCMAX], o[DCMAX];
  if (F.slot_desc) {
    const uint32_t* sd = F.slot_desc + G.w / nchk;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) vv[i] = (i < d) ? desc_var(__ldg(&sd[i]), t, nchk, g) : -1;
  } else {
#pragma unroll
    for (int i = 0; i < DCMAX; i++) vv[i] = (i < d) ? __ldg(&F.slot_var[s0 + i * nchk]) : -1;
  }
#pragma unroll
  for (int i = 0; i < DCMAX; i++) ap[i] = app[vv[i] < 0 ? 0 : vv[i]];
  if (first) {
#pragma unroll
    for (int i = 0; i < DCMAX; i++) o[i] = 0.0f;
  } else {
#pragma unroll
    for (int i = 0; i < DCMAX; i++) o[i] = IO::ld(c2v, (i < d) ? s0 + i * nchk : s0);
  }
  int par = 0;
  MaskT neg = 0, real = 0;
#pragma unroll
  for (int i = 0; i < DCMAX; i++) {
    const bool r = vv[i] >= 0;
    par ^= (int)(r && ap[i] < 0.0f);  // hard decision of the APP
    ap[i] = __fsub_rn(ap[i], o[i]);   // v2c
    real |= (MaskT)r << i;
    neg |= (MaskT)(r && ap[i] < 0.0f) << i;
  }
  const int negp = MaskOf<DCMAX>::popc(neg) & 1;
  const bool single = MaskOf<DCMAX>::popc(real) == 1;
  if (ALGO == ALGO_MS || ALGO == ALGO_NMS) {
    float m1 = __int_as_float(0x7f800000), m2 = m1;
    int i1 = -1;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float ax = ((real >> i) & 1) ? fabsf(ap[i]) : __int_as_float(0x7f800000);
      if (ax < m1) {
        m2 = m1;
        m1 = ax;
        i1 = i;
      } else if (ax < m2) {
        m2 = ax;
      }
    }
    float mag1 = single ? 0.0f : m1, mag2 = single ? 0.0f : m2;
    if (ALGO == ALGO_NMS) {
      const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
      mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
      mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
    }
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if ((real >> i) & 1) {
        const float mag = (i == i1) ? mag2 : mag1;
        IO::st(c2v, s0 + i * nchk, (negp ^ (int)((neg >> i) & 1)) ? -mag : mag);
      }
    }
  } else if (ALGO == ALGO_SPA_FAST) {
    // |c2v_i| = ln((D n_i + N d_i) / (D n_i - N d_i)), n = 1 - e, d = 1 + e, e = exp(-|x|)
    float N = 1.0f, D = 1.0f;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float e = ((real >> i) & 1) ? sfu_ex2(fabsf(ap[i]) * -1.4426950408889634f) : 0.0f;
      ap[i] = e;
      N *= fmaxf(1.0f - e, 5.9604645e-08f);
      D = __fmaf_rn(D, e, D);
    }
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if ((real >> i) & 1) {
        const float ni = fmaxf(1.0f - ap[i], 5.9604645e-08f), di = 1.0f + ap[i];
        const float num = __fmaf_rn(D, ni, N * di);
        const float den = fmaxf(__fmaf_rn(D, ni, -N * di), num * 5.9604645e-08f);
        float mag = 0.69314718055994531f * sfu_lg2(num * sfu_rcp(den));
        mag = single ? 0.0f : fminf(mag, 16.635532f);
        IO::st(c2v, s0 + i * nchk, (negp ^ (int)((neg >> i) & 1)) ? -mag : mag);
      }
    }
  } else {  // sum-product with the library's exact numerics
    float suf[DCMAX];
#pragma unroll
    for (int i = 0; i < DCMAX; i++) ap[i] = ((real >> i) & 1) ? tanh_half_f(ap[i]) : 1.0f;
    suf[DCMAX - 1] = 1.0f;
#pragma unroll
    for (int i = DCMAX - 2; i >= 0; i--) suf[i] = (i + 1 < d) ? __fmul_rn(ap[i + 1], suf[i + 1]) : 1.0f;
    float pre = 1.0f;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if ((real >> i) & 1) {
        float p = __fmul_rn(pre, suf[i]);
        p = p > GF2C_SPA_PMAX ? GF2C_SPA_PMAX : (p < -GF2C_SPA_PMAX ? -GF2C_SPA_PMAX : p);
        IO::st(c2v, s0 + i * nchk, single ? 0.0f : two_atanh_f(p));
      }
      if (i < d) pre = (i == 0) ? ap[0] : __fmul_rn(pre, ap[i]);
    }
  }
  return par;
}

// belief[v] = llr[v] + sum of c2v over v's checks in ascending original check
// index, for two variables per thread with their slot and message loads
// interleaved (4 slots per round).
template <int MSG16>
__device__ __forceinline__ void var_update2(const FrameCtx& F, int v0, int v1, const float* __restrict__ llr,
                                            const typename MsgIO<MSG16>::T* __restrict__ c2v, float* app,
                                            float& b0, float& b1) {
  typedef MsgIO<MSG16> IO;
  const int vgs = F.vgs;
  int dv[2] = {0, 0};
  const int* sl[2] = {F.vg_slot, F.vg_slot};
  float b[2] = {0.0f, 0.0f};
  const int vs[2] = {v0, v1};
#pragma unroll
  for (int u = 0; u < 2; u++) {
    if (vs[u] >= 0) {
      const int h = vs[u] / vgs, j = vs[u] - h * vgs;
      const int2 V = F.vg[h];
      dv[u] = V.x;
      sl[u] = F.vg_slot + V.y + j;
      b[u] = llr[vs[u]];
    }
  }
  const int dmax = max(dv[0], dv[1]);
  for (int i0 = 0; i0 < dmax; i0 += 4) {
    int s[2][4];
    float c[2][4];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int q = 0; q < 4; q++) s[u][q] = (i0 + q < dv[u]) ? __ldg(&sl[u][(i0 + q) * vgs]) : -1;
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int q = 0; q < 4; q++) c[u][q] = IO::ld(c2v, s[u][q] < 0 ? 0 : s[u][q]);
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (s[u][q] >= 0) b[u] = __fadd_rn(b[u], c[u][q]);
  }
  if (v0 >= 0) app[v0] = b[0];
  if (v1 >= 0) app[v1] = b[1];
  b0 = b[0];
  b1 = b[1];
}

// Parity of the hard decisions (from the bitmap) over all checks; block-wide OR.
__device__ __forceinline__ int syndrome_any(const FrameCtx& F, const uint32_t* bitmap) {
  int par = 0;
  for (int cc = threadIdx.x; cc < F.m; cc += blockDim.x) {
    const int g = F.chk_cg[cc];
    const int4 G = F.cg[g];
    const int t = cc - G.x;
    int p = 0;
    for (int i = 0; i < G.z; i++) {
      const int v = __ldg(&F.slot_var[G.w + i * G.y + t]);
      if (v >= 0) p ^= (bitmap[v >> 5] >> (v & 31)) & 1;
    }
    par |= p;
  }
  return __syncthreads_or(par);
}

template <int ALGO, int MSG16, int DCMAX, int MAXT = 512>
__global__ void __launch_bounds__(MAXT) bp_decode_kernel(const DecodeArgs a) {
  typedef MsgIO<MSG16> IO;
  typedef typename IO::T MsgT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_frame;
  __shared__ DevCode C;
  uint32_t* bitmap = (uint32_t*)smem_raw;
  float* smem_app = (float*)(smem_raw + ((a.bitmap_words * 4 + 15) & ~15));
  char* work = a.work + (long long)blockIdx.x * a.work_stride;
  MsgT* __restrict__ c2v = (MsgT*)work;
  float* gapp = (float*)(work + a.app_offset);
  const int tid = threadIdx.x, NT = blockDim.x;

  for (;;) {
    if (tid == 0) {
      const long long q = (long long)atomicAdd(a.queue, 1ull);
      const long long nq = a.frames_dev ? *a.frames_dev : a.frames;  // queue entries
      s_frame = (q < nq) ? (a.order != nullptr ? a.order[q] : q) : -1;
    }
    __syncthreads();
    const long long f = s_frame;
    if (f < 0 || f >= a.frames) break;
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
    FrameCtx F{C.n, C.m, C.k, C.ncg, C.vgs, C.cg, C.slot_var, C.slot_desc, C.chk_cg, C.vg, C.vg_slot};
    const int n = F.n;
    const float* __restrict__ llr = a.llr + (a.llr_off ? a.llr_off[f] : f * (long long)n);
    const int maxit = a.max_iter_arr ? a.max_iter_arr[f] : a.max_iter;
    float* app = (n <= a.smem_app_floats) ? smem_app : gapp;
    const int wn = (n + 31) >> 5;
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

    // APP = channel LLR; hard-decision bitmap
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
      int par = 0;
      for (int cc = tid; cc < F.m; cc += NT) {
        float al = 1.0f, be = 0.0f;
        if (ALGO == ALGO_NMS) {
          const int lay = (a.nms_L == F.ncg) ? (int)F.chk_cg[cc] : 0;
          al = __ldg(&a.alpha[tw * a.nms_L + lay]);
          be = __ldg(&a.beta[tw * a.nms_L + lay]);
        }
        par |= check_update<ALGO, MSG16, DCMAX>(F, cc, app, c2v, it == 0, al, be);
      }
      par = __syncthreads_or(par);
      if (it > 0 && a.early_stop && !par) {
        converged = 1;
        synd = 0;
        break;
      }
      // variable nodes, two per thread per round
      for (int base = 0; base < n; base += 2 * NT) {
        const int v0 = base + tid, v1 = base + NT + tid;
        float b0 = 0.0f, b1 = 0.0f;
        var_update2<MSG16>(F, v0 < n ? v0 : -1, v1 < n ? v1 : -1, llr, c2v, app, b0, b1);
        const unsigned m0 = __ballot_sync(0xffffffffu, v0 < n && b0 < 0.0f);
        const unsigned m1 = __ballot_sync(0xffffffffu, v1 < n && b1 < 0.0f);
        if ((tid & 31) == 0) {
          if (v0 < n) bitmap[v0 >> 5] = m0;
          if (v1 < n) bitmap[v1 >> 5] = m1;
        }
      }
      __syncthreads();
      ++it;
      if (it >= maxit) break;
    }
    if (!converged) {
      synd = syndrome_any(F, bitmap);
      converged = !synd;
    }

    // results
    if (mo) {
      for (int w = tid; w < C.words_k; w += NT) {
        const uint32_t lo = bitmap[2 * w];
        const uint32_t hi = (2 * w + 1 < wn) ? bitmap[2 * w + 1] : 0u;
        unsigned long long word = (unsigned long long)lo | ((unsigned long long)hi << 32);
        const int rem = F.k - 64 * w;
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

int decode_dcmax_bucket(int max_dc) {
  if (max_dc <= 8) return 8;
  if (max_dc <= 16) return 16;
  if (max_dc <= 24) return 24;
  if (max_dc <= 32) return 32;
  if (max_dc <= 64) return 64;
  return -1;
}

size_t decode_smem_bytes(int smem_app_floats, int bitmap_words) {
  return (size_t)((bitmap_words * 4 + 15) & ~15) + (size_t)smem_app_floats * 4;
}

template <int ALGO, int MSG16>
static const void* kernel_dc(int dcmax, int threads) {
  // up to 1024 threads per frame for checks of at most 8 slots (64 registers
  // suffice; short batches, where a frame's latency sets the step, gain)
  if (threads > 512) return dcmax == 8 ? (const void*)bp_decode_kernel<ALGO, MSG16, 8, 1024> : nullptr;
  switch (dcmax) {
    case 8: return (const void*)bp_decode_kernel<ALGO, MSG16, 8>;
    case 16: return (const void*)bp_decode_kernel<ALGO, MSG16, 16>;
    case 24: return (const void*)bp_decode_kernel<ALGO, MSG16, 24>;
    case 32: return (const void*)bp_decode_kernel<ALGO, MSG16, 32>;
    case 64: return (const void*)bp_decode_kernel<ALGO, MSG16, 64>;
  }
  return nullptr;
}

// Frame order of a mixed batch: for each rank, a block-wide stable compaction
// of the frames of that rank (ballot + popc within a warp, warp totals in
// shared memory).  Decoding the frames of one code together keeps the SMs on
// one slot count's code path at a time.
__global__ void __launch_bounds__(1024) mixed_order_kernel(const int32_t* __restrict__ code_id, int64_t frames,
                                                           const int32_t* __restrict__ rank_of, int ncodes,
                                                           int64_t* __restrict__ order) {
  __shared__ int s_warp[32];
  __shared__ long long s_pos;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) s_pos = 0;
  __syncthreads();
  for (int r = 0; r <= ncodes; r++) {
    for (long long base = 0; base < frames; base += blockDim.x) {
      const long long f = base + tid;
      bool hit = false;
      if (f < frames) {
        const int c = code_id[f];
        hit = ((c >= 0 && c < ncodes) ? __ldg(&rank_of[c]) : ncodes) == r;
      }
      const unsigned b = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) s_warp[wid] = __popc(b);
      __syncthreads();
      int before = 0, total = 0;
      for (int w = 0; w < nw; w++) {
        const int x = s_warp[w];
        before += (w < wid) ? x : 0;
        total += x;
      }
      const long long p0 = s_pos;
      if (hit) order[p0 + before + __popc(b & ((1u << lane) - 1u))] = f;
      __syncthreads();  // s_warp and s_pos read by all
      if (tid == 0) s_pos = p0 + total;
      __syncthreads();
    }
  }
}

cudaError_t launch_mixed_order(const int32_t* code_id, int64_t frames, const int32_t* rank_of, int ncodes,
                               int64_t* order, cudaStream_t st) {
  mixed_order_kernel<<<1, 1024, 0, st>>>(code_id, frames, rank_of, ncodes, order);
  return cudaGetLastError();
}

// The frames a first decoder left with a failing syndrome, for the fallback
// pass: the same block-wide stable compaction (ballot + popc per warp, warp
// totals in shared memory), ascending frame index, count written last.
__global__ void __launch_bounds__(1024) failed_list_kernel(const uint8_t* __restrict__ synd_ok, int64_t frames,
                                                           int64_t* __restrict__ list, long long* __restrict__ count) {
  __shared__ int s_warp[32];
  __shared__ long long s_pos;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) s_pos = 0;
  __syncthreads();
  for (long long base = 0; base < frames; base += blockDim.x) {
    const long long f = base + tid;
    const bool hit = f < frames && synd_ok[f] == 0;
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_warp[wid] = __popc(b);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < nw; w++) {
      const int x = s_warp[w];
      before += (w < wid) ? x : 0;
      total += x;
    }
    const long long p0 = s_pos;
    if (hit) list[p0 + before + __popc(b & ((1u << lane) - 1u))] = f;
    __syncthreads();
    if (tid == 0) s_pos = p0 + total;
    __syncthreads();
  }
  if (tid == 0) *count = s_pos;
}

cudaError_t launch_failed_list(const uint8_t* synd_ok, int64_t frames, int64_t* list, long long* count,
                               cudaStream_t st) {
  failed_list_kernel<<<1, 1024, 0, st>>>(synd_ok, frames, list, count);
  return cudaGetLastError();
}

// Sum of |LLR| of each frame (one CTA per frame, a fixed summation order).
__global__ void __launch_bounds__(256) frame_key_kernel(const float* __restrict__ llr, int n,
                                                        float* __restrict__ key) {
  __shared__ float s_part[8];
  const float* __restrict__ p = llr + (long long)blockIdx.x * n;
  float s = 0.0f;
  for (int v = threadIdx.x; v < n; v += blockDim.x) s += fabsf(__ldg(&p[v]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_part[w];
    key[blockIdx.x] = t;
  }
}

// One CTA: bitonic sort of (key bits << 32 | frame) over the next power of two
// (padding sorts last), ascending; non-negative keys order like their bits.
__global__ void __launch_bounds__(1024) key_order_kernel(const float* __restrict__ key, int frames, int P,
                                                         int64_t* __restrict__ order) {
  extern __shared__ unsigned long long kv[];
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int i = tid; i < P; i += NT)
    kv[i] = i < frames ? ((unsigned long long)__float_as_uint(key[i]) << 32) | (unsigned)i : ~0ull;
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P; i += NT) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned long long x = kv[i], y = kv[l];
          if ((x > y) == ((i & k) == 0)) {
            kv[i] = y;
            kv[l] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < frames; i += NT) order[i] = (int64_t)(kv[i] & 0xffffffffull);
}

cudaError_t launch_key_order(const float* llr, int n, int64_t frames, float* key, int64_t* order, cudaStream_t st) {
  if (frames <= 0 || frames > kKeyOrderMax) return cudaErrorInvalidValue;
  int P = 1;
  while (P < frames) P <<= 1;
  cudaError_t e = cudaFuncSetAttribute(key_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kKeyOrderMax * 8);
  if (e != cudaSuccess) return e;
  frame_key_kernel<<<(unsigned)frames, 256, 0, st>>>(llr, n, key);
  key_order_kernel<<<1, 1024, (size_t)P * 8, st>>>(key, (int)frames, P, order);
  return cudaGetLastError();
}

// Flooding-schedule kernel for (algorithm, message type, degree bucket,
// threads per block); nullptr where none exists.
const void* flood_kernel_ptr(int algo, int msg16, int dcmax, int threads) {
  switch (algo) {
    case ALGO_MS: return msg16 ? kernel_dc<ALGO_MS, 1>(dcmax, threads) : kernel_dc<ALGO_MS, 0>(dcmax, threads);
    case ALGO_SPA: return msg16 ? kernel_dc<ALGO_SPA, 1>(dcmax, threads) : kernel_dc<ALGO_SPA, 0>(dcmax, threads);
    case ALGO_NMS: return msg16 ? kernel_dc<ALGO_NMS, 1>(dcmax, threads) : kernel_dc<ALGO_NMS, 0>(dcmax, threads);
    case ALGO_SPA_FAST:
      return msg16 ? kernel_dc<ALGO_SPA_FAST, 1>(dcmax, threads) : kernel_dc<ALGO_SPA_FAST, 0>(dcmax, threads);
  }
  return nullptr;
}

}  // namespace gf2c
