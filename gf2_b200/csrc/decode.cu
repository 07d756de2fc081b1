// gf2cuda decode kernels (sm_100a).
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
// Schedules
//   flooding: LdpcDecoder::decode_iterative (crates/gf2-coding/src/ldpc/core.rs:889-938).
//     The reference stores v2c and c2v; here only c2v and the belief are
//     stored and v2c = belief - c2v is formed inside the check node, which is
//     the same IEEE subtraction the reference performs (core.rs:831-836), so
//     messages and beliefs agree bit for bit.  The belief sum runs over the
//     variable's checks in ascending original check index (core.rs:824-827,
//     the CSC order of sparse.rs:297-328).  The syndrome of iteration t is
//     evaluated while the check nodes of iteration t+1 read the beliefs.
//   layered (no reference counterpart): row group by row group, v2c from the
//     pre-layer APP, APP += (c2v_new - c2v_old); a variable with several edges
//     in one row group adds its deltas in ascending circulant shift, ordered by
//     barriers between same-block slots.
#include <cuda_fp16.h>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

enum { ALGO_MS = 0, ALGO_SPA = 1, ALGO_NMS = 2 };

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
  const uint32_t* cg_sync;
  const int* slot_var;
  const uint16_t* chk_cg;
  const int2* vg;
  const int* vg_slot;
};

// Check-node update of one check (slots s0 + i*nchk, i < d).  Reads the current
// APP and the old c2v, writes the new c2v.  Returns the parity of the hard
// decisions of the APP over the check (the syndrome bit of the previous
// iteration).  In the layered schedule the deltas are returned in delta[] and
// the variable indices in var[].
template <int ALGO, int MSG16, int DCMAX, bool LAYERED>
__device__ __forceinline__ int check_update(const FrameCtx& F, int g, int s0, int nchk, int d,
                                            const float* __restrict__ app,
                                            typename MsgIO<MSG16>::T* __restrict__ c2v,
                                            bool first, float al, float be, float* delta,
                                            int* var) {
  typedef MsgIO<MSG16> IO;
  typedef typename MaskOf<DCMAX>::T MaskT;
  int par = 0;
  MaskT neg = 0, real = 0;
  float old[DCMAX];
  if (ALGO == ALGO_MS || ALGO == ALGO_NMS) {
    float m1 = __int_as_float(0x7f800000), m2 = __int_as_float(0x7f800000);
    int i1 = -1;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      var[i] = -1;
      old[i] = 0.0f;
      if (i < d) {
        const int s = s0 + i * nchk;
        const int v = __ldg(&F.slot_var[s]);
        var[i] = v;
        if (v >= 0) {
          const float ap = app[v];
          par ^= (ap < 0.0f);
          const float o = first ? 0.0f : IO::ld(c2v, s);
          old[i] = o;
          const float x = __fsub_rn(ap, o);
          const float ax = fabsf(x);
          if (ax < m1) {
            m2 = m1;
            m1 = ax;
            i1 = i;
          } else if (ax < m2) {
            m2 = ax;
          }
          neg |= (MaskT)(x < 0.0f) << i;
          real |= (MaskT)1 << i;
        }
      }
    }
    const int negp = MaskOf<DCMAX>::popc(neg) & 1;
    const bool single = MaskOf<DCMAX>::popc(real) == 1;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if (i < d && ((real >> i) & 1)) {
        float mag = (i == i1) ? m2 : m1;
        if (single) mag = 0.0f;
        if (ALGO == ALGO_NMS) {
          float dd = __fsub_rn(mag, be);
          dd = dd > 0.0f ? dd : 0.0f;
          mag = __fmul_rn(al, dd);
        }
        const int sg = negp ^ (int)((neg >> i) & 1);
        const float out = sg ? -mag : mag;
        IO::st(c2v, s0 + i * nchk, out);
        if (LAYERED) delta[i] = __fsub_rn(IO::rt(out), old[i]);
      }
    }
  } else {  // sum-product
    float tv[DCMAX];
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      var[i] = -1;
      old[i] = 0.0f;
      tv[i] = 1.0f;
      if (i < d) {
        const int s = s0 + i * nchk;
        const int v = __ldg(&F.slot_var[s]);
        var[i] = v;
        if (v >= 0) {
          const float ap = app[v];
          par ^= (ap < 0.0f);
          const float o = first ? 0.0f : IO::ld(c2v, s);
          old[i] = o;
          tv[i] = tanh_half_f(__fsub_rn(ap, o));
          real |= (MaskT)1 << i;
        }
      }
    }
    const bool single = MaskOf<DCMAX>::popc(real) == 1;
    float suf[DCMAX];
    suf[DCMAX - 1] = 1.0f;
#pragma unroll
    for (int i = DCMAX - 2; i >= 0; i--) suf[i] = (i + 1 < d) ? __fmul_rn(tv[i + 1], suf[i + 1]) : 1.0f;
    float pre = 1.0f;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if (i < d && ((real >> i) & 1)) {
        float p = __fmul_rn(pre, suf[i]);
        p = p > GF2C_SPA_PMAX ? GF2C_SPA_PMAX : (p < -GF2C_SPA_PMAX ? -GF2C_SPA_PMAX : p);
        const float out = single ? 0.0f : two_atanh_f(p);
        IO::st(c2v, s0 + i * nchk, out);
        if (LAYERED) delta[i] = __fsub_rn(IO::rt(out), old[i]);
      }
      if (i < d) pre = (i == 0) ? tv[0] : __fmul_rn(pre, tv[i]);
    }
  }
  return par;
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

template <int ALGO, int MSG16, int SCHED, int DCMAX>
__global__ void __launch_bounds__(1024) bp_decode_kernel(const DecodeArgs a) {
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
    FrameCtx F{C.n, C.m, C.k, C.ncg, C.vgs, C.cg, C.cg_sync, C.slot_var, C.chk_cg, C.vg, C.vg_slot};
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
    float delta[DCMAX];
    int var[DCMAX];
    if (SCHED == 0) {
      for (;;) {
        const int tw = (a.nms_iters > 0) ? min(it, a.nms_iters - 1) : 0;
        int par = 0;
        for (int cc = tid; cc < F.m; cc += NT) {
          const int g = F.chk_cg[cc];
          const int4 G = F.cg[g];
          float al = 1.0f, be = 0.0f;
          if (ALGO == ALGO_NMS) {
            const int lay = (a.nms_L == F.ncg) ? g : 0;
            al = a.alpha[tw * a.nms_L + lay];
            be = a.beta[tw * a.nms_L + lay];
          }
          par |= check_update<ALGO, MSG16, DCMAX, false>(F, g, G.w + (cc - G.x), G.y, G.z, app, c2v,
                                                         it == 0, al, be, delta, var);
        }
        par = __syncthreads_or(par);
        if (it > 0 && a.early_stop && !par) {
          converged = 1;
          synd = 0;
          break;
        }
        // variable nodes: belief = llr + sum c2v, ascending original check index
        for (int base = 0; base < n; base += NT) {
          const int v = base + tid;
          float b = 0.0f;
          if (v < n) {
            const int h = v / F.vgs;
            const int j = v - h * F.vgs;
            const int2 V = F.vg[h];
            b = llr[v];
            const int* sl = F.vg_slot + V.y + j;
            for (int i = 0; i < V.x; i++) {
              const int s = __ldg(&sl[i * F.vgs]);
              if (s < 0) break;
              b = __fadd_rn(b, IO::ld(c2v, s));
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
        synd = syndrome_any(F, bitmap);
        converged = !synd;
      }
    } else {
      for (;;) {
        const int tw = (a.nms_iters > 0) ? min(it, a.nms_iters - 1) : 0;
        for (int g = 0; g < F.ncg; g++) {
          const int4 G = F.cg[g];
          const uint32_t sync = F.cg_sync[g];
          const bool act = tid < G.y;
          float al = 1.0f, be = 0.0f;
          if (ALGO == ALGO_NMS) {
            const int lay = (a.nms_L == F.ncg) ? g : 0;
            al = a.alpha[tw * a.nms_L + lay];
            be = a.beta[tw * a.nms_L + lay];
          }
          if (act)
            check_update<ALGO, MSG16, DCMAX, true>(F, g, G.w + tid, G.y, G.z, app, c2v, it == 0, al,
                                                   be, delta, var);
          __syncthreads();
          if (sync == 0) {
            if (act) {
#pragma unroll
              for (int i = 0; i < DCMAX; i++) {
                if (i < G.z && var[i] >= 0) {
                  const int v = var[i];
                  const float o = app[v];
                  const float nw = __fadd_rn(o, delta[i]);
                  app[v] = nw;
                  if ((o < 0.0f) != (nw < 0.0f)) atomicXor(&bitmap[v >> 5], 1u << (v & 31));
                }
              }
            }
          } else {
#pragma unroll
            for (int i = 0; i < DCMAX; i++) {
              if (i < G.z) {
                if (act && var[i] >= 0) {
                  const int v = var[i];
                  const float o = app[v];
                  const float nw = __fadd_rn(o, delta[i]);
                  app[v] = nw;
                  if ((o < 0.0f) != (nw < 0.0f)) atomicXor(&bitmap[v >> 5], 1u << (v & 31));
                }
                if ((sync >> i) & 1u) __syncthreads();
              }
            }
          }
          __syncthreads();
        }
        ++it;
        synd = syndrome_any(F, bitmap);
        if (a.early_stop && !synd) {
          converged = 1;
          break;
        }
        if (it >= maxit) break;
      }
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

template <int ALGO, int MSG16, int SCHED>
static const void* kernel_dc(int dcmax) {
  switch (dcmax) {
    case 8: return (const void*)bp_decode_kernel<ALGO, MSG16, SCHED, 8>;
    case 16: return (const void*)bp_decode_kernel<ALGO, MSG16, SCHED, 16>;
    case 24: return (const void*)bp_decode_kernel<ALGO, MSG16, SCHED, 24>;
    case 32: return (const void*)bp_decode_kernel<ALGO, MSG16, SCHED, 32>;
    case 64: return (const void*)bp_decode_kernel<ALGO, MSG16, SCHED, 64>;
  }
  return nullptr;
}

template <int ALGO, int MSG16>
static const void* kernel_sched(int sched, int dcmax) {
  return sched == 0 ? kernel_dc<ALGO, MSG16, 0>(dcmax) : kernel_dc<ALGO, MSG16, 1>(dcmax);
}

const void* decode_kernel_ptr(int algo, int msg16, int sched, int dcmax) {
  if (algo == ALGO_MS) return msg16 ? kernel_sched<ALGO_MS, 1>(sched, dcmax) : kernel_sched<ALGO_MS, 0>(sched, dcmax);
  if (algo == ALGO_SPA)
    return msg16 ? kernel_sched<ALGO_SPA, 1>(sched, dcmax) : kernel_sched<ALGO_SPA, 0>(sched, dcmax);
  return msg16 ? kernel_sched<ALGO_NMS, 1>(sched, dcmax) : kernel_sched<ALGO_NMS, 0>(sched, dcmax);
}

int prepare_decode(int algo, int msg16, int sched, int dcmax, size_t smem, int threads, int* blocks_per_sm) {
  const void* k = decode_kernel_ptr(algo, msg16, sched, dcmax);
  if (!k) return set_error(GF2C_ERR_UNSUPPORTED, "no decode kernel for this configuration");
  GF2C_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (blocks_per_sm) {
    int b = 0;
    GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, threads, smem));
    *blocks_per_sm = b;
  }
  return GF2C_OK;
}

int launch_decode(int algo, int msg16, int sched, int dcmax, const DecodeArgs& a, int grid, int threads,
                  size_t smem, cudaStream_t st) {
  const void* k = decode_kernel_ptr(algo, msg16, sched, dcmax);
  if (!k) return set_error(GF2C_ERR_UNSUPPORTED, "no decode kernel for this configuration");
  void* args[] = {(void*)&a};
  GF2C_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(threads), args, smem, st));
  return GF2C_OK;
}

}  // namespace gf2c
