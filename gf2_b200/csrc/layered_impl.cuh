// gf2cuda layered-schedule decoder (sm_100a): device code and kernel templates.
//
// Included by the translation units that instantiate the kernels (one per
// check-node rule and message type, compiled in parallel) and by layered.cu,
// which holds the host-side dispatch.
//
// The layered schedule has no counterpart in the reference (its decoder is the
// flooding loop of crates/gf2-coding/src/ldpc/core.rs:889-938; layered decoding
// is listed as future work in crates/gf2-coding/docs/LDPC_PERFORMANCE.md).  Row
// groups of a QC / DVB-T2 code are processed in order; inside a row group every
// check reads v2c = APP - c2v_old from the pre-layer APP, computes c2v_new and
// adds (c2v_new - c2v_old) to the APP of its variables.
//
// One CTA decodes one frame at a time (persistent, frames from an atomic
// queue), one thread per check of the row group.  The posteriors are kept in
// the u order of the check-state plan (DVB-T2 parity bit k + a + q t at
// k + a Z + t), where every slot of a row group is a rotated run of Z
// consecutive variables: check t reads start + t - (t >= wrap ? Z : 0) from a
// per-(row group, slot) descriptor, so no index table is read in the hot loop
// and every slot load of a warp is coalesced.  All loads of a check are issued back to back from
// always-valid addresses before any arithmetic (memory-level parallelism), and
// then the check node, the message stores and the APP updates follow.
//
// Old messages: the sum-product rules keep one message per edge, a row
// group's messages one contiguous block that a TMA copy stages in shared
// memory while the previous row group is decoded; the min-sum family keeps one
// compressed state per check instead (its two magnitudes, sign bits, argmin),
// read and written by the check's own thread, and one warp has the copy engine
// prefetch into L2 the variable groups (and states) of the next row group.
//
// A row group whose variables are all distinct writes the new APP directly
// from the thread that read it (one barrier per row group); a row group with
// repeated variables (DVB-T2 blocks holding several circulants) applies its
// deltas slot by slot with a barrier between slots of the same block, i.e. in
// ascending circulant shift.
//
// Early stop: the hard decisions live in a shared-memory bitmap that a
// posterior update toggles when its sign flips (one shared atomic, rare after
// the first iterations); at the end of an iteration a syndrome pass over the
// bitmap, row group by row group, stops at the first unsatisfied check.  That
// is the reference's syndrome test (core.rs:918-922) at the cost of one row
// group's bit gathers while a frame is far from a codeword.  (Keeping every
// check's parity up to date on each flip instead, which needs the flipped
// variable's check list from global memory, cost 30 % of the min-sum kernel.)
//
// Check-node rules: min-sum / normalised-offset min-sum / sum-product with the
// exact library numerics (bit-identical to the CPU restatement), and a fast
// sum-product (GF2C_ALGO_SPA_FAST) evaluated with the SFU: e = 2^(-|x| log2 e),
// n = 1 - e, d = 1 + e, N = prod n, D = prod d, and for edge i
//   |c2v_i| = ln((D n_i + N d_i) / (D n_i - N d_i)) = 2 atanh(prod_{j != i} tanh(|x_j| / 2))
// (three SFU operations per edge, no per-edge division of the products); its
// APP update is v2c + c2v_new.
#pragma once
#include <cuda_fp16.h>

#include <type_traits>

#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

enum { L_MS = 0, L_SPA = 1, L_NMS = 2, L_SPA_FAST = 3 };

__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <int MSG16>
__device__ __forceinline__ float ld_msg(const typename MsgIO<MSG16>::T* p, int s);
template <>
__device__ __forceinline__ float ld_msg<0>(const float* p, int s) { return __ldcs(p + s); }
template <>
__device__ __forceinline__ float ld_msg<1>(const __half* p, int s) {
  return __half2float(__ushort_as_half(__ldcs((const unsigned short*)p + s)));
}
template <int MSG16>
__device__ __forceinline__ void st_msg(typename MsgIO<MSG16>::T* p, int s, float v);
template <>
__device__ __forceinline__ void st_msg<0>(float* p, int s, float v) { __stcs(p + s, v); }
template <>
__device__ __forceinline__ void st_msg<1>(__half* p, int s, float v) {
  __stcs((unsigned short*)p + s, __half_as_ushort(__float2half_rn(v)));
}

// Sum-product message of magnitude |v| <= 16.64 (the SFU rows cap it there,
// far inside binary16's range, so the rounding needs no clamp): stores it
// through the message type and returns the rounded value, one conversion for
// both (the result equals st_msg(p, s, IO::rt(v))).
template <int MSG16>
__device__ __forceinline__ float put_capped_msg(typename MsgIO<MSG16>::T* p, int s, float v) {
  if constexpr (MSG16) {
    const __half h = __float2half_rn(v);
    __stcs((unsigned short*)p + s, __half_as_ushort(h));
    return __half2float(h);
  } else {
    __stcs(p + s, v);
    return v;
  }
}

// Old messages of one check: slot i at p[i * nchk] of the (streamed) global
// message array, or at a shared-memory stage that a TMA copy filled.
template <int MSG16>
struct GlobalOld {
  const typename MsgIO<MSG16>::T* p;  // c2v + edge0 + t
  int nchk;
  __device__ __forceinline__ float ld(int i) const { return ld_msg<MSG16>(p, i * nchk); }
};
template <int MSG16>
struct SharedOld {
  uint32_t a;       // shared address of slot 0 of the check
  uint32_t stride;  // bytes between slots (nchk messages)
  __device__ __forceinline__ float ld(int i) const {
    if constexpr (MSG16) {
      unsigned short h;
      asm volatile("ld.shared.u16 %0, [%1];" : "=h"(h) : "r"(a + i * stride));
      return __half2float(__ushort_as_half(h));
    } else {
      float x;
      asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x) : "r"(a + i * stride));
      return x;
    }
  }
};

// Min-sum family (min-sum, normalised / offset min-sum): every message a check
// sends is +-r1 or +-r2 (the two magnitudes rounded through the message type),
// r2 on slot i1 only, so a check keeps one compressed state instead of one
// message per edge: binary16 messages {r1 | r2 << 16, sign bits | i1 << 24}
// (8 bytes, up to 22 slots), FP32 messages {r1, r2, sign bits, i1} (16
// bytes).  Bit i of the sign bits flips slot i's message.  The messages it
// gives back are bit-identical to the per-edge ones.
struct StateOld {
  float r1, r2;
  uint32_t sig;
  int i1;
  __device__ __forceinline__ float ld(int i) const {
    return __uint_as_float(__float_as_uint(i == i1 ? r2 : r1) ^ (((sig >> i) & 1u) << 31));
  }
};
template <int MSG16>
__device__ __forceinline__ StateOld load_state(const void* cst, int ci) {
  if constexpr (MSG16) {
    const uint2 v = __ldcs((const uint2*)cst + ci);
    return StateOld{__half2float(__ushort_as_half((unsigned short)(v.x & 0xffffu))),
                    __half2float(__ushort_as_half((unsigned short)(v.x >> 16))), v.y & 0xffffffu,
                    (int)(v.y >> 24) == 31 ? -1 : (int)(v.y >> 24)};
  } else {
    const uint4 v = __ldcs((const uint4*)cst + ci);
    return StateOld{__uint_as_float(v.x), __uint_as_float(v.y), v.z, (int)v.w};
  }
}
// r1, r2 already rounded through the message type; i1 = -1: no slot takes r2
template <int MSG16>
__device__ __forceinline__ void store_state(void* cst, int ci, float r1, float r2, uint32_t sig, int i1) {
  if constexpr (MSG16) {
    const uint32_t h1 = __half_as_ushort(__float2half_rn(r1)), h2 = __half_as_ushort(__float2half_rn(r2));
    __stcs((uint2*)cst + ci, make_uint2(h1 | (h2 << 16), sig | ((uint32_t)(i1 & 31) << 24)));
  } else {
    __stcs((uint4*)cst + ci, make_uint4(__float_as_uint(r1), __float_as_uint(r2), sig, (uint32_t)i1));
  }
}

// TMA (bulk copy engine) helpers: a 1-D global -> shared copy whose bytes an
// mbarrier counts, and bounded waits on the mbarrier's phase.
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Every wait is bounded in time (the global nanosecond timer): a copy that
// never lands makes the kernel report an error and stop instead of spinning.
constexpr unsigned long long kStageWaitNs = 2000000000ull;
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kStageWaitNs) return false;
  }
}
__device__ __forceinline__ void tma_load_1d(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
// Bulk prefetch of [p, p + bytes) into L2 (no shared memory, no completion to
// wait for); the range is widened to 16-byte boundaries.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  const uintptr_t a = (uintptr_t)p & ~(uintptr_t)15;
  const uint32_t n = (uint32_t)(((uintptr_t)p + bytes - a + 15) & ~(uintptr_t)15);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
}

// Shared-memory message stage of the layered kernel: two buffers of one row
// group's messages each (the row group being decoded and the next one, whose
// old messages a TMA copy brings in meanwhile) and one mbarrier per buffer.
struct Stage {
  uint32_t buf;     // shared address of buffer 0; buffer b at buf + b * bytes
  uint32_t bytes;   // bytes per buffer
  uint32_t bar;     // shared address of mbarrier 0 (mbarrier b at bar + 8 b)
  uint32_t phase;   // bit b: parity of the next completion of mbarrier b
  uint32_t step;    // row groups decoded so far (buffer of a row group = step & 1)
  bool pending;     // a copy was issued that no row group has consumed yet
};

struct LayerSmem {
  uint32_t* bitmap;   // hard decisions, n bits
  float* dbuf;        // slots x checks of a row group: old messages / deltas (nullptr: none)
};

// u-order variable of slot descriptor D = {start, wrap} for check t of a row
// group of Z checks (every result is a valid index; a slot without an edge at
// t = 0 is masked separately).
__device__ __forceinline__ int slot_u(const int2 D, int t, int Z) { return D.x + t - (t >= D.y ? Z : 0); }

// A hard decision flipped: toggle its bit (the bitmap is the syndrome pass's
// input at the end of the iteration).
__device__ __forceinline__ void flip_var(int u, const LayerSmem& S) { atomicXor(&S.bitmap[u >> 5], 1u << (u & 31)); }

__device__ __forceinline__ void app_put(float* app, int v, bool old_neg, float nw, const LayerSmem& S) {
  app[v] = nw;
  if (old_neg != (nw < 0.0f)) flip_var(v, S);
}

// Syndrome of the hard decisions in the bitmap: true when every check is
// satisfied (the reference's test, core.rs:918-922).  Row groups in order, the
// CTA's threads over the checks of a row group, one barrier per row group; the
// pass stops at the first row group with an unsatisfied check, so a frame that
// is still far from a codeword pays one row group.  Every thread returns after
// the same barrier.
template <int DCMAX>
__device__ __forceinline__ bool syndrome_zero(const DevCode& C, const uint32_t* bitmap) {
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int g = 0; g < C.ncg; g++) {
    const int4 G = C.sp_cg[g];  // {first check, checks, slots, first slot descriptor}
    const int2* __restrict__ sd = C.sp_desc + G.w;
    const uint32_t ab0 = __ldg(&C.sp_absent[g]);
    uint32_t bad = 0;
    for (int t = tid; t < G.y; t += NT) {
      const uint32_t keep = (t == 0) ? ~ab0 : ~0u;  // slots without an edge at t = 0
      uint32_t p = 0;
#pragma unroll
      for (int i = 0; i < DCMAX; i++) {
        if (i < G.z) {
          const int u = slot_u(__ldg(&sd[i]), t, G.y);
          p ^= (bitmap[u >> 5] >> (u & 31)) & (keep >> i);
        }
      }
      bad |= p & 1u;
    }
    if (__syncthreads_or(bad)) return false;
  }
  return true;
}

// Fast sum-product update of check t of a row group whose D slots all hold an
// edge and whose variables are all distinct (the common case): loads, check
// node, message stores and posterior updates in one pass; flipped hard
// decisions are collected in a mask and handled after the loop (one call
// site).  Same arithmetic as the general path of bp_layered_kernel.  PART:
// the row group has d < D slots; slots d..D-1 take a neutral input (e = 0,
// positive, as the general path's missing edges) and store nothing.
template <int MSG16, int D, bool PART, class OM>
__device__ __forceinline__ void spa_fast_row(const int2* __restrict__ sd, int t, int nchk, int s0, float* app,
                                             typename MsgIO<MSG16>::T* __restrict__ c2v, const OM& om, bool first,
                                             const LayerSmem& S, int d) {
  float x[D], e[D];
#pragma unroll
  for (int i = 0; i < D; i++) x[i] = (!PART || i < d) ? app[slot_u(__ldg(&sd[i]), t, nchk)] : 3.402823466e38f;
  uint32_t neg = 0, apneg = 0;
#pragma unroll
  for (int i = 0; i < D; i++) apneg |= (uint32_t)(x[i] < 0.0f) << i;
  if (!first) {
#pragma unroll
    for (int i = 0; i < D; i++)
      if (!PART || i < d) x[i] = __fsub_rn(x[i], om.ld(i));
  }
  float N = 1.0f, Dp = 1.0f;
#pragma unroll
  for (int i = 0; i < D; i++) {
    neg |= (uint32_t)(x[i] < 0.0f) << i;
    e[i] = ex2_approx(fabsf(x[i]) * -1.4426950408889634f);
    N *= fmaxf(1.0f - e[i], 5.9604645e-08f);
    Dp = __fmaf_rn(Dp, e[i], Dp);
  }
  const uint32_t negp = __popc(neg) & 1u;
  uint32_t flips = 0;
#pragma unroll
  for (int i = 0; i < D; i++) {
    const float ni = fmaxf(1.0f - e[i], 5.9604645e-08f), di = 1.0f + e[i];
    const float num = __fmaf_rn(Dp, ni, N * di);
    const float den = fmaxf(__fmaf_rn(Dp, ni, -N * di), num * 5.9604645e-08f);
    const float mag = fminf(0.69314718055994531f * lg2_approx(num * rcp_approx(den)), 16.635532f);
    if (!PART || i < d) {
      const float out = put_capped_msg<MSG16>(c2v, s0 + i * nchk, (negp ^ ((neg >> i) & 1u)) ? -mag : mag);
      const float nw = x[i] + out;
      app[slot_u(__ldg(&sd[i]), t, nchk)] = nw;
      flips |= (uint32_t)(((apneg >> i) & 1u) != (uint32_t)(nw < 0.0f)) << i;
    }
  }
  while (flips) {  // rare after the first iterations
    const int i = __ffs(flips) - 1;
    flips &= flips - 1;
    flip_var(slot_u(__ldg(&sd[i]), t, nchk), S);
  }
}

// Fast sum-product update of check t of a row group with repeated variables
// (an info block holding several circulants: runs of consecutive slots of the
// same block, marked by the sync bits).  Phase A: the same check node as
// spa_fast_row; dbuf[i * nchk + t] receives the old message, then the delta
// c2v_new - c2v_old; slots outside the runs update their (unique) variable
// now, APP_old + delta.  Phase B, after a barrier: the thread of the first
// slot of each run adds the run's deltas to its variable in slot order
// (ascending circulant shift).  The result is the one of the slot-by-slot
// update with a barrier between the slots of a block, with one barrier.
template <int MSG16, int D, bool PART, class OM>
__device__ __forceinline__ void spa_fast_rep_a(const int2* __restrict__ sd, int t, int nchk, int s0, float* app,
                                               typename MsgIO<MSG16>::T* __restrict__ c2v, const OM& om, bool first,
                                               uint32_t sync, float* dbuf, const LayerSmem& S,
                                               int d) {
  const uint32_t rep = sync | (sync << 1);  // slots inside a run
  float x[D], e[D];
#pragma unroll
  for (int i = 0; i < D; i++) x[i] = (!PART || i < d) ? app[slot_u(__ldg(&sd[i]), t, nchk)] : 3.402823466e38f;
#pragma unroll
  for (int i = 0; i < D; i++) {
    if (!PART || i < d) {
      const float o = first ? 0.0f : om.ld(i);
      dbuf[i * nchk + t] = o;
      if (!first) x[i] = __fsub_rn(x[i], o);
    }
  }
  uint32_t neg = 0;
  float N = 1.0f, Dp = 1.0f;
#pragma unroll
  for (int i = 0; i < D; i++) {
    neg |= (uint32_t)(x[i] < 0.0f) << i;
    e[i] = ex2_approx(fabsf(x[i]) * -1.4426950408889634f);
    N *= fmaxf(1.0f - e[i], 5.9604645e-08f);
    Dp = __fmaf_rn(Dp, e[i], Dp);
  }
  const uint32_t negp = __popc(neg) & 1u;
#pragma unroll
  for (int i = 0; i < D; i++) {
    const float ni = fmaxf(1.0f - e[i], 5.9604645e-08f), di = 1.0f + e[i];
    const float num = __fmaf_rn(Dp, ni, N * di);
    const float den = fmaxf(__fmaf_rn(Dp, ni, -N * di), num * 5.9604645e-08f);
    const float mag = fminf(0.69314718055994531f * lg2_approx(num * rcp_approx(den)), 16.635532f);
    if (!PART || i < d) {
      const float out = put_capped_msg<MSG16>(c2v, s0 + i * nchk, (negp ^ ((neg >> i) & 1u)) ? -mag : mag);
      const float delta = out - dbuf[i * nchk + t];
      if ((rep >> i) & 1u) {
        dbuf[i * nchk + t] = delta;
      } else {
        const int v = slot_u(__ldg(&sd[i]), t, nchk);
        const float ov = app[v];
        app_put(app, v, ov < 0.0f, __fadd_rn(ov, delta), S);
      }
    }
  }
}

template <int D>
__device__ __forceinline__ void spa_fast_rep_b(const int2* __restrict__ sd, int t, int nchk, float* app,
                                               uint32_t sync, const float* dbuf, const LayerSmem& S) {
#pragma unroll
  for (int i = 0; i < D; i++) {
    const bool head = ((sync >> i) & 1u) && !(i > 0 && ((sync >> (i - 1)) & 1u));
    if (head) {
      const int v = slot_u(__ldg(&sd[i]), t, nchk);
      const float ov = app[v];
      float nw = __fadd_rn(ov, dbuf[i * nchk + t]);
      for (int j = i + 1; j < D && ((sync >> (j - 1)) & 1u); j++) {
        int tj = v - __ldg(&sd[j]).x;  // the check of slot j that holds v
        if (tj < 0) tj += nchk;
        nw = __fadd_rn(nw, dbuf[j * nchk + tj]);
      }
      app_put(app, v, ov < 0.0f, nw, S);
    }
  }
}

// Min-sum / normalised-offset min-sum update of check t of a row group whose D
// slots all hold an edge and whose variables are all distinct: loads, check
// node, message stores and posterior updates in one pass, with the arithmetic
// of the general path of layered_iterations (v2c = APP - c2v_old, min1 / min2
// / first argmin, sign parity, sign * alpha * max(min - beta, 0), the stored
// message rounded through the message type, APP + (c2v_new - c2v_old)), so
// results are bit-identical.  PART: the row group has d < D slots; slots
// d..D-1 are absent (no load, no store).
template <int ALGO, int MSG16, int D, bool PART, class OM, bool ST = false>
__device__ __forceinline__ void ms_row(const int2* __restrict__ sd, int t, int nchk, int s0, float* app,
                                       typename MsgIO<MSG16>::T* __restrict__ c2v, const OM& om, bool first,
                                       float al, float be,
                                       const LayerSmem& S, int d, int ci = 0) {
  typedef MsgIO<MSG16> IO;
  float ap[D], o[D];
#pragma unroll
  for (int i = 0; i < D; i++) ap[i] = (!PART || i < d) ? app[slot_u(__ldg(&sd[i]), t, nchk)] : 0.0f;
#pragma unroll
  for (int i = 0; i < D; i++) o[i] = (first || (PART && i >= d)) ? 0.0f : om.ld(i);
  float m1 = __int_as_float(0x7f800000), m2 = m1;
  int i1 = -1;
  uint32_t neg = 0, apneg = 0;
#pragma unroll
  for (int i = 0; i < D; i++) {
    if (PART && i >= d) continue;
    const float w = __fsub_rn(ap[i], o[i]);
    const float ax = fabsf(w);
    // the two smallest magnitudes and the first argmin, branch-free (a NaN
    // magnitude changes none of them, as with the comparisons of the rule)
    i1 = (ax < m1) ? i : i1;
    m2 = fmaxf(m1, fminf(m2, ax));
    m1 = fminf(m1, ax);
    neg |= (uint32_t)(w < 0.0f) << i;
    apneg |= (uint32_t)(ap[i] < 0.0f) << i;
  }
  float mag1 = m1, mag2 = m2;  // d >= 2 edges: never a single-edge check
  if (ALGO == L_NMS) {
    const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
    mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
    mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
  }
  // every message is +-mag1 or +-mag2: round the two through the message type
  // once (the rounding is odd-symmetric, so the sign can follow)
  const float r1 = IO::rt(mag1), r2 = IO::rt(mag2);
  const uint32_t negp = __popc(neg) & 1u;
  uint32_t flips = 0;
#pragma unroll
  for (int i = 0; i < D; i++) {
    if (PART && i >= d) continue;
    const uint32_t sflip = ((neg >> i) ^ negp) & 1u;
    const float out = __uint_as_float(__float_as_uint((i == i1) ? r2 : r1) ^ (sflip << 31));
    if constexpr (ST) {
      // one compressed state per check, stored after the loop
    } else if constexpr (MSG16) {
      const uint32_t h = (i == i1) ? __half_as_ushort(__float2half_rn(r2)) : __half_as_ushort(__float2half_rn(r1));
      __stcs((unsigned short*)c2v + s0 + i * nchk, (unsigned short)(h ^ (sflip << 15)));
    } else {
      st_msg<MSG16>(c2v, s0 + i * nchk, out);
    }
    const float nw = __fadd_rn(ap[i], __fsub_rn(out, o[i]));
    app[slot_u(__ldg(&sd[i]), t, nchk)] = nw;
    flips |= (uint32_t)(((apneg >> i) & 1u) != (uint32_t)(nw < 0.0f)) << i;
  }
  if constexpr (ST) {
    const uint32_t real = PART ? ((1u << d) - 1u) : (uint32_t)((1ull << D) - 1ull);
    store_state<MSG16>(c2v, ci, r1, r2, (neg ^ (0u - negp)) & real, i1);
  }
  while (flips) {  // rare after the first iterations
    const int i = __ffs(flips) - 1;
    flips &= flips - 1;
    flip_var(slot_u(__ldg(&sd[i]), t, nchk), S);
  }
}

// Phase A of a min-sum / normalised-offset min-sum row group with repeated
// variables (the counterpart of spa_fast_rep_a): the same check node as
// ms_row; slots inside a run of one block leave their delta in dbuf for phase
// B (spa_fast_rep_b, after one barrier), the other slots update their unique
// variable now.  Same additions in the same order as the slot-by-slot general
// path, so results are bit-identical.
template <int ALGO, int MSG16, int D, bool PART, class OM, bool ST = false>
__device__ __forceinline__ void ms_rep_a(const int2* __restrict__ sd, int t, int nchk, int s0, float* app,
                                         typename MsgIO<MSG16>::T* __restrict__ c2v, const OM& om, bool first,
                                         float al, float be,
                                         uint32_t sync, float* dbuf, const LayerSmem& S, int d, int ci = 0) {
  typedef MsgIO<MSG16> IO;
  const uint32_t rep = sync | (sync << 1);  // slots inside a run
  float ap[D], o[D];
#pragma unroll
  for (int i = 0; i < D; i++) ap[i] = (!PART || i < d) ? app[slot_u(__ldg(&sd[i]), t, nchk)] : 0.0f;
#pragma unroll
  for (int i = 0; i < D; i++) o[i] = (first || (PART && i >= d)) ? 0.0f : om.ld(i);
  float m1 = __int_as_float(0x7f800000), m2 = m1;
  int i1 = -1;
  uint32_t neg = 0;
#pragma unroll
  for (int i = 0; i < D; i++) {
    if (PART && i >= d) continue;
    const float w = __fsub_rn(ap[i], o[i]);
    const float ax = fabsf(w);
    if (ax < m1) {
      m2 = m1;
      m1 = ax;
      i1 = i;
    } else if (ax < m2) {
      m2 = ax;
    }
    neg |= (uint32_t)(w < 0.0f) << i;
  }
  float mag1 = m1, mag2 = m2;
  if (ALGO == L_NMS) {
    const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
    mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
    mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
  }
  const uint32_t negp = __popc(neg) & 1u;
#pragma unroll
  for (int i = 0; i < D; i++) {
    if (PART && i >= d) continue;
    const float mag = (i == i1) ? mag2 : mag1;
    const float out = IO::rt((negp ^ ((neg >> i) & 1u)) ? -mag : mag);
    if constexpr (!ST) st_msg<MSG16>(c2v, s0 + i * nchk, out);
    const float delta = __fsub_rn(out, o[i]);
    if ((rep >> i) & 1u) {
      dbuf[i * nchk + t] = delta;
    } else {
      const int v = slot_u(__ldg(&sd[i]), t, nchk);
      app_put(app, v, ap[i] < 0.0f, __fadd_rn(ap[i], delta), S);
    }
  }
  if constexpr (ST) {
    const uint32_t real = PART ? ((1u << d) - 1u) : (uint32_t)((1ull << D) - 1ull);
    store_state<MSG16>(c2v, ci, IO::rt(mag1), IO::rt(mag2), (neg ^ (0u - negp)) & real, i1);
  }
}

// General check update (any algorithm, absent slots, repeated variables):
// 1. indices, 2. all loads, 3. arithmetic, 4. message stores.  With
// `direct` (a row group without repeated variables) the posteriors are
// updated here; otherwise the deltas to add (slot order) are returned in wd[]
// with the slot's variable in vd[] (-1: no edge).
template <int ALGO, int MSG16, int DCMAX, class OM, bool ST = false>
__device__ __forceinline__ void general_row(const DecodeArgs& a, const int2* __restrict__ sd, int t, int nchk, int s0,
                                            float* app, typename MsgIO<MSG16>::T* __restrict__ c2v, const OM& om,
                                            bool first, int d, uint32_t ab, bool direct, float al, float be,
                                            const LayerSmem& S, float (&wd)[DCMAX],
                                            int (&vv)[DCMAX], int ci = 0) {
  typedef MsgIO<MSG16> IO;
  float smag1 = 0.0f, smag2 = 0.0f;  // min-sum family: the check's two magnitudes and argmin
  int si1 = -1;
  float ap[DCMAX], o[DCMAX], w[DCMAX];
  uint32_t real = 0, neg = 0, apneg = 0;
#pragma unroll
  for (int i = 0; i < DCMAX; i++) vv[i] = (i < d && !((ab >> i) & 1u)) ? slot_u(__ldg(&sd[i]), t, nchk) : -1;
#pragma unroll
  for (int i = 0; i < DCMAX; i++) ap[i] = app[vv[i] < 0 ? 0 : vv[i]];
  if (first) {
#pragma unroll
    for (int i = 0; i < DCMAX; i++) o[i] = 0.0f;
  } else {
#pragma unroll
    for (int i = 0; i < DCMAX; i++) o[i] = om.ld(i < d ? i : 0);
  }
#pragma unroll
  for (int i = 0; i < DCMAX; i++) {
    const bool r = vv[i] >= 0;
    w[i] = __fsub_rn(ap[i], o[i]);  // v2c
    real |= (uint32_t)r << i;
    neg |= (uint32_t)(r && w[i] < 0.0f) << i;
    apneg |= (uint32_t)(ap[i] < 0.0f) << i;
  }
  const int negp = __popc(neg) & 1;
  const bool single = __popc(real) == 1;
  if (ALGO == L_MS || ALGO == L_NMS) {
    float m1 = __int_as_float(0x7f800000), m2 = m1;
    int i1 = -1;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float ax = ((real >> i) & 1u) ? fabsf(w[i]) : __int_as_float(0x7f800000);
      if (ax < m1) {
        m2 = m1;
        m1 = ax;
        i1 = i;
      } else if (ax < m2) {
        m2 = ax;
      }
    }
    float mag1 = single ? 0.0f : m1, mag2 = single ? 0.0f : m2;
    if (ALGO == L_NMS) {
      const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
      mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
      mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
    }
    smag1 = mag1;
    smag2 = mag2;
    si1 = i1;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float mag = (i == i1) ? mag2 : mag1;
      w[i] = (negp ^ ((neg >> i) & 1u)) ? -mag : mag;
    }
  } else if (ALGO == L_SPA) {
    float suf[DCMAX];
#pragma unroll
    for (int i = 0; i < DCMAX; i++) w[i] = ((real >> i) & 1u) ? tanh_half_f(w[i]) : 1.0f;
    suf[DCMAX - 1] = 1.0f;
#pragma unroll
    for (int i = DCMAX - 2; i >= 0; i--) suf[i] = (i + 1 < d) ? __fmul_rn(w[i + 1], suf[i + 1]) : 1.0f;
    float pre = 1.0f;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      float p = __fmul_rn(pre, suf[i]);
      p = p > GF2C_SPA_PMAX ? GF2C_SPA_PMAX : (p < -GF2C_SPA_PMAX ? -GF2C_SPA_PMAX : p);
      const float out = single ? 0.0f : two_atanh_f(p);
      if (i < d) pre = (i == 0) ? w[0] : __fmul_rn(pre, w[i]);
      w[i] = out;
    }
  } else {  // fast sum-product; ap[] keeps v2c for the APP update
    float N = 1.0f, Dp = 1.0f;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float x = w[i];
      ap[i] = x;
      const float e = ((real >> i) & 1u) ? ex2_approx(fabsf(x) * -1.4426950408889634f) : 0.0f;
      w[i] = e;
      N *= fmaxf(1.0f - e, 5.9604645e-08f);
      Dp = __fmaf_rn(Dp, e, Dp);
    }
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      const float ni = fmaxf(1.0f - w[i], 5.9604645e-08f), di = 1.0f + w[i];
      const float num = __fmaf_rn(Dp, ni, N * di);
      const float den = fmaxf(__fmaf_rn(Dp, ni, -N * di), num * 5.9604645e-08f);
      float mag = 0.69314718055994531f * lg2_approx(num * rcp_approx(den));
      mag = single ? 0.0f : fminf(mag, 16.635532f);
      w[i] = (negp ^ ((neg >> i) & 1u)) ? -mag : mag;
    }
  }
  // message stores; APP update for row groups without repeated variables
#pragma unroll
  for (int i = 0; i < DCMAX; i++) {
    wd[i] = 0.0f;
    if ((real >> i) & 1u) {
      const float out = IO::rt(w[i]);
      if constexpr (!ST) st_msg<MSG16>(c2v, s0 + i * nchk, out);
      if (ALGO == L_SPA_FAST) {
        if (direct) app_put(app, vv[i], (apneg >> i) & 1u, ap[i] + out, S);
        else wd[i] = out - o[i];
      } else {
        const float dl = __fsub_rn(out, o[i]);  // delta
        if (direct) app_put(app, vv[i], (apneg >> i) & 1u, __fadd_rn(ap[i], dl), S);
        else wd[i] = dl;
      }
    }
  }
  if constexpr (ST) store_state<MSG16>(c2v, ci, IO::rt(smag1), IO::rt(smag2), (neg ^ (0u - (uint32_t)negp)) & real, si1);
}

// Iterations of one frame with row groups of at most DCMAX slots; returns the
// iteration count and whether the syndrome test passed at an early stop.
//
// STG: the old messages of each row group are read from a shared-memory stage
// instead of global memory.  While row group g is decoded, one thread has a
// TMA bulk copy bring the old messages of the next row group (of the next
// iteration after the last row group) into the other buffer; every thread
// waits on that buffer's mbarrier (bounded) before reading it.  New messages
// are stored to global memory by the threads as before, each thread ordering
// its stores before later TMA reads of them with a proxy fence.  A wait that
// runs out sets the status word to 2 and *abort, and the kernel returns.
// MULTI: a kernel of fewer threads than checks in a row group (several checks
// per thread); without it each thread has at most one check, and the loops
// over a thread's checks run at most once.
template <int ALGO, int MSG16, int DCMAX, bool STG, bool MULTI>
__device__ __forceinline__ void layered_iterations(const DecodeArgs& a, const DevCode& C, float* app,
                                                   typename MsgIO<MSG16>::T* __restrict__ c2v, const LayerSmem& S,
                                                   int maxit, int& it, int& converged, Stage& stg, int* abort) {
  typedef MsgIO<MSG16> IO;
  const int tid = threadIdx.x, ncg = C.ncg;
  // stride of the loops over a thread's checks (one pass without MULTI)
  const int NT = MULTI ? (int)blockDim.x : (1 << 30);
  const int4* __restrict__ cgp = C.cg;
  const int4* __restrict__ spcg = C.sp_cg;
  const uint32_t* __restrict__ cgs = C.cg_sync;
  const int2* __restrict__ sdesc = C.sp_desc;
  const uint32_t* __restrict__ absent = C.sp_absent;
  it = 0;
  converged = 0;
  // fused row paths: every algorithm but the exact sum-product
  constexpr bool kFused = (ALGO == L_SPA_FAST || ALGO == L_MS || ALGO == L_NMS) && DCMAX <= 22;
  constexpr int kMsgBytes = MSG16 ? 2 : 4;
  // the min-sum family on the single-code (staged) kernels keeps one compressed
  // state per check (flattened check index) instead of per-edge messages, read
  // and written by the check's thread; nothing is staged
  constexpr bool ST = layered_state_mode(ALGO, DCMAX, STG);
  const bool pf = __isGlobal(app);  // posteriors in the workspace (not on chip)
  for (;;) {
    const int tw = (a.nms_iters > 0) ? min(it, a.nms_iters - 1) : 0;
    const bool first = (it == 0);
    for (int g = 0; g < ncg; g++) {
      const int4 G = cgp[g];
      const uint32_t sync = cgs[g];
      const bool act = tid < G.y;
      const int d = G.z, nchk = G.y;
      const int t = act ? tid : 0;
      const int s0 = G.w + t;
      const int2* __restrict__ sd = sdesc + spcg[g].w;
      const int c0 = spcg[g].x;  // flattened index of the row group's first check
      typedef typename std::conditional<
          ST, StateOld, typename std::conditional<STG, SharedOld<MSG16>, GlobalOld<MSG16>>::type>::type OM;
      OM om;
      if constexpr (ST) {
        om = (act && !first) ? load_state<MSG16>(c2v, c0 + t) : StateOld{};
      } else if constexpr (STG) {
        const uint32_t b = stg.step & 1u;
        if (!first) {  // this row group's old messages: wait for the copy into buffer b
          if (!mbar_wait_bounded(stg.bar + 8 * b, (stg.phase >> b) & 1u)) {
            *abort = 1;
            atomicExch(a.status, 2);
          }
          stg.phase ^= 1u << b;
          stg.pending = false;
        }
        // the next row group's old messages (the next iteration's first after the last)
        const bool issue = (g + 1 < ncg) ? !first : (it + 1 < maxit);
        if (issue) {
          const int gn = (g + 1 < ncg) ? g + 1 : 0;
          if (tid == 0) {
            const int4 Gn = cgp[gn];
            const uint32_t nb = b ^ 1u, bytes = (uint32_t)(Gn.z * Gn.y * kMsgBytes);
            fence_proxy_async_shared();  // the buffer's last reads (previous row group) before the copy
            mbar_expect_tx(stg.bar + 8 * nb, bytes);
            tma_load_1d(stg.buf + nb * stg.bytes, c2v + Gn.w, bytes, stg.bar + 8 * nb);
          }
          stg.pending = true;
        }
        om = OM{stg.buf + b * stg.bytes + (uint32_t)(t * kMsgBytes), (uint32_t)(nchk * kMsgBytes)};
      } else {
        om = OM{c2v + s0, nchk};
      }
      // Several checks per thread, posteriors in the workspace and no message
      // stage running on the copy engine: the next row group's slots each read
      // one whole variable group (Z consecutive posteriors); lane i of the last
      // warp has slot i's group (lane 31: the compressed states of the row
      // group) prefetched into L2, so that those gathers wait on L2 rather than
      // DRAM.  (With one check per thread, issued by one thread in a loop, or
      // next to the sum-product stage copies, it was slower.)
      if constexpr ((!STG || ST) && MULTI) {
        if (pf && (tid >> 5) == ((int)blockDim.x >> 5) - 1) {  // lane i of the last warp: slot i
          const int lane = tid & 31;
          const int gn = (g + 1 < ncg) ? g + 1 : 0;
          const int4 Gn = spcg[gn];
          if (lane < Gn.z) {
            const int2 D = __ldg(&sdesc[Gn.w + lane]);
            prefetch_l2(app + (D.x + D.y - Gn.y), (uint32_t)Gn.y * 4u);
          } else if (ST && lane == 31) {
            prefetch_l2((const char*)c2v + (size_t)Gn.x * (MSG16 ? 8 : 16), (uint32_t)Gn.y * (MSG16 ? 8u : 16u));
          }
        }
      }
      // row group with repeated variables, all slots real everywhere: one barrier
      // (fewer slots than DCMAX: the PART variants)
      const bool rep_row = kFused && S.dbuf != nullptr && sync != 0 && d >= 2 && d <= DCMAX &&
                           __ldg(&absent[g]) == 0u;
      float al = 1.0f, be = 0.0f;
      if (ALGO == L_NMS) {
        const int lay = (a.nms_L == ncg) ? g : 0;
        al = __ldg(&a.alpha[tw * a.nms_L + lay]);
        be = __ldg(&a.beta[tw * a.nms_L + lay]);
      }
      // old-message reader of check tc of this row group
      auto old_of = [&](int tc) -> OM {
        if constexpr (ST)
          return first ? StateOld{} : load_state<MSG16>(c2v, c0 + tc);
        else if constexpr (STG)
          return OM{om.a + (uint32_t)((tc - t) * kMsgBytes), om.stride};
        else
          return OM{c2v + G.w + tc, nchk};
      };
      if (rep_row) {
        for (int tc = tid; tc < nchk; tc += NT) {
          const OM omc = old_of(tc);
          const int sc = G.w + tc;
          if constexpr (ALGO == L_SPA_FAST) {
            if (d == DCMAX)
              spa_fast_rep_a<MSG16, DCMAX, false>(sd, tc, nchk, sc, app, c2v, omc, first, sync, S.dbuf, S, d);
            else
              spa_fast_rep_a<MSG16, DCMAX, true>(sd, tc, nchk, sc, app, c2v, omc, first, sync, S.dbuf, S, d);
          } else if constexpr (kFused) {
            if (d == DCMAX)
              ms_rep_a<ALGO, MSG16, DCMAX, false, OM, ST>(sd, tc, nchk, sc, app, c2v, omc, first, al, be, sync, S.dbuf, S,
                                                     d, c0 + tc);
            else
              ms_rep_a<ALGO, MSG16, DCMAX, true, OM, ST>(sd, tc, nchk, sc, app, c2v, omc, first, al, be, sync, S.dbuf, S,
                                                    d, c0 + tc);
          }
        }
        __syncthreads();
        for (int tc = tid; tc < nchk; tc += NT) spa_fast_rep_b<DCMAX>(sd, tc, nchk, app, sync, S.dbuf, S);
      } else if (sync == 0) {
        for (int tc = tid; tc < nchk; tc += NT) {
          const OM omc = old_of(tc);
          const int sc = G.w + tc;
          const uint32_t ab = (tc == 0) ? __ldg(&absent[g]) : 0u;
          if (kFused && d >= 2 && d <= DCMAX && ab == 0) {
            if constexpr (ALGO == L_SPA_FAST) {
              if (d == DCMAX)
                spa_fast_row<MSG16, DCMAX, false>(sd, tc, nchk, sc, app, c2v, omc, first, S, d);
              else
                spa_fast_row<MSG16, DCMAX, true>(sd, tc, nchk, sc, app, c2v, omc, first, S, d);
            } else if constexpr (kFused) {
              if (d == DCMAX)
                ms_row<ALGO, MSG16, DCMAX, false, OM, ST>(sd, tc, nchk, sc, app, c2v, omc, first, al, be, S, d,
                                                          c0 + tc);
              else
                ms_row<ALGO, MSG16, DCMAX, true, OM, ST>(sd, tc, nchk, sc, app, c2v, omc, first, al, be, S, d,
                                                         c0 + tc);
            }
          } else {
            float wd[DCMAX];
            int vd[DCMAX];
            general_row<ALGO, MSG16, DCMAX, OM, ST>(a, sd, tc, nchk, sc, app, c2v, omc, first, d, ab, true, al, be, S, wd,
                                                   vd, c0 + tc);
          }
        }
      } else if (!MULTI || NT >= nchk) {
        // repeated variables (general path, one check per thread): deltas in
        // registers, applied slot by slot with a barrier after each repeated block slot
        float wd[DCMAX];
        int vd[DCMAX];
        if (act) {
          const uint32_t ab = (t == 0) ? __ldg(&absent[g]) : 0u;
          general_row<ALGO, MSG16, DCMAX, OM, ST>(a, sd, t, nchk, s0, app, c2v, om, first, d, ab, false, al, be, S, wd, vd,
                                                 c0 + t);
        }
        __syncthreads();  // all pre-layer APP reads done
#pragma unroll
        for (int i = 0; i < DCMAX; i++) {
          if (i < d) {
            if (act && vd[i] >= 0) {
              const int v = vd[i];
              const float ov = app[v];
              app_put(app, v, ov < 0.0f, __fadd_rn(ov, wd[i]), S);
            }
            if ((sync >> i) & 1u) __syncthreads();
          }
        }
      } else {
        // repeated variables, several checks per thread: deltas in the shared
        // buffer (slot i of check tc at dbuf[i * nchk + tc], NaN-free; absent
        // slots hold nothing and are skipped), then applied slot by slot
        for (int tc = tid; tc < nchk; tc += NT) {
          float wd[DCMAX];
          int vd[DCMAX];
          const uint32_t ab = (tc == 0) ? __ldg(&absent[g]) : 0u;
          general_row<ALGO, MSG16, DCMAX, OM, ST>(a, sd, tc, nchk, G.w + tc, app, c2v, old_of(tc), first, d, ab, false,
                                                 al, be, S, wd, vd, c0 + tc);
#pragma unroll
          for (int i = 0; i < DCMAX; i++)
            if (i < d && vd[i] >= 0) S.dbuf[i * nchk + tc] = wd[i];
        }
        __syncthreads();  // all pre-layer APP reads done
        for (int i = 0; i < d; i++) {
          for (int tc = tid; tc < nchk; tc += NT) {
            const uint32_t ab = (tc == 0) ? __ldg(&absent[g]) : 0u;
            if ((ab >> i) & 1u) continue;
            const int v = slot_u(__ldg(&sd[i]), tc, nchk);
            const float ov = app[v];
            app_put(app, v, ov < 0.0f, __fadd_rn(ov, S.dbuf[i * nchk + tc]), S);
          }
          if ((sync >> i) & 1u) __syncthreads();
        }
      }
      if constexpr (STG && !ST) fence_proxy_async_global();  // this thread's message stores before later TMA reads
      __syncthreads();
      if constexpr (STG && !ST) {
        stg.step++;
        if (*abort) return;
      }
    }
    ++it;
    // the syndrome after each iteration (early stop) or after the last one; the
    // barrier ending the last row group ordered every bitmap toggle before it
    if ((a.early_stop || it >= maxit) && syndrome_zero<DCMAX>(C, S.bitmap)) {
      converged = 1;
      break;
    }
    if (it >= maxit) break;
  }
}

template <int ALGO, int MSG16, int DCMAX, int MAXT, int MINB, bool STG>
__global__ void __launch_bounds__(MAXT, MINB) bp_layered_kernel(const DecodeArgs a) {
  typedef typename MsgIO<MSG16>::T MsgT;
  typedef MsgIO<MSG16> IO;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_frame;
  __shared__ int s_abort;
  __shared__ DevCode C;
  uint32_t* bitmap = (uint32_t*)smem_raw;
  float* smem_app = (float*)(smem_raw + ((a.bitmap_words * 4 + 15) & ~15));
  char* work = a.work + (long long)blockIdx.x * a.work_stride;
  MsgT* __restrict__ c2v = (MsgT*)work;
  float* gapp = (float*)(work + a.app_offset);
  const int tid = threadIdx.x, NT = blockDim.x;
  LayerSmem S{bitmap, a.lay_dbuf_floats ? (float*)(smem_raw + a.lay_dbuf_off) : nullptr};
  Stage stg{};
  if constexpr (STG) {
    stg.buf = (uint32_t)__cvta_generic_to_shared(smem_raw + a.lay_stage_off);
    stg.bytes = (uint32_t)a.lay_stage_bytes;
    stg.bar = stg.buf + 2 * stg.bytes;
    if (tid == 0) {
      mbar_init(stg.bar, 1);
      mbar_init(stg.bar + 8, 1);
      s_abort = 0;
    }
    __syncthreads();
  }

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
    const int n = C.n;
    const int* __restrict__ u2v = C.sp_u2v;
    const float* __restrict__ llr = a.llr + (a.llr_off ? a.llr_off[f] : f * (long long)n);
    const int maxit = a.max_iter_arr ? a.max_iter_arr[f] : a.max_iter;
    float* app = (n <= a.smem_app_floats) ? smem_app : gapp;
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

    // APP = llr (u order); hard decisions
    for (int base = 0; base < n; base += NT) {
      const int u = base + tid;
      float x = 0.0f;
      if (u < n) {
        x = u2v ? llr[__ldg(&u2v[u])] : __ldcs(llr + u);
        app[u] = x;
      }
      const unsigned b = __ballot_sync(0xffffffffu, u < n && x < 0.0f);
      if ((tid & 31) == 0 && u < n) bitmap[u >> 5] = b;
    }
    __syncthreads();
    int it = 0, converged = 0;
    if constexpr (DCMAX > 0) {
      layered_iterations<ALGO, MSG16, DCMAX, STG, (MAXT < 384)>(a, C, app, c2v, S, maxit, it, converged, stg,
                                                               &s_abort);
    } else {  // mixed batch: the exact slot count of this frame's code
#define GF2C_LAY_CASE(D) \
  layered_iterations<ALGO, MSG16, D, STG, (MAXT < 384)>(a, C, app, c2v, S, maxit, it, converged, stg, &s_abort)
      switch (C.lay_bucket) {
        case 7: GF2C_LAY_CASE(7); break;
        case 9: GF2C_LAY_CASE(9); break;
        case 10: GF2C_LAY_CASE(10); break;
        case 11: GF2C_LAY_CASE(11); break;
        case 13: GF2C_LAY_CASE(13); break;
        case 14: GF2C_LAY_CASE(14); break;
        case 18: GF2C_LAY_CASE(18); break;
        case 19: GF2C_LAY_CASE(19); break;
        default: GF2C_LAY_CASE(22); break;
      }
#undef GF2C_LAY_CASE
    }
    if constexpr (STG) {
      // a copy issued for an iteration that did not run (early stop): let it land
      if (stg.pending) {
        const uint32_t b = stg.step & 1u;
        if (!mbar_wait_bounded(stg.bar + 8 * b, (stg.phase >> b) & 1u)) {
          s_abort = 1;
          atomicExch(a.status, 2);
        }
        stg.phase ^= 1u << b;
        stg.pending = false;
      }
      __syncthreads();
      if (s_abort) return;
    }

    if (mo) {
      const int wn = (n + 31) >> 5;
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
      for (int u = tid; u < n; u += NT) bo[u2v ? __ldg(&u2v[u]) : u] = app[u];
    if (tid == 0) {
      if (a.iters) a.iters[f] = it + a.iters_add;
      if (a.conv) a.conv[f] = (uint8_t)converged;
      if (a.synd_ok) a.synd_ok[f] = (uint8_t)converged;
    }
    __syncthreads();
  }
}

// Row groups of up to 384 checks: one kernel per slot count of the DVB-T2
// codes (an exact fit wastes no slot and keeps the all-edges fast path).
// STG: the TMA-staged variant (not for the exact sum-product, which is
// arithmetic-bound).
template <int ALGO, int MSG16, int MINB, bool STG, int MAXT = 384>
static const void* lay_exact(int dcmax) {
  switch (dcmax) {
    case 7: return (const void*)bp_layered_kernel<ALGO, MSG16, 7, MAXT, MINB, STG>;
    case 9: return (const void*)bp_layered_kernel<ALGO, MSG16, 9, MAXT, MINB, STG>;
    case 10: return (const void*)bp_layered_kernel<ALGO, MSG16, 10, MAXT, MINB, STG>;
    case 11: return (const void*)bp_layered_kernel<ALGO, MSG16, 11, MAXT, MINB, STG>;
    case 13: return (const void*)bp_layered_kernel<ALGO, MSG16, 13, MAXT, MINB, STG>;
    case 14: return (const void*)bp_layered_kernel<ALGO, MSG16, 14, MAXT, MINB, STG>;
    case 18: return (const void*)bp_layered_kernel<ALGO, MSG16, 18, MAXT, MINB, STG>;
    case 19: return (const void*)bp_layered_kernel<ALGO, MSG16, 19, MAXT, MINB, STG>;
    case 22: return (const void*)bp_layered_kernel<ALGO, MSG16, 22, MAXT, MINB, STG>;
  }
  if constexpr (MAXT == 384) {
    switch (dcmax) {
      case 26: return (const void*)bp_layered_kernel<ALGO, MSG16, 26, 384, MINB, STG>;
      case 32: return (const void*)bp_layered_kernel<ALGO, MSG16, 32, 384, MINB, STG>;
      case 0:  // mixed batches: each frame runs the iterations of its code's exact slot count
        if constexpr (ALGO == L_SPA_FAST && !STG)
          return (const void*)bp_layered_kernel<ALGO, MSG16, 0, 384, MINB, false>;
        return nullptr;
    }
  }
  return nullptr;
}

// Row groups of up to 1024 checks (generic QC codes): coarser slot buckets.
template <int ALGO, int MSG16>
static const void* lay_wide(int dcmax) {
  if (dcmax <= 8) return (const void*)bp_layered_kernel<ALGO, MSG16, 8, 1024, 1, false>;
  if (dcmax <= 12) return (const void*)bp_layered_kernel<ALGO, MSG16, 12, 1024, 1, false>;
  if (dcmax <= 16) return (const void*)bp_layered_kernel<ALGO, MSG16, 16, 1024, 1, false>;
  if (dcmax <= 24) return (const void*)bp_layered_kernel<ALGO, MSG16, 24, 1024, 1, false>;
  if (dcmax <= 32) return (const void*)bp_layered_kernel<ALGO, MSG16, 32, 1024, 1, false>;
  return nullptr;
}

// Several checks per thread (192 or 128 threads, 4 or 6 CTAs per SM at the
// same 80 registers): staged FP16 kernels of the fused-row algorithms.
// 192 threads with five CTAs per SM: the same kernel compiled for 64 registers.
template <int ALGO, int MSG16>
static const void* lay_t(int dcmax, int maxt, bool stage, int bps) {
  if (maxt > 384) return stage ? nullptr : lay_wide<ALGO, MSG16>(dcmax);
  if (dcmax == 0 && maxt == 192 && !stage) {  // mixed batches, two checks per thread
    if constexpr (ALGO == L_SPA_FAST && MSG16) return (const void*)bp_layered_kernel<ALGO, MSG16, 0, 192, 4, false>;
    return nullptr;
  }
  if constexpr (ALGO == L_SPA) {
    return (stage || maxt < 384) ? nullptr : lay_exact<ALGO, MSG16, 1, false>(dcmax);
  } else {
    if (maxt == 192 && bps >= 5) return (stage && MSG16) ? lay_exact<ALGO, MSG16, 5, true, 192>(dcmax) : nullptr;
    if (maxt == 192) return (stage && MSG16) ? lay_exact<ALGO, MSG16, 4, true, 192>(dcmax) : nullptr;
    if (maxt == 128) return (stage && MSG16) ? lay_exact<ALGO, MSG16, 6, true, 128>(dcmax) : nullptr;
    if (maxt < 384) return nullptr;
    return stage ? lay_exact<ALGO, MSG16, 2, true>(dcmax) : lay_exact<ALGO, MSG16, 2, false>(dcmax);
  }
}

}  // namespace gf2c
