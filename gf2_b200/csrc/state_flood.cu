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
// shared memory when they fit together (DVB-T2 short frames, ALL_SMEM);
// otherwise both live in the CTA's global workspace slice, which the L1 and the
// 126 MB L2 cache for the frames in flight.  The u-order copy of the channel
// LLRs (read once per iteration) is in the workspace.
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

// Posteriors in u order (shared memory or the CTA workspace).
template <bool ALL_SMEM>
struct Post {
  float* p;
  __device__ __forceinline__ float* at(int u) const { return p + u; }
  __device__ __forceinline__ float* run(int) const { return p; }
};

struct SlotTables {
  const int2* desc;      // DevCode::sp_desc
  const uint32_t* absent;
  const int* slot_var;
};

// Posteriors of the slots of check t of row group g (slot i in ap[i]); returns
// the mask of the slots that hold an edge.  Every address is valid, so the
// loads are issued unconditionally, back to back.
template <int DCMAX, bool ALL_SMEM>
__device__ __forceinline__ uint32_t load_slots(const SlotTables T, int g, const int4 G, int t, uint32_t dmask,
                                               const Post<ALL_SMEM> P, float (&ap)[DCMAX]) {
  if (T.desc) {
    const int2* __restrict__ sd = T.desc + G.w;
#pragma unroll
    for (int i = 0; i < DCMAX; i++) {
      if (i < G.z) {
        const int2 D = __ldg(&sd[i]);
        ap[i] = P.run(D.x)[D.x + t - (t >= D.y ? G.y : 0)];
      }
    }
    return t == 0 ? dmask & ~__ldg(&T.absent[g]) : dmask;
  }
  const int* __restrict__ sv = T.slot_var + G.w + t;
  uint32_t real = 0;
#pragma unroll
  for (int i = 0; i < DCMAX; i++) {
    if (i < G.z) {
      const int u = __ldg(&sv[i * G.y]);
      real |= (uint32_t)(u >= 0) << i;
      ap[i] = *P.at(u < 0 ? 0 : u);
    }
  }
  return real;
}

// Check-node update from the slot posteriors ap[] and the old state `so`:
// writes the new state and returns the parity of the hard decisions of the
// posteriors.  ALLREAL: every slot below d holds an edge; FIRST: the old
// messages are all zero.
template <int DCMAX, bool FIRST, bool ALLREAL>
__device__ __forceinline__ int check_node(const float (&ap)[DCMAX], uint32_t real, int d, const uint4 so,
                                          uint4* st_cc, bool nms, float al, float be, bool msg16) {
  float m1 = __int_as_float(0x7f800000), m2 = m1;
  uint32_t i1 = 0xffu, neg = 0u;
  int hp = 0;
#pragma unroll
  for (int i = 0; i < DCMAX; i++) {
    if (i < d && (ALLREAL || ((real >> i) & 1u))) {
      hp ^= (int)(ap[i] < 0.0f);
      const float x = FIRST ? ap[i] : __fsub_rn(ap[i], state_c2v(so, i));
      const float ax = fabsf(x);
      const bool lt1 = ax < m1, lt2 = ax < m2;
      m2 = lt1 ? m1 : (lt2 ? ax : m2);
      m1 = lt1 ? ax : m1;
      i1 = lt1 ? (uint32_t)i : i1;
      neg |= (uint32_t)(x < 0.0f) << i;
    }
  }
  const bool single = ALLREAL ? d == 1 : __popc(real) == 1;
  float mag1 = single ? 0.0f : m1, mag2 = single ? 0.0f : m2;
  if (nms) {  // normalised / offset min-sum
    const float d1 = __fsub_rn(mag1, be), d2 = __fsub_rn(mag2, be);
    mag1 = __fmul_rn(al, d1 > 0.0f ? d1 : 0.0f);
    mag2 = __fmul_rn(al, d2 > 0.0f ? d2 : 0.0f);
  }
  if (msg16) {
    mag1 = round_mag16(mag1);
    mag2 = round_mag16(mag2);
  }
  const uint32_t sgn = (__popc(neg) & 1) ? ~neg : neg;
  *st_cc = make_uint4(__float_as_uint(mag1), __float_as_uint(mag2), sgn, i1);
  return hp;
}

// The code descriptor of the frame a CTA is decoding (shared by the passes).
__shared__ DevCode sf_code;

// Check-node pass: every check reads its slot posteriors and its old state and
// writes its new state.  Returns this thread's part of the parity of the hard
// decisions over all checks (the syndrome of the previous iteration).  NMS
// weights of this iteration start at alpha / beta + nms_row, one per row group
// when per_layer, else one for the whole code.
template <int DCMAX, bool ALL_SMEM>
__device__ __forceinline__ int sf_check_pass(uint4* st, const Post<ALL_SMEM> P, bool first, bool nms, bool msg16,
                                             const float* alpha, const float* beta, int nms_row, bool per_layer) {
  const DevCode& C = sf_code;
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const SlotTables T{C.sp_desc, C.sp_absent, C.slot_var};
  const int2* __restrict__ cch = C.sp_cchunk;
  const int4* __restrict__ spcg = C.sp_cg;
  const int ncc = C.sp_ncchunk;
  int par = 0;
  for (int ch = threadIdx.x >> 5; ch < ncc; ch += nwarps) {
    const int2 CH = cch[ch];
    const int4 G = spcg[CH.x];
    const int t = CH.y + lane;
    if (t >= G.y) continue;
    const int cc = G.x + t;
    const uint32_t dmask = G.z >= 32 ? 0xffffffffu : (1u << G.z) - 1u;
    float ap[DCMAX];
    const uint32_t real = load_slots<DCMAX, ALL_SMEM>(T, CH.x, G, t, dmask, P, ap);
    float al = 1.0f, be = 0.0f;
    if (nms) {
      const int idx = nms_row + (per_layer ? CH.x : 0);
      al = __ldg(&alpha[idx]);
      be = __ldg(&beta[idx]);
    }
    if (real == dmask) {
      if (first)
        par |= check_node<DCMAX, true, true>(ap, real, G.z, make_uint4(0u, 0u, 0u, 0xffu), st + cc, nms, al, be,
                                             msg16);
      else
        par |= check_node<DCMAX, false, true>(ap, real, G.z, st[cc], st + cc, nms, al, be, msg16);
    } else {
      const uint4 so = first ? make_uint4(0u, 0u, 0u, 0xffu) : st[cc];
      par |= check_node<DCMAX, false, false>(ap, real, G.z, so, st + cc, nms, al, be, msg16);
    }
  }
  return par;
}

// Variable-node pass: belief = llr + sum of c2v in ascending original check index.
template <bool ALL_SMEM>
__device__ __forceinline__ void sf_var_pass(const uint4* st, const Post<ALL_SMEM> P, const float* lu) {
  const DevCode& C = sf_code;
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int nvc = C.sp_nvchunk, vgs = C.vgs, n = C.n;
  const int2* __restrict__ vch = C.sp_vchunk;
  const int2* __restrict__ svg = C.sp_vg;
  const int* __restrict__ sci = C.sp_ci;
  for (int ch = threadIdx.x >> 5; ch < nvc; ch += nwarps) {
    const int2 CH = vch[ch];
    const int2 V = svg[CH.x];
    const int j = CH.y + lane;
    const int u = CH.x * vgs + j;
    if (j >= vgs || u >= n) continue;
    float b = lu[u];
    const int* __restrict__ ci = sci + V.y + j;
    // batches of 4 edges, the last one partial: the edge-table loads of a
    // batch, then its state gathers, are in flight together (two dependent
    // round trips per batch, whatever the degree)
    for (int i = 0; i < V.x; i += 4) {
      int e[4];
      uint4 s[4];
#pragma unroll
      for (int q = 0; q < 4; q++) e[q] = i + q < V.x ? __ldg(&ci[(i + q) * vgs]) : -1;
#pragma unroll
      for (int q = 0; q < 4; q++) s[q] = st[e[q] < 0 ? 0 : (e[q] & 0xffffff)];
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (e[q] >= 0) b = __fadd_rn(b, state_c2v(s[q], e[q] >> 24));
    }
    *P.at(u) = b;
  }
}

// Parity of the hard decisions over all checks (this thread's part).
template <int DCMAX, bool ALL_SMEM>
__device__ __forceinline__ int sf_syndrome_pass(const Post<ALL_SMEM> P) {
  const DevCode& C = sf_code;
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const SlotTables T{C.sp_desc, C.sp_absent, C.slot_var};
  int p = 0;
  for (int ch = threadIdx.x >> 5; ch < C.sp_ncchunk; ch += nwarps) {
    const int2 CH = C.sp_cchunk[ch];
    const int4 G = C.sp_cg[CH.x];
    const int t = CH.y + lane;
    if (t >= G.y) continue;
    float ap[DCMAX];
    const uint32_t real =
        load_slots<DCMAX, ALL_SMEM>(T, CH.x, G, t, G.z >= 32 ? 0xffffffffu : (1u << G.z) - 1u, P, ap);
#pragma unroll
    for (int i = 0; i < DCMAX; i++)
      if (i < G.z && ((real >> i) & 1u)) p ^= (int)(ap[i] < 0.0f);
  }
  return p;
}

template <int DCMAX, bool ALL_SMEM>
__global__ void __launch_bounds__(kStateThreads, 1) bp_state_flood_kernel(const DecodeArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_frame;
  const DevCode& C = sf_code;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31;
  char* work = a.work + (long long)blockIdx.x * a.work_stride;
  uint4* st = ALL_SMEM ? (uint4*)smem_raw : (uint4*)(work + a.sf_st_off);
  const Post<ALL_SMEM> P{ALL_SMEM ? (float*)(smem_raw + a.sf_app_soff) : (float*)(work + a.sf_app_off)};
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
    if (tid == 0) sf_code = a.codes[cid];
    __syncthreads();
    const int n = C.n;
    const float* __restrict__ llr = a.llr + (a.llr_off ? a.llr_off[f] : f * (long long)n);
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
    const int* __restrict__ u2v = C.sp_u2v;
    float* llr_u = (float*)(work + a.sf_llr_off);
    for (int u = tid; u < n; u += NT) {
      const float x = u2v ? llr[__ldg(&u2v[u])] : llr[u];
      if (u2v) llr_u[u] = x;
      *P.at(u) = x;
    }
    const float* lu = u2v ? llr_u : llr;
    __syncthreads();

    const bool nms = a.nms_iters > 0;
    int it = 0, converged = 0, synd = 1;
    for (;;) {
      const int nms_row = nms ? min(it, a.nms_iters - 1) * a.nms_L : 0;
      int par = sf_check_pass<DCMAX, ALL_SMEM>(st, P, it == 0, nms, a.sf_msg16 != 0, a.alpha, a.beta, nms_row,
                                               a.nms_L == C.ncg);
      par = __syncthreads_or(par);
      if (it > 0 && a.early_stop && !par) {
        converged = 1;
        synd = 0;
        break;
      }
      sf_var_pass<ALL_SMEM>(st, P, lu);
      __syncthreads();
      ++it;
      if (it >= maxit) break;
    }
    if (!converged) {
      synd = __syncthreads_or(sf_syndrome_pass<DCMAX, ALL_SMEM>(P));
      converged = !synd;
    }
    if (mo) {  // message bits: the first k variables (identical in u order)
      uint32_t* mo32 = (uint32_t*)mo;
      const int k = C.k, wk = C.words_k;
      for (int base = 0; base < 64 * wk; base += NT) {
        const int u = base + tid;
        const unsigned bits = __ballot_sync(0xffffffffu, u < k && *P.at(u < n ? u : 0) < 0.0f);
        if (lane == 0 && u < 64 * wk) mo32[u >> 5] = bits;
      }
    }
    if (bo)
      for (int u = tid; u < n; u += NT) bo[u2v ? __ldg(&u2v[u]) : u] = *P.at(u);
    if (tid == 0) {
      if (a.iters) a.iters[f] = it;
      if (a.conv) a.conv[f] = (uint8_t)converged;
      if (a.synd_ok) a.synd_ok[f] = (uint8_t)(!synd);
    }
    __syncthreads();
  }
}

int state_flood_threads() { return kStateThreads; }

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
