// gf2cuda encoder, syndrome and AWGN channel kernels (sm_100a).
//
// Encoder: the reference encodes with a dense k x m generator block
// (RuEncodingMatrices::encode, crates/gf2-coding/src/ldpc/encoding/richardson_urbanke.rs:263-289,
// 97.5% of its encode time in BitMatrix::matvec_transpose).  For DVB-T2 codes the
// parity part of H is the staircase, so the same unique codeword is
//   s = H_info u,  p[i] = s[0] ^ ... ^ s[i].
// With the checks of row group a = p mod q at positions t = p div q, s of a
// row group is a XOR of the 360-bit info blocks rotated by their addresses
// (32-bit windows), and p is a prefix over row groups plus a prefix along t;
// a warp-shuffle bit transpose puts the parity into natural order.  Other codes use the dense generator
// block of the right-to-left pivot search (the reference's columns).
//
// Syndrome: LdpcCode::syndrome (crates/gf2-coding/src/ldpc/core.rs:129-133).
// Channel: BpskModulator / AwgnChannel (crates/gf2-coding/src/channel.rs:51-218) with
// Philox4x32-10 and Box-Muller in place of rand_distr::Normal.
#include "internal.h"
#include "numeric.cuh"

namespace gf2c {

static constexpr int kEncThreads = 1024;     // channel kernel (Philox + LLRs for one frame)
static constexpr int kEncodeThreads = 256;   // encode kernel (several frames per SM)

// Bit i of a u32-word bit array.
__device__ __forceinline__ uint32_t getbit(const uint32_t* w, int i) { return (w[i >> 5] >> (i & 31)) & 1u; }

// Block-wide exclusive XOR scan of one bit per thread slot (count <= blockDim.x).
__device__ __forceinline__ uint32_t block_xor_scan_excl(uint32_t bit, uint32_t* warp_tot) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(0xffffffffu, bit);
  const uint32_t below = __popc(bal & ((1u << lane) - 1u)) & 1u;
  if (lane == 0) warp_tot[wid] = __popc(bal) & 1u;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    const uint32_t t = lane < nw ? warp_tot[lane] : 0u;
    const uint32_t b2 = __ballot_sync(0xffffffffu, t);
    const uint32_t ex = __popc(b2 & ((1u << lane) - 1u)) & 1u;
    __syncwarp();
    if (lane < nw) warp_tot[lane] = ex;
  }
  __syncthreads();
  const uint32_t r = below ^ warp_tot[wid];
  __syncthreads();
  return r;
}

// 32 x 32 bit transpose across a warp: lane c returns bit r = bit c of lane r's x.
template <int J, uint32_t M>
__device__ __forceinline__ uint32_t transpose_step(uint32_t x, int lane) {
  const uint32_t y = __shfl_xor_sync(0xffffffffu, x, J);
  return (lane & J) ? ((x & ~M) | ((y >> J) & M)) : ((x & M) | ((y & M) << J));
}
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
  x = transpose_step<16, 0x0000ffffu>(x, lane);
  x = transpose_step<8, 0x00ff00ffu>(x, lane);
  x = transpose_step<4, 0x0f0f0f0fu>(x, lane);
  x = transpose_step<2, 0x33333333u>(x, lane);
  return transpose_step<1, 0x55555555u>(x, lane);
}

// DVB-T2 structure (row group a holds the checks p = a + q t, t < 360): the
// info syndrome of row group a is
//   S_a[t] = XOR over its addresses x = a + q tau (info block b) of u[360 b + (t - tau) mod 360],
// a XOR of the info blocks rotated by tau, i.e. one 32-bit window per word and
// address taken from a cyclic copy of each block.

// Cyclic copies of the info blocks: 23 words per block, bit j = block bit j mod 360.
__device__ __forceinline__ void dvbt2_build_blocks(const uint32_t* u, int wk, int nblk, uint32_t* U2) {
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const int base = (360 * b) >> 5, sh = (360 * b) & 31;
    uint32_t x[12];
#pragma unroll
    for (int i = 0; i < 12; i++) {
      const uint32_t lo = u[base + i], hi = base + i + 1 < wk ? u[base + i + 1] : 0u;
      x[i] = __funnelshift_r(lo, hi, sh);
    }
    x[11] = (x[11] & 0xffu) | (x[0] << 8);  // block bits 352..359, then 0..23
    uint32_t* d = U2 + 23 * b;
#pragma unroll
    for (int i = 0; i < 12; i++) d[i] = x[i];
#pragma unroll
    for (int i = 12; i < 23; i++) d[i] = __funnelshift_r(x[i - 12], x[i - 11], 24);
  }
}

// S[12 a + w] = word w (t = 32 w + bit) of the info syndrome of row group a.
__device__ __forceinline__ void dvbt2_row_syndromes(const DevCode& C, const uint32_t* U2, int q, uint32_t* S) {
  for (int idx = threadIdx.x; idx < 12 * q; idx += blockDim.x) {
    const int a = idx / 12, w = idx - 12 * a;
    uint32_t acc = 0;
    const int e1 = __ldg(&C.enc_rg_ptr[a + 1]);
    for (int e = __ldg(&C.enc_rg_ptr[a]); e < e1; e++) {
      const int ent = __ldg(&C.enc_rg_ent[e]);
      int s = 32 * w - (ent & 0xffff);
      if (s < 0) s += 360;
      const uint32_t* d = U2 + 23 * (ent >> 16) + (s >> 5);
      acc ^= __funnelshift_r(d[0], d[1], s & 31);
    }
    S[idx] = w == 11 ? acc & 0xffu : acc;
  }
}

// OR bit t of row vector a (X[12 a + w] ^ xor_t[w]; xor_t nullable) into
// dst at bit offset + t q + a (natural order): 32 row groups x 32 positions
// per warp task, transposed in registers.  dst starts at zero there.
__device__ __forceinline__ void dvbt2_scatter_natural(const uint32_t* X, const uint32_t* xor_t, int q, uint32_t* dst,
                                                      int offset) {
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5, nA = (q + 31) >> 5;
  for (int task = threadIdx.x >> 5; task < 12 * nA; task += nwarps) {
    const int A = task / 12, T = task - 12 * A;
    const int a = 32 * A + lane;
    uint32_t x = a < q ? X[12 * a + T] ^ (xor_t ? xor_t[T] : 0u) : 0u;
    x = transpose32(x, lane);
    const int t = 32 * T + lane;
    if (t < 360) {
      const int nb = min(32, q - 32 * A);
      const uint32_t seg = nb < 32 ? x & ((1u << nb) - 1u) : x;
      const int p0 = offset + t * q + 32 * A, w0 = p0 >> 5, sh = p0 & 31;
      if (seg) {
        atomicOr(&dst[w0], seg << sh);
        if (sh && (seg >> (32 - sh))) atomicOr(&dst[w0 + 1], seg >> (32 - sh));
      }
    }
  }
}

// Encodes the message bits u (k bits, u32 words in shared memory) into the
// codeword cw (n bits, u32 words in shared memory); scratch as encode_smem sizes it.
__device__ void encode_frame(const DevCode& C, const uint32_t* u, uint32_t* cw, uint32_t* scratch) {
  const int n = C.n, k = C.k, m = C.m;
  const int wn = (n + 31) >> 5, wk = (k + 31) >> 5;
  if (C.enc_kind == 0) {
    // parity bit p = a + q t is the XOR of the info syndromes of all checks up
    // to p in natural order: (all row groups at t' < t) ^ (row groups a' <= a at t)
    const int q = C.enc_q, nblk = k / 360;
    uint32_t* U2 = scratch;        // cyclic info blocks
    uint32_t* S = U2 + 23 * nblk;  // row-group syndromes, then their prefix over a
    uint32_t* ctot = S + 12 * q;   // XOR over all row groups
    uint32_t* cpre = ctot + 12;    // exclusive prefix of ctot along t
    // codeword: the message, zero parity (the parity bits are OR-ed in below)
    for (int w = threadIdx.x; w < wn; w += blockDim.x) {
      const int lo = 32 * w;
      cw[w] = lo + 32 <= k ? u[w] : (lo < k ? u[w] & ((1u << (k - lo)) - 1u) : 0u);
    }
    dvbt2_build_blocks(u, wk, nblk, U2);
    __syncthreads();
    dvbt2_row_syndromes(C, U2, q, S);
    __syncthreads();
    {
      const int lane = threadIdx.x & 31;
      for (int w = threadIdx.x >> 5; w < 12; w += blockDim.x >> 5) {  // one warp per word: XOR scan over a
        uint32_t carry = 0;
        for (int a0 = 0; a0 < q; a0 += 32) {
          const int a = a0 + lane;
          uint32_t v = a < q ? S[12 * a + w] : 0u;
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v ^= y;
          }
          v ^= carry;
          if (a < q) S[12 * a + w] = v;
          carry = __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) ctot[w] = carry;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t carry = 0;
      for (int w = 0; w < 12; w++) {
        const uint32_t x = ctot[w];
        uint32_t inc = x;
        inc ^= inc << 1;
        inc ^= inc << 2;
        inc ^= inc << 4;
        inc ^= inc << 8;
        inc ^= inc << 16;
        inc ^= carry;
        cpre[w] = inc ^ x;
        carry = (inc >> 31) ? ~0u : 0u;
      }
    }
    __syncthreads();
    dvbt2_scatter_natural(S, cpre, q, cw, k);
    __syncthreads();
  } else {
    // parity word j (64 bits) = XOR over message bits i of P[i][j]
    const int Wm = C.words_m;
    uint64_t* par64 = (uint64_t*)scratch;  // Wm words (scratch sized for it)
    for (int j = threadIdx.x; j < Wm; j += blockDim.x) {
      uint64_t acc = 0;
      for (int i = 0; i < k; i++)
        if (getbit(u, i)) acc ^= __ldg(&C.enc_p[(size_t)i * Wm + j]);
      par64[j] = acc;
    }
    for (int w = threadIdx.x; w < wn; w += blockDim.x) cw[w] = 0u;
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += blockDim.x)
      if (getbit(u, i)) {
        const int c = __ldg(&C.enc_msg_cols[i]);
        atomicOr(&cw[c >> 5], 1u << (c & 31));
      }
    for (int j = threadIdx.x; j < m; j += blockDim.x)
      if ((par64[j >> 6] >> (j & 63)) & 1ull) {
        const int c = __ldg(&C.enc_par_cols[j]);
        atomicOr(&cw[c >> 5], 1u << (c & 31));
      }
    __syncthreads();
  }
  (void)wk;
}

// shared memory: u (wk32) + cw (wn32) + scratch (max(wm32 + 64, 2*Wm))
static size_t encode_smem(const DevCode& C) {
  const int wn = (C.n + 31) / 32, wk = (C.k + 31) / 32, wm = (C.m + 31) / 32;
  const int scratch = std::max(std::max(wm + 64, 2 * C.words_m), C.enc_kind == 0 ? 23 * (C.k / 360) + 12 * C.enc_q + 24 : 0);
  return (size_t)(((wk + 3) & ~3) + ((wn + 3) & ~3) + scratch + 4) * 4;
}

__global__ void __launch_bounds__(kEncodeThreads) encode_kernel(const DevCode* __restrict__ Cp,
                                                             const uint64_t* __restrict__ msg,
                                                             long long frames, uint64_t* __restrict__ cw) {
  extern __shared__ __align__(16) uint32_t sm[];
  const DevCode C = *Cp;
  const int wn = (C.n + 31) / 32, wk = (C.k + 31) / 32;
  uint32_t* u = sm;
  uint32_t* c = sm + ((wk + 3) & ~3);  // 16-byte aligned carve-up (scratch holds u64 words)
  uint32_t* scratch = c + ((wn + 3) & ~3);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const uint32_t* mi = (const uint32_t*)(msg + f * (long long)C.words_k);
    for (int w = threadIdx.x; w < wk; w += blockDim.x) {
      uint32_t x = mi[w];
      const int rem = C.k - 32 * w;
      if (rem < 32) x &= (1u << rem) - 1u;
      u[w] = x;
    }
    __syncthreads();
    encode_frame(C, u, c, scratch);
    uint32_t* co = (uint32_t*)(cw + f * (long long)C.words_n);
    for (int w = threadIdx.x; w < 2 * C.words_n; w += blockDim.x) co[w] = w < wn ? c[w] : 0u;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) syndrome_kernel(const DevCode* __restrict__ Cp,
                                                       const uint64_t* __restrict__ cw, long long frames,
                                                       uint64_t* __restrict__ synd, int32_t* __restrict__ weight) {
  extern __shared__ __align__(16) uint32_t sm[];
  __shared__ int s_w;
  const DevCode C = *Cp;
  const int wn = (C.n + 31) / 32;
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const uint32_t* ci = (const uint32_t*)(cw + f * (long long)C.words_n);
    for (int w = threadIdx.x; w < wn; w += blockDim.x) sm[w] = ci[w];
    if (threadIdx.x == 0) s_w = 0;
    __syncthreads();
    uint32_t* so = synd ? (uint32_t*)(synd + f * (long long)C.words_m) : nullptr;
    int cnt = 0;
    if (C.enc_kind == 0) {
      // s_p = (info syndrome of check p) ^ c[k + p] ^ c[k + p - 1], natural order
      const int k = C.k, m = C.m, q = C.enc_q, nblk = k / 360, wm = (m + 31) >> 5;
      uint32_t* U2 = sm + wn;
      uint32_t* S = U2 + 23 * nblk;
      uint32_t* nat = S + 12 * q;  // wm words
      for (int w = threadIdx.x; w < wm; w += blockDim.x) nat[w] = 0u;
      dvbt2_build_blocks(sm, (k + 31) >> 5, nblk, U2);
      __syncthreads();
      dvbt2_row_syndromes(C, U2, q, S);
      __syncthreads();
      dvbt2_scatter_natural(S, nullptr, q, nat, 0);
      __syncthreads();
      auto par_word = [&](int w) -> uint32_t {  // codeword bits k + 32 w .. + 31
        const int pos = k + 32 * w, i = pos >> 5;
        return __funnelshift_r(sm[i], i + 1 < wn ? sm[i + 1] : 0u, pos & 31);
      };
      for (int w = threadIdx.x; w < 2 * C.words_m; w += blockDim.x) {
        uint32_t x = 0;
        if (w < wm) {
          const uint32_t pw = par_word(w), prev = w > 0 ? par_word(w - 1) : 0u;
          x = nat[w] ^ pw ^ ((pw << 1) | (prev >> 31));
          if (w == wm - 1 && (m & 31)) x &= (1u << (m & 31)) - 1u;
        }
        cnt += __popc(x);
        if (so) so[w] = x;
      }
      atomicAdd(&s_w, cnt);
      __syncthreads();
      if (threadIdx.x == 0 && weight) weight[f] = s_w;
      __syncthreads();
      continue;
    }
    for (int base = 0; base < 32 * 2 * C.words_m; base += blockDim.x) {
      const int p = base + threadIdx.x;
      uint32_t s = 0;
      if (p < C.m) {
        const int e1 = __ldg(&C.csr_ptr[p + 1]);
        for (int e = __ldg(&C.csr_ptr[p]); e < e1; e++) s ^= getbit(sm, __ldg(&C.csr_idx[e]));
      }
      cnt += s;
      const uint32_t b = __ballot_sync(0xffffffffu, s);
      // a frame owns 2 * words_m 32-bit words; base is a multiple of 32, so lane
      // 0 bounds the whole warp's word
      if ((threadIdx.x & 31) == 0 && so && p < 64 * C.words_m) so[p >> 5] = b;
    }
    atomicAdd(&s_w, cnt);
    __syncthreads();
    if (threadIdx.x == 0 && weight) weight[f] = s_w;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kEncThreads) channel_kernel(const DevCode* __restrict__ Cp, uint2 key,
                                                              unsigned long long frame0, long long frames,
                                                              const double* __restrict__ sigma2,
                                                              uint64_t* __restrict__ info,
                                                              uint64_t* __restrict__ cwo, float* __restrict__ llr) {
  extern __shared__ __align__(16) uint32_t sm[];
  const DevCode C = *Cp;
  const int wn = (C.n + 31) / 32, wk = (C.k + 31) / 32;
  uint32_t* u = sm;
  uint32_t* c = sm + ((wk + 3) & ~3);  // 16-byte aligned carve-up (scratch holds u64 words)
  uint32_t* scratch = c + ((wn + 3) & ~3);
  for (long long f = blockIdx.x; f < frames; f += gridDim.x) {
    const uint32_t fr = (uint32_t)(frame0 + (unsigned long long)f);
    // info bits: 128 per Philox call, counter (block, frame, 1, 0)
    for (int blk = threadIdx.x; blk * 128 < C.k; blk += blockDim.x) {
      const uint4 r = philox4x32_10(make_uint4((uint32_t)blk, fr, 1u, 0u), key);
      const uint32_t wv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int w = blk * 4 + q;
        if (w < wk) {
          uint32_t x = wv[q];
          const int rem = C.k - 32 * w;
          if (rem < 32) x &= (1u << rem) - 1u;
          u[w] = x;
        }
      }
    }
    __syncthreads();
    encode_frame(C, u, c, scratch);
    if (info) {
      uint32_t* io = (uint32_t*)(info + f * (long long)C.words_k);
      for (int w = threadIdx.x; w < 2 * C.words_k; w += blockDim.x) io[w] = w < wk ? u[w] : 0u;
    }
    if (cwo) {
      uint32_t* co = (uint32_t*)(cwo + f * (long long)C.words_n);
      for (int w = threadIdx.x; w < 2 * C.words_n; w += blockDim.x) co[w] = w < wn ? c[w] : 0u;
    }
    if (llr) {
      const double s2 = sigma2[f];
      const double sigma = __dsqrt_rn(s2);
      float* lo = llr + f * (long long)C.n;
      for (int pair = threadIdx.x; 2 * pair < C.n; pair += blockDim.x) {
        const uint4 r = philox4x32_10(make_uint4((uint32_t)pair, fr, 2u, 0u), key);
        const unsigned long long a = (((unsigned long long)r.x << 32) | r.y) >> 11;
        const unsigned long long b = (((unsigned long long)r.z << 32) | r.w) >> 11;
        const double u1 = __dmul_rn((double)(a + 1ull), 1.1102230246251565404e-16);
        const double u2 = __dmul_rn((double)b, 1.1102230246251565404e-16);
        const double rad = __dsqrt_rn(__dmul_rn(-2.0, log_d(u1)));
        double sn, cs;
        sincos_2pi_d(u2, &sn, &cs);
        const double z[2] = {__dmul_rn(rad, cs), __dmul_rn(rad, sn)};
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = 2 * pair + h;
          if (i < C.n) {
            const double sym = getbit(c, i) ? -1.0 : 1.0;
            const double y = __dadd_rn(sym, __dmul_rn(sigma, z[h]));
            lo[i] = __double2float_rn(__ddiv_rn(__dmul_rn(2.0, y), s2));
          }
        }
      }
    }
    __syncthreads();
  }
}

// Bit and frame errors between two packed bit batches (the FER / BER counters
// of a Monte Carlo point; the reference's counterpart is the uncoded runner
// SimulationRunner, crates/gf2-coding/src/simulation.rs:140-193).
// totals[0] += frames with at least one error, totals[1] += bit errors.
__global__ void __launch_bounds__(256) count_errors_kernel(const uint64_t* __restrict__ a,
                                                           const uint64_t* __restrict__ b, long long frames,
                                                           int words, int32_t* __restrict__ per_frame,
                                                           unsigned long long* __restrict__ totals) {
  __shared__ unsigned long long s_bits, s_frames;
  if (threadIdx.x == 0) {
    s_bits = 0;
    s_frames = 0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (long long f = (long long)blockIdx.x * nwarp + warp; f < frames; f += (long long)gridDim.x * nwarp) {
    int e = 0;
    for (int w = lane; w < words; w += 32) e += __popcll(a[f * words + w] ^ b[f * words + w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (lane == 0) {
      if (per_frame) per_frame[f] = e;
      if (e) {
        atomicAdd(&s_bits, (unsigned long long)e);
        atomicAdd(&s_frames, 1ull);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_frames) atomicAdd(&totals[0], s_frames);
    if (s_bits) atomicAdd(&totals[1], s_bits);
  }
}

int launch_count_errors(const uint64_t* a, const uint64_t* b, long long frames, int words, int32_t* per_frame,
                        unsigned long long* totals, cudaStream_t st) {
  if (frames <= 0) return GF2C_OK;
  int grid = (int)std::min<long long>((frames + 7) / 8, 148 * 8);
  count_errors_kernel<<<grid, 256, 0, st>>>(a, b, frames, words, per_frame, totals);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

static int grid_for(long long frames) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long g = std::min<long long>(frames, (long long)sms * 2);
  return (int)std::max<long long>(g, 1);
}

int launch_encode(const DevCode* dcode, const DevCode& h, const uint64_t* msg, long long frames,
                  uint64_t* cw, cudaStream_t st) {
  if (frames <= 0) return GF2C_OK;
  size_t smem = encode_smem(h);
  GF2C_CUDA(cudaFuncSetAttribute(encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 148, per_sm = 1;
  GF2C_CUDA(cudaGetDevice(&dev));
  GF2C_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, encode_kernel, kEncodeThreads, smem));
  const long long grid = std::max<long long>(1, std::min<long long>(frames, (long long)sms * std::max(per_sm, 1)));
  encode_kernel<<<(int)grid, kEncodeThreads, smem, st>>>(dcode, msg, frames, cw);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_syndrome(const DevCode* dcode, const DevCode& h, const uint64_t* cw, long long frames,
                    uint64_t* synd, int32_t* weight, cudaStream_t st) {
  if (frames <= 0) return GF2C_OK;
  size_t smem = (size_t)((h.n + 31) / 32) * 4;
  if (h.enc_kind == 0) smem += (size_t)(23 * (h.k / 360) + 12 * h.enc_q + (h.m + 31) / 32) * 4;
  GF2C_CUDA(cudaFuncSetAttribute(syndrome_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  syndrome_kernel<<<grid_for(frames), 256, smem, st>>>(dcode, cw, frames, synd, weight);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

int launch_channel(const DevCode* dcode, const DevCode& h, uint64_t seed, uint64_t frame0,
                   long long frames, const double* sigma2, uint64_t* info, uint64_t* cw, float* llr,
                   cudaStream_t st) {
  if (frames <= 0) return GF2C_OK;
  size_t smem = encode_smem(h);
  GF2C_CUDA(cudaFuncSetAttribute(channel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  channel_kernel<<<grid_for(frames), kEncThreads, smem, st>>>(dcode, key, frame0, frames, sigma2, info, cw, llr);
  GF2C_CUDA(cudaGetLastError());
  return GF2C_OK;
}

}  // namespace gf2c
