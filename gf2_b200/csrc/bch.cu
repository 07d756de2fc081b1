// gf2cuda DVB-T2 outer BCH code (sm_100a): batch encoder and decoder.
//
// The reference's binary BCH outer code of DVB-T2 (crates/gf2-coding/src/bch):
//   parameters DvbBchParams::for_code          bch/dvb_t2/params.rs:56-85
//   generator g = g_1 ... g_t                  bch/dvb_t2/generators.rs:14-62
//   BchEncoder::encode: [message | parity], bit i at polynomial degree n-1-i,
//     parity = x^r m(x) mod g(x)               bch/core.rs:421-480
//   BchDecoder::decode: syndromes S_j = r(alpha^j), j = 1..2t; all zero ->
//     the received message; else Berlekamp-Massey, Chien search over
//     alpha^-i, flip bit n-1-i for every root i, first k bits
//                                            bch/core.rs:562-818
// alpha = x in GF(2^m) modulo the DVB-T2 primitive polynomial.
//
// GPU layout: one warp per frame.
//  * Odd syndromes S_j, j = 2s+1 < 2t (shared by encoder and decoder):
//    S_j = alpha^(j(n-1)) sum_i b_i beta^i, beta = alpha^-j.  Lane l takes the
//    64-bit words w = l + 32u (coalesced) and runs Horner over u from the top,
//    acc <- acc * beta^2048 + q_w, where q_w = sum over the word's 8 bytes of a
//    per-(byte position, value) table entry that packs four syndromes in 8
//    bytes; the multiply by the constant beta^2048 is two byte lookups.  The
//    lane's sum is scaled by alpha^(j(n-1-64l)) and XOR-reduced over the warp.
//    All tables live in shared memory.  Even syndromes are squares:
//    S_(2^a o) = S_o^(2^a) for a binary received word.
//  * Encoder: the odd syndromes of [message | 0] fix the parity, because the
//    map from the r parity bits to the r = t m odd-syndrome bits is invertible
//    (g is the product of the minimal polynomials of alpha^j, j odd < 2t).
//    parity = A s with A the inverse of that GF(2) matrix (host-built); it
//    equals x^r m(x) mod g, the unique systematic parity.
//  * Decoder, kernel 1: syndromes, the message copy, and the reference's
//    Berlekamp-Massey step for step with lane i holding coefficient i of the
//    locator and of the correction polynomial (the discrepancy is a warp XOR
//    reduction).  It stores the locator as logarithms per frame.
//  * Decoder, kernel 2 (Chien search): the antilog table of the field in
//    shared memory, stored with an offset so that the exponents are reduced
//    mod N once per 8 position steps and the steps in between are constant
//    load offsets; lane l evaluates positions i = l + 32s with the terms'
//    exponents in registers (locator degrees 1..12 unrolled); a root i flips
//    bit n-1-i when it lies in the message.  A frame stops once it has found
//    deg(lambda) roots (a polynomial has no more), which returns the same
//    roots as the full search.  Kernel 1 files each frame under its locator
//    degree; kernel 2 takes the frames degree by degree, highest first.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "internal.h"

namespace gf2c {

static constexpr int kBchWarps = 8;          // warps per CTA in the syndrome kernels
static constexpr int kChienThreads = 1024;   // Chien kernel CTA size
static constexpr int kChienFastMax = 12;     // locator degrees with an unrolled evaluator
static constexpr int kChienSeg = 8;          // positions steps between exponent reductions
static constexpr int kChienOff = 32 * kChienFastMax * kChienSeg;  // antilog table offset
static constexpr uint16_t kLogZero = 0xFFFF; // stored log of a zero coefficient

struct BchDev {
  int n, k, t, r, m, N, words_n, words_k, rw;  // rw = 32-bit words of the parity
  const uint16_t* exp;   // [2N]
  const uint16_t* log;   // [N + 1]
  const uint2* quad;     // [3][8][256]: 4 odd syndromes per entry, byte position p
  const uint16_t* mul;   // [t][512]: (v * gamma_s), (v << 8) * gamma_s
  const uint32_t* lf;    // [t][32]: exponent of alpha^(j(n-1-64 lane)) mod N
  const uint32_t* acol;  // [r][rw]: parity pattern of syndrome bit b
};

// shared-memory image of the syndrome tables
struct SynTab {
  const uint2* quad;
  const uint16_t* mul;
  const uint32_t* lf;
};

__device__ __forceinline__ uint32_t gf_mul(const BchDev& B, uint32_t a, uint32_t b) {
  if (!a || !b) return 0;
  return __ldg(&B.exp[__ldg(&B.log[a]) + __ldg(&B.log[b])]);
}

__device__ __forceinline__ uint32_t warp_xor(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Stage the syndrome tables into shared memory; returns the end of the area.
template <int T>
__device__ __forceinline__ SynTab load_syn_tables(const BchDev& B, unsigned char* smem) {
  uint2* q = (uint2*)smem;
  uint16_t* mu = (uint16_t*)(q + 3 * 8 * 256);
  uint32_t* lf = (uint32_t*)(mu + T * 512);
  for (int i = threadIdx.x; i < 3 * 8 * 256; i += blockDim.x) q[i] = B.quad[i];
  for (int i = threadIdx.x; i < T * 512; i += blockDim.x) mu[i] = B.mul[i];
  for (int i = threadIdx.x; i < T * 32; i += blockDim.x) lf[i] = B.lf[i];
  return SynTab{q, mu, lf};
}

template <int T>
__host__ __device__ constexpr size_t syn_smem_bytes() {
  return (size_t)3 * 8 * 256 * 8 + (size_t)T * 512 * 2 + (size_t)T * 32 * 4;
}

// Odd syndromes S_(2s+1), s < T, of the first `nbits` bits of the packed frame
// `c` (the remaining codeword bits zero); every lane returns all T values.
// Words below `copy_words` are also written to `copy` (the last one masked to
// `copy_bits`).
template <int T>
__device__ __forceinline__ void odd_syndromes(const BchDev& B, const SynTab& S, const uint64_t* __restrict__ c,
                                              int nbits, uint64_t* __restrict__ copy, int copy_bits, int lane,
                                              uint32_t so[T]) {
  const int nwords = (nbits + 63) >> 6;
  const int cwords = (copy_bits + 63) >> 6;
  uint32_t acc[T];
#pragma unroll
  for (int s = 0; s < T; s++) acc[s] = 0;
  const int U = (nwords + 31) >> 5;
  for (int u = U - 1; u >= 0; u--) {
    const int w = lane + 32 * u;
    uint64_t word = 0;
    if (w < nwords) {
      word = __ldg(&c[w]);
      if (copy && w < cwords) copy[w] = (w == cwords - 1 && (copy_bits & 63)) ? word & ((1ull << (copy_bits & 63)) - 1ull) : word;
      if (w == nwords - 1 && (nbits & 63)) word &= (1ull << (nbits & 63)) - 1ull;
    }
#pragma unroll
    for (int s = 0; s < T; s++) {
      const uint32_t a = acc[s];
      acc[s] = (uint32_t)S.mul[s * 512 + (a & 0xffu)] ^ (uint32_t)S.mul[s * 512 + 256 + (a >> 8)];
    }
    if (word) {
      const uint32_t lo = (uint32_t)word, hi = (uint32_t)(word >> 32);
#pragma unroll
      for (int q = 0; q < (T + 3) / 4; q++) {
        uint32_t x0 = 0, x1 = 0;
#pragma unroll
        for (int p = 0; p < 8; p++) {
          const uint32_t v = ((p < 4 ? lo : hi) >> (8 * (p & 3))) & 0xffu;
          const uint2 e = S.quad[(q * 8 + p) * 256 + v];
          x0 ^= e.x;
          x1 ^= e.y;
        }
        if (4 * q + 0 < T) acc[4 * q + 0] ^= x0 & 0xffffu;
        if (4 * q + 1 < T) acc[4 * q + 1] ^= x0 >> 16;
        if (4 * q + 2 < T) acc[4 * q + 2] ^= x1 & 0xffffu;
        if (4 * q + 3 < T) acc[4 * q + 3] ^= x1 >> 16;
      }
    }
  }
  // scale by alpha^(j(n-1-64 lane)), then reduce two syndromes per shuffle
#pragma unroll
  for (int s = 0; s < T; s++)
    acc[s] = acc[s] ? __ldg(&B.exp[__ldg(&B.log[acc[s]]) + S.lf[s * 32 + lane]]) : 0u;
#pragma unroll
  for (int s = 0; s < T; s += 2) {
    uint32_t v = acc[s] | (s + 1 < T ? acc[s + 1] << 16 : 0u);
    v = warp_xor(v);
    so[s] = v & 0xffffu;
    if (s + 1 < T) so[s + 1] = v >> 16;
  }
}

template <int T>
__global__ void __launch_bounds__(kBchWarps * 32) bch_encode_kernel(const BchDev B, const uint64_t* __restrict__ msg,
                                                                    long long frames, uint64_t* __restrict__ cw) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SynTab S = load_syn_tables<T>(B, smem);
  uint32_t* par_s = (uint32_t*)(smem + syn_smem_bytes<T>());  // [warps][8]
  uint16_t* syn_s = (uint16_t*)(par_s + kBchWarps * 8);         // [warps][16]
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* par = par_s + wib * 8;
  uint16_t* sy = syn_s + wib * 16;
  const long long warps = (long long)gridDim.x * kBchWarps;
  for (long long f = (long long)blockIdx.x * kBchWarps + wib; f < frames; f += warps) {
    const uint64_t* m = msg + f * B.words_k;
    uint64_t* c = cw + f * B.words_n;
    uint32_t so[T];
    odd_syndromes<T>(B, S, m, B.k, c, B.k, lane, so);
#pragma unroll
    for (int s = 0; s < T; s++)
      if (lane == s) sy[s] = (uint16_t)so[s];
    __syncwarp();
    // parity = A s: lane takes syndrome bits b = lane + 32 z
    uint32_t p[6] = {0, 0, 0, 0, 0, 0};
    for (int b = lane; b < B.r; b += 32) {
      if ((sy[b / B.m] >> (b % B.m)) & 1u) {
        const uint32_t* col = B.acol + (size_t)b * B.rw;
#pragma unroll
        for (int q = 0; q < 6; q++)
          if (q < B.rw) p[q] ^= __ldg(&col[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) p[q] = warp_xor(p[q]);
    uint32_t mine = 0;
#pragma unroll
    for (int q = 0; q < 6; q++)
      if (lane == q) mine = p[q];
    if (lane < 8) par[lane] = mine;
    __syncwarp();
    // codeword words from bit k on: parity bit q sits at codeword bit k + q
    for (int w = (B.k >> 6) + lane; w < B.words_n; w += 32) {
      const int o = 64 * w - B.k;  // parity bit at the word's bit 0 (negative in the message's tail word)
      uint64_t word;
      if (o >= 0) {
        const int q0 = o >> 5, sh = o & 31;
        const uint64_t lo = ((uint64_t)par[q0 + 1] << 32) | par[q0];
        const uint64_t hi = q0 + 2 < 8 ? par[q0 + 2] : 0u;
        word = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
      } else {
        const uint64_t low = ((uint64_t)par[1] << 32) | par[0];
        word = (m[w] & ((1ull << (B.k & 63)) - 1ull)) | (low << (-o));
      }
      if (w == B.words_n - 1 && (B.n & 63)) word &= (1ull << (B.n & 63)) - 1ull;
      c[w] = word;
    }
    __syncwarp();
  }
}

// Kernel 1 of the decoder: syndromes, message copy, Berlekamp-Massey.
template <int T>
__global__ void __launch_bounds__(kBchWarps * 32) bch_syndrome_bm_kernel(
    const BchDev B, const uint64_t* __restrict__ cw, long long frames, uint64_t* __restrict__ msg,
    int32_t* __restrict__ nflips, uint16_t* __restrict__ synd_out, uint16_t* __restrict__ loc,
    int32_t* __restrict__ degs, uint32_t* __restrict__ bcnt, int32_t* __restrict__ blist) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SynTab S = load_syn_tables<T>(B, smem);
  uint16_t* syn_s = (uint16_t*)(smem + syn_smem_bytes<T>());  // [warps][32]
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint16_t* sS = syn_s + wib * 32;
  const long long warps = (long long)gridDim.x * kBchWarps;
  for (long long f = (long long)blockIdx.x * kBchWarps + wib; f < frames; f += warps) {
    uint32_t so[T];
    odd_syndromes<T>(B, S, cw + f * B.words_n, B.n, msg + f * B.words_k, B.k, lane, so);
    uint32_t any = 0;
#pragma unroll
    for (int s = 0; s < T; s++) {
      any |= so[s];
      if (lane == s) sS[2 * s] = (uint16_t)so[s];
    }
    __syncwarp();
    // even syndromes: S_(2^a o) = S_o^(2^a)
    uint32_t ev = 0;
    const int j = lane + 1;
    const bool even = lane < 2 * T && !(j & 1);
    if (even) {
      const int a = __ffs(j) - 1;
      const uint32_t so_ = sS[(j >> a) - 1];
      ev = so_ ? __ldg(&B.exp[((uint32_t)__ldg(&B.log[so_]) << a) % (uint32_t)B.N]) : 0u;
    }
    __syncwarp();
    if (even) sS[lane] = (uint16_t)ev;
    __syncwarp();
    if (synd_out && lane < 2 * T) synd_out[f * 2 * T + lane] = sS[lane];
    if (!any) {
      if (lane == 0) {
        degs[f] = 0;
        if (nflips) nflips[f] = 0;
      }
      __syncwarp();
      continue;
    }
    // Berlekamp-Massey: lane i holds lambda_i and b_i
    uint32_t lam = lane == 0, bb = lane == 0;
    int l = 0, mm = 1;
    for (int nn = 0; nn < 2 * T; nn++) {
      uint32_t prod = 0;
      if (lane == 0) prod = sS[nn];
      else if (lane <= l && lane <= nn) prod = gf_mul(B, lam, sS[nn - lane]);
      const uint32_t delta = warp_xor(prod);
      if (delta == 0) {
        mm += 1;
        continue;
      }
      const uint32_t tl = lam;
      const uint32_t bsh = __shfl_up_sync(0xffffffffu, bb, mm);
      if (lane >= mm) lam ^= gf_mul(B, delta, bsh);
      if (2 * l <= nn) {
        l = nn + 1 - l;
        const uint32_t di = __ldg(&B.exp[(B.N - __ldg(&B.log[delta])) % B.N]);
        bb = gf_mul(B, tl, di);
        mm = 1;
      } else {
        mm += 1;
      }
    }
    const int deg = 31 - __clz(__ballot_sync(0xffffffffu, lam != 0));
    const bool zero_coef = __any_sync(0xffffffffu, lane >= 1 && lane <= deg && lam == 0);
    loc[f * 32 + lane] = lam ? __ldg(&B.log[lam]) : kLogZero;
    if (lane == 0) {
      degs[f] = deg;
      if (deg == 0) {
        if (nflips) nflips[f] = 0;
      } else {  // Chien work list of the frame's bucket: its degree, or 0 for the generic evaluator
        const int bk = (deg <= kChienFastMax && !zero_coef) ? deg : 0;
        const uint32_t pos = atomicAdd(&bcnt[bk], 1u);
        blist[(size_t)bk * frames + pos] = (int32_t)f;
      }
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void flip_root(const BchDev& B, int i, uint64_t* mo) {
  if (i >= B.r) {
    const int bit = B.n - 1 - i;
    atomicXor((unsigned long long*)&mo[bit >> 6], 1ull << (bit & 63));
  }
}

// Chien search of a locator of degree D with no zero coefficient below D.
// sexp[x] = alpha^(x - kChienOff); term j keeps Ep = (its exponent mod N) +
// kChienOff, which stays in [0, N + kChienOff) over a segment of kChienSeg
// steps of -32 j each, so the steps inside a segment are constant offsets of
// the load and the reduction mod N happens once per segment.
template <int D>
__device__ __forceinline__ int chien_fast(const BchDev& B, const uint16_t* __restrict__ sexp, uint32_t myL, int lane,
                                          uint64_t* mo) {
  const uint32_t N = (uint32_t)B.N;
  uint32_t Ep[D];
#pragma unroll
  for (int j = 1; j <= D; j++) {
    const uint32_t Lj = __shfl_sync(0xffffffffu, myL, j);
    Ep[j - 1] = (Lj + N - (uint32_t)(j * lane)) % N + kChienOff;
  }
  int roots = 0;
  const int steps = (B.n + 31) >> 5;
  for (int s0 = 0; s0 < steps; s0 += kChienSeg) {
#pragma unroll
    for (int g = 0; g < kChienSeg; g++) {
      uint32_t acc = 0;
#pragma unroll
      for (int j = 1; j <= D; j++) acc ^= sexp[Ep[j - 1] - 32u * j * g];
      const int i = 32 * (s0 + g) + lane;
      if (acc == 1u && i < B.n) {
        roots++;
        flip_root(B, i, mo);
      }
    }
#pragma unroll
    for (int j = 1; j <= D; j++) {
      const uint32_t e = Ep[j - 1] - 32u * j * kChienSeg;
      Ep[j - 1] = e < (uint32_t)kChienOff ? e + N : e;
    }
    if ((int)__reduce_add_sync(0xffffffffu, (unsigned)roots) == D) break;
  }
  return (int)__reduce_add_sync(0xffffffffu, (unsigned)roots);
}

// Any degree (up to 31) and zero coefficients.
__device__ __forceinline__ int chien_generic(const BchDev& B, const uint16_t* __restrict__ sexp, uint32_t myL, int deg,
                                          int lane, uint64_t* mo) {
  const uint32_t N = (uint32_t)B.N;
  uint32_t E[31], M[31];
  for (int j = 1; j <= deg; j++) {
    const uint32_t Lj = __shfl_sync(0xffffffffu, myL, j);
    M[j - 1] = Lj == kLogZero ? 0u : 0xffffu;
    E[j - 1] = Lj == kLogZero ? 0u : (Lj + N - (uint32_t)(j * lane)) % N;
  }
  int roots = 0;
  const int steps = (B.n + 31) >> 5;
  for (int s = 0; s < steps; s++) {
    uint32_t acc = 0;
    for (int j = 1; j <= deg; j++) {
      acc ^= sexp[E[j - 1] + kChienOff] & M[j - 1];
      const uint32_t e = E[j - 1] - 32u * j;
      E[j - 1] = min(e, e + N);
    }
    const int i = 32 * s + lane;
    if (acc == 1u && i < B.n) {
      roots++;
      flip_root(B, i, mo);
    }
    if ((s & 7) == 7 && (int)__reduce_add_sync(0xffffffffu, (unsigned)roots) == deg) break;
  }
  return (int)__reduce_add_sync(0xffffffffu, (unsigned)roots);
}

// Kernel 2 of the decoder: Chien search of the frames with a nonzero locator.
// Work is taken from the per-degree lists in the order generic, 12, 11, ..., 1,
// so the warps of an SM mostly run the same unrolled evaluator (one
// instruction stream) and the longest frames start first.
__global__ void __launch_bounds__(kChienThreads, 1) bch_chien_kernel(const BchDev B, long long frames,
                                                                     const uint16_t* __restrict__ loc,
                                                                     const int32_t* __restrict__ degs,
                                                                     const uint32_t* __restrict__ bcnt,
                                                                     const int32_t* __restrict__ blist,
                                                                     uint64_t* __restrict__ msg,
                                                                     int32_t* __restrict__ nflips,
                                                                     unsigned long long* __restrict__ next) {
  extern __shared__ __align__(16) uint16_t sexp[];  // [N + kChienOff]: alpha^(x - kChienOff)
  __shared__ long long s_pre[kChienFastMax + 2];     // work offsets of the buckets in fetch order
  for (int i = threadIdx.x; i < B.N + kChienOff; i += blockDim.x) sexp[i] = B.exp[i + B.N - kChienOff];
  if (threadIdx.x == 0) {
    s_pre[0] = 0;
    for (int k = 0; k <= kChienFastMax; k++) s_pre[k + 1] = s_pre[k] + bcnt[k == 0 ? 0 : kChienFastMax + 1 - k];
  }
  __syncthreads();
  const long long total = s_pre[kChienFastMax + 1];
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(next, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if ((long long)w >= total) break;
    int k = 0;
    while ((long long)w >= s_pre[k + 1]) k++;
    const int bk = k == 0 ? 0 : kChienFastMax + 1 - k;
    const long long f = blist[(size_t)bk * frames + (size_t)((long long)w - s_pre[k])];
    const uint32_t myL = loc[f * 32 + lane];
    uint64_t* mo = msg + f * B.words_k;
    int roots;
    switch (bk) {
      case 1: roots = chien_fast<1>(B, sexp, myL, lane, mo); break;
      case 2: roots = chien_fast<2>(B, sexp, myL, lane, mo); break;
      case 3: roots = chien_fast<3>(B, sexp, myL, lane, mo); break;
      case 4: roots = chien_fast<4>(B, sexp, myL, lane, mo); break;
      case 5: roots = chien_fast<5>(B, sexp, myL, lane, mo); break;
      case 6: roots = chien_fast<6>(B, sexp, myL, lane, mo); break;
      case 7: roots = chien_fast<7>(B, sexp, myL, lane, mo); break;
      case 8: roots = chien_fast<8>(B, sexp, myL, lane, mo); break;
      case 9: roots = chien_fast<9>(B, sexp, myL, lane, mo); break;
      case 10: roots = chien_fast<10>(B, sexp, myL, lane, mo); break;
      case 11: roots = chien_fast<11>(B, sexp, myL, lane, mo); break;
      case 12: roots = chien_fast<12>(B, sexp, myL, lane, mo); break;
      default: roots = chien_generic(B, sexp, myL, degs[f], lane, mo); break;
    }
    if (lane == 0 && nflips) nflips[f] = roots;
  }
}

}  // namespace gf2c

using namespace gf2c;

struct gf2c_bch {
  int frame = 0, rate = 0, dev = -1, sms = 148;
  int occ_syn = 1, occ_enc = 1, occ_chien = 1;
  BchDev d{};
  std::vector<uint16_t> h_exp, h_log, h_mul;
  std::vector<uint64_t> h_quad;
  std::vector<uint32_t> h_lf, h_acol;
  std::vector<uint8_t> g;
  std::vector<void*> allocs;
  static constexpr int kStages = 8;
  void* stage[kStages] = {};
  size_t stage_bytes[kStages] = {};
  ~gf2c_bch() {
    for (void* p : allocs) cudaFree(p);
    for (void* p : stage)
      if (p) cudaFree(p);
  }
  int ensure_stage(int i, size_t bytes) {
    if (bytes <= stage_bytes[i]) return GF2C_OK;
    if (stage[i]) cudaFree(stage[i]);
    stage[i] = nullptr;
    stage_bytes[i] = 0;
    GF2C_CUDA(cudaMalloc(&stage[i], std::max(bytes, (size_t)256)));
    stage_bytes[i] = std::max(bytes, (size_t)256);
    return GF2C_OK;
  }
};

namespace {

// ETSI EN 302 755 generator factors g_1..g_12 (exponent lists of binary
// polynomials; standard data).
const int kShortGen[12][12] = {
    {0, 1, 3, 5, 14, -1},          {0, 6, 8, 11, 14, -1},         {0, 1, 2, 6, 9, 10, 14, -1},
    {0, 4, 7, 8, 10, 12, 14, -1},  {0, 2, 4, 6, 8, 9, 11, 13, 14, -1}, {0, 3, 7, 8, 9, 13, 14, -1},
    {0, 2, 5, 6, 7, 10, 11, 13, 14, -1}, {0, 5, 8, 9, 10, 11, 14, -1}, {0, 1, 2, 3, 9, 10, 14, -1},
    {0, 3, 6, 9, 11, 12, 14, -1},  {0, 4, 11, 12, 14, -1},        {0, 1, 2, 3, 5, 6, 7, 8, 10, 13, 14, -1}};
const int kNormalGen[12][14] = {
    {0, 2, 3, 5, 16, -1},
    {0, 1, 4, 5, 6, 8, 16, -1},
    {0, 2, 3, 4, 5, 7, 8, 9, 10, 11, 16, -1},
    {0, 2, 4, 6, 9, 11, 12, 14, 16, -1},
    {0, 1, 2, 3, 5, 8, 9, 10, 11, 12, 16, -1},
    {0, 2, 4, 5, 7, 8, 9, 10, 12, 13, 14, 15, 16, -1},
    {0, 2, 5, 6, 8, 9, 10, 11, 13, 15, 16, -1},
    {0, 1, 2, 5, 6, 8, 9, 12, 13, 14, 16, -1},
    {0, 5, 7, 9, 10, 11, 16, -1},
    {0, 1, 2, 5, 7, 8, 10, 12, 13, 14, 16, -1},
    {0, 2, 3, 5, 9, 11, 12, 13, 16, -1},
    {0, 1, 5, 6, 7, 9, 11, 12, 16, -1}};

template <class T>
int dev_upload(gf2c_bch* b, const std::vector<T>& v, const T** out) {
  void* p = nullptr;
  GF2C_CUDA(cudaMalloc(&p, std::max(sizeof(T) * v.size(), (size_t)16)));
  b->allocs.push_back(p);
  GF2C_CUDA(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  *out = (const T*)p;
  return GF2C_OK;
}

template <int T>
size_t enc_smem() { return syn_smem_bytes<T>() + kBchWarps * 8 * 4 + kBchWarps * 16 * 2; }
template <int T>
size_t syn_smem() { return syn_smem_bytes<T>() + kBchWarps * 32 * 2; }

template <int T>
int set_kernel_attrs(gf2c_bch* b) {
  GF2C_CUDA(cudaFuncSetAttribute(bch_encode_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)enc_smem<T>()));
  GF2C_CUDA(cudaFuncSetAttribute(bch_syndrome_bm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)syn_smem<T>()));
  GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_enc, bch_encode_kernel<T>, kBchWarps * 32,
                                                          enc_smem<T>()));
  GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_syn, bch_syndrome_bm_kernel<T>, kBchWarps * 32,
                                                          syn_smem<T>()));
  return GF2C_OK;
}

int bch_upload(gf2c_bch* b) {
  int dev = 0;
  GF2C_CUDA(cudaGetDevice(&dev));
  if (b->dev == dev) return GF2C_OK;
  if (b->dev >= 0) return set_error(GF2C_ERR_UNSUPPORTED, "BCH code already bound to another device");
  int rc;
  const uint64_t* quad = nullptr;
  if ((rc = dev_upload(b, b->h_exp, &b->d.exp)) || (rc = dev_upload(b, b->h_log, &b->d.log)) ||
      (rc = dev_upload(b, b->h_quad, &quad)) || (rc = dev_upload(b, b->h_mul, &b->d.mul)) ||
      (rc = dev_upload(b, b->h_lf, &b->d.lf)) || (rc = dev_upload(b, b->h_acol, &b->d.acol)))
    return rc;
  b->d.quad = (const uint2*)quad;
  GF2C_CUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev));
  if ((rc = b->d.t == 12 ? set_kernel_attrs<12>(b) : set_kernel_attrs<10>(b))) return rc;
  const int chien_smem = (b->d.N + kChienOff) * 2;
  GF2C_CUDA(cudaFuncSetAttribute(bch_chien_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, chien_smem));
  GF2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_chien, bch_chien_kernel, kChienThreads, chien_smem));
  b->occ_enc = std::max(b->occ_enc, 1);
  b->occ_syn = std::max(b->occ_syn, 1);
  b->occ_chien = std::max(b->occ_chien, 1);
  b->dev = dev;
  return GF2C_OK;
}

int warp_grid(long long frames, int sms, int occ) {
  const long long want = (frames + kBchWarps - 1) / kBchWarps;
  return (int)std::max<long long>(1, std::min<long long>(want, (long long)sms * occ));
}

// Inverse over GF(2) of the r x r matrix given as rows of bits; false if singular.
bool gf2_invert(int r, std::vector<std::vector<uint64_t>>& rows, std::vector<std::vector<uint64_t>>& inv) {
  const int W = (r + 63) / 64;
  inv.assign(r, std::vector<uint64_t>(W, 0));
  for (int i = 0; i < r; i++) inv[i][i >> 6] |= 1ull << (i & 63);
  for (int c = 0; c < r; c++) {
    int piv = -1;
    for (int i = c; i < r; i++)
      if ((rows[i][c >> 6] >> (c & 63)) & 1) {
        piv = i;
        break;
      }
    if (piv < 0) return false;
    std::swap(rows[c], rows[piv]);
    std::swap(inv[c], inv[piv]);
    for (int i = 0; i < r; i++)
      if (i != c && ((rows[i][c >> 6] >> (c & 63)) & 1))
        for (int w = 0; w < W; w++) {
          rows[i][w] ^= rows[c][w];
          inv[i][w] ^= inv[c][w];
        }
  }
  return true;
}

}  // namespace

extern "C" {

int gf2c_bch_create_dvbt2(int32_t frame_size, int32_t rate, gf2c_bch** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (frame_size < 0 || frame_size > 1 || rate < 0 || rate > 5)
    return set_error(GF2C_ERR_INVALID_ARG, "DVB-T2 frame size must be 0/1 and rate 0..5");
  static const int kShortN[6] = {7200, 9720, 10800, 11880, 12600, 13320};
  static const int kShortK[6] = {7032, 9552, 10632, 11712, 12432, 13152};
  static const int kNormalN[6] = {32400, 38880, 43200, 48600, 51840, 54000};
  static const int kNormalK[6] = {32208, 38688, 43040, 48408, 51648, 53840};
  static const int kNormalT[6] = {12, 12, 10, 12, 12, 10};
  std::unique_ptr<gf2c_bch> b(new (std::nothrow) gf2c_bch());
  if (!b) return set_error(GF2C_ERR_NOMEM, "out of host memory");
  const bool shortf = frame_size == 1;
  BchDev& d = b->d;
  b->frame = frame_size;
  b->rate = rate;
  d.n = shortf ? kShortN[rate] : kNormalN[rate];
  d.k = shortf ? kShortK[rate] : kNormalK[rate];
  d.t = shortf ? 12 : kNormalT[rate];
  d.r = d.n - d.k;
  d.m = shortf ? 14 : 16;
  const uint32_t prim = shortf ? 0b100000000101011u : 0b10000000000101101u;
  const int q = 1 << d.m;
  d.N = q - 1;
  d.words_n = (d.n + 63) / 64;
  d.words_k = (d.k + 63) / 64;
  d.rw = (d.r + 31) / 32;
  // antilog / log tables of GF(2^m), alpha = x
  b->h_exp.assign(2 * d.N, 0);
  b->h_log.assign(q, 0);
  uint32_t x = 1;
  for (int e = 0; e < d.N; e++) {
    b->h_exp[e] = (uint16_t)x;
    b->h_log[x] = (uint16_t)e;
    x <<= 1;
    if (x & (uint32_t)q) x ^= prim;
  }
  for (int e = d.N; e < 2 * d.N; e++) b->h_exp[e] = b->h_exp[e - d.N];
  auto apow = [&](long long e) -> uint32_t { return b->h_exp[((e % d.N) + d.N) % d.N]; };
  auto mul = [&](uint32_t a, uint32_t c) -> uint32_t {
    return (a && c) ? b->h_exp[b->h_log[a] + b->h_log[c]] : 0u;
  };
  // generator g = g_1 ... g_t (binary)
  std::vector<uint8_t> g{1};
  for (int i = 0; i < d.t; i++) {
    std::vector<uint8_t> fct(d.m + 1, 0);
    for (int j = 0;; j++) {
      const int e = shortf ? kShortGen[i][j] : kNormalGen[i][j];
      if (e < 0) break;
      fct[e] = 1;
    }
    std::vector<uint8_t> p(g.size() + fct.size() - 1, 0);
    for (size_t a = 0; a < g.size(); a++)
      if (g[a])
        for (size_t c = 0; c < fct.size(); c++) p[a + c] ^= fct[c];
    g = p;
  }
  if ((int)g.size() - 1 != d.r || d.r != d.t * d.m)
    return set_error(GF2C_ERR_KERNEL, "internal: BCH generator degree mismatch");
  b->g = g;
  // syndrome tables, odd j = 2s+1, beta = alpha^-j
  b->h_quad.assign((size_t)3 * 8 * 256, 0);
  b->h_mul.assign((size_t)d.t * 512, 0);
  b->h_lf.assign((size_t)d.t * 32, 0);
  for (int s = 0; s < d.t; s++) {
    const long long j = 2 * s + 1;
    for (int p = 0; p < 8; p++) {
      uint32_t unit[8];
      for (int e = 0; e < 8; e++) unit[e] = apow(-j * (8 * p + e));
      for (int v = 0; v < 256; v++) {
        uint64_t acc = 0;
        for (int e = 0; e < 8; e++)
          if ((v >> e) & 1) acc ^= unit[e];
        b->h_quad[((size_t)(s / 4) * 8 + p) * 256 + v] |= acc << (16 * (s % 4));
      }
    }
    const uint32_t gamma = apow(-j * 2048);
    for (int v = 0; v < 256; v++) {
      b->h_mul[(size_t)s * 512 + v] = (uint16_t)mul((uint32_t)v, gamma);
      const uint32_t hv = (uint32_t)v << 8;
      b->h_mul[(size_t)s * 512 + 256 + v] = hv < (uint32_t)q ? (uint16_t)mul(hv, gamma) : 0;
    }
    for (int lane = 0; lane < 32; lane++)
      b->h_lf[(size_t)s * 32 + lane] = (uint32_t)((j * (d.n - 1 - 64 * lane)) % d.N);
  }
  // parity from odd syndromes: P[b][q] = bit (b % m) of S_(2(b/m)+1) of parity bit q
  // (codeword bit k+q, degree r-1-q); A = P^-1, stored by column b
  {
    const int W = (d.r + 63) / 64;
    std::vector<std::vector<uint64_t>> P(d.r, std::vector<uint64_t>(W, 0)), A;
    for (int qb = 0; qb < d.r; qb++)
      for (int s = 0; s < d.t; s++) {
        const uint32_t v = apow((long long)(2 * s + 1) * (d.r - 1 - qb));
        for (int bp = 0; bp < d.m; bp++)
          if ((v >> bp) & 1) P[s * d.m + bp][qb >> 6] |= 1ull << (qb & 63);
      }
    if (!gf2_invert(d.r, P, A)) return set_error(GF2C_ERR_KERNEL, "internal: BCH parity map is singular");
    b->h_acol.assign((size_t)d.r * d.rw, 0);
    for (int qb = 0; qb < d.r; qb++)
      for (int bb = 0; bb < d.r; bb++)
        if ((A[qb][bb >> 6] >> (bb & 63)) & 1) b->h_acol[(size_t)bb * d.rw + (qb >> 5)] |= 1u << (qb & 31);
  }
  *out = b.release();
  return GF2C_OK;
}

int gf2c_bch_destroy(gf2c_bch* bch) {
  delete bch;
  return GF2C_OK;
}

int gf2c_bch_dims(const gf2c_bch* bch, int64_t* n, int64_t* k, int32_t* t, int32_t* field_m) {
  if (!bch) return set_error(GF2C_ERR_INVALID_ARG, "bch is NULL");
  if (n) *n = bch->d.n;
  if (k) *k = bch->d.k;
  if (t) *t = bch->d.t;
  if (field_m) *field_m = bch->d.m;
  return GF2C_OK;
}

int gf2c_bch_generator(const gf2c_bch* bch, uint8_t* coeffs) {
  if (!bch || !coeffs) return set_error(GF2C_ERR_INVALID_ARG, "NULL argument");
  std::memcpy(coeffs, bch->g.data(), bch->g.size());
  return GF2C_OK;
}

int gf2c_bch_encode_batch(gf2c_bch* bch, const uint64_t* msg_bits, int64_t frames, uint64_t* cw_bits,
                          int32_t mem, void* stream) {
  if (!bch || frames < 0 || (frames > 0 && (!msg_bits || !cw_bits)) || (mem != GF2C_MEM_HOST && mem != GF2C_MEM_DEVICE))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (frames == 0) return GF2C_OK;
  int rc = bch_upload(bch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const BchDev& d = bch->d;
  const size_t bin = (size_t)frames * d.words_k * 8, bout = (size_t)frames * d.words_n * 8;
  const uint64_t* in = msg_bits;
  uint64_t* out = cw_bits;
  if (mem == GF2C_MEM_HOST) {
    if ((rc = bch->ensure_stage(0, bin)) || (rc = bch->ensure_stage(1, bout))) return rc;
    GF2C_CUDA(cudaMemcpyAsync(bch->stage[0], msg_bits, bin, cudaMemcpyHostToDevice, st));
    in = (const uint64_t*)bch->stage[0];
    out = (uint64_t*)bch->stage[1];
  }
  const int grid = warp_grid(frames, bch->sms, bch->occ_enc);
  if (d.t == 12) bch_encode_kernel<12><<<grid, kBchWarps * 32, enc_smem<12>(), st>>>(d, in, frames, out);
  else bch_encode_kernel<10><<<grid, kBchWarps * 32, enc_smem<10>(), st>>>(d, in, frames, out);
  GF2C_CUDA(cudaGetLastError());
  if (mem == GF2C_MEM_HOST) {
    GF2C_CUDA(cudaMemcpyAsync(cw_bits, out, bout, cudaMemcpyDeviceToHost, st));
    GF2C_CUDA(cudaStreamSynchronize(st));
  }
  return GF2C_OK;
}

int gf2c_bch_decode_batch(gf2c_bch* bch, const uint64_t* cw_bits, int64_t frames, uint64_t* msg_bits,
                          int32_t* corrected, uint16_t* syndromes, int32_t mem, void* stream) {
  if (!bch || frames < 0 || (frames > 0 && (!cw_bits || !msg_bits)) || (mem != GF2C_MEM_HOST && mem != GF2C_MEM_DEVICE))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (frames == 0) return GF2C_OK;
  int rc = bch_upload(bch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const BchDev& d = bch->d;
  const size_t bin = (size_t)frames * d.words_n * 8, bout = (size_t)frames * d.words_k * 8;
  const size_t bc = (size_t)frames * 4, bs = (size_t)frames * 2 * d.t * 2;
  if ((rc = bch->ensure_stage(4, (size_t)frames * 32 * 2)) || (rc = bch->ensure_stage(5, (size_t)frames * 4)) ||
      (rc = bch->ensure_stage(6, 128)) || (rc = bch->ensure_stage(7, (size_t)(kChienFastMax + 1) * frames * 4)))
    return rc;
  const uint64_t* in = cw_bits;
  uint64_t* out = msg_bits;
  int32_t* cor = corrected;
  uint16_t* syn = syndromes;
  if (mem == GF2C_MEM_HOST) {
    if ((rc = bch->ensure_stage(0, bin)) || (rc = bch->ensure_stage(1, bout)) ||
        (corrected && (rc = bch->ensure_stage(2, bc))) || (syndromes && (rc = bch->ensure_stage(3, bs))))
      return rc;
    GF2C_CUDA(cudaMemcpyAsync(bch->stage[0], cw_bits, bin, cudaMemcpyHostToDevice, st));
    in = (const uint64_t*)bch->stage[0];
    out = (uint64_t*)bch->stage[1];
    cor = corrected ? (int32_t*)bch->stage[2] : nullptr;
    syn = syndromes ? (uint16_t*)bch->stage[3] : nullptr;
  }
  uint16_t* loc = (uint16_t*)bch->stage[4];
  int32_t* degs = (int32_t*)bch->stage[5];
  unsigned long long* next = (unsigned long long*)bch->stage[6];  // work counter, then bucket sizes
  uint32_t* bcnt = (uint32_t*)((char*)bch->stage[6] + 64);
  int32_t* blist = (int32_t*)bch->stage[7];
  GF2C_CUDA(cudaMemsetAsync(bch->stage[6], 0, 128, st));
  const int grid = warp_grid(frames, bch->sms, bch->occ_syn);
  if (d.t == 12)
    bch_syndrome_bm_kernel<12><<<grid, kBchWarps * 32, syn_smem<12>(), st>>>(d, in, frames, out, cor, syn, loc, degs, bcnt, blist);
  else
    bch_syndrome_bm_kernel<10><<<grid, kBchWarps * 32, syn_smem<10>(), st>>>(d, in, frames, out, cor, syn, loc, degs, bcnt, blist);
  GF2C_CUDA(cudaGetLastError());
  bch_chien_kernel<<<bch->sms * bch->occ_chien, kChienThreads, (size_t)(d.N + kChienOff) * 2, st>>>(
      d, frames, loc, degs, bcnt, blist, out, cor, next);
  GF2C_CUDA(cudaGetLastError());
  if (mem == GF2C_MEM_HOST) {
    GF2C_CUDA(cudaMemcpyAsync(msg_bits, out, bout, cudaMemcpyDeviceToHost, st));
    if (corrected) GF2C_CUDA(cudaMemcpyAsync(corrected, cor, bc, cudaMemcpyDeviceToHost, st));
    if (syndromes) GF2C_CUDA(cudaMemcpyAsync(syndromes, syn, bs, cudaMemcpyDeviceToHost, st));
    GF2C_CUDA(cudaStreamSynchronize(st));
  }
  return GF2C_OK;
}

}  // extern "C"
