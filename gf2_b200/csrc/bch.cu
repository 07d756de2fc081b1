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
// GPU layout: one warp per frame, frames from a grid-stride loop.
//  * Encoder: parity = XOR over the set message bits i of the remainder row
//    x^(r + k-1-i) mod g (precomputed per code, r bits, L2-resident); lanes
//    split the message bits and XOR-reduce their rows.
//  * Syndromes: S_j = alpha^(j(n-1)) * sum_i b_i beta^i with beta = alpha^-j.
//    Per 64-bit word of the codeword the inner sum is 8 lookups in per-(j,
//    byte position) tables of 256 entries (shared memory, odd j only), then
//    one multiplication by beta^(64 w); even syndromes are squares (binary
//    received word: r(alpha^2j) = r(alpha^j)^2).
//  * Frames with a nonzero syndrome: lane 0 runs the reference's
//    Berlekamp-Massey step for step, then the lanes evaluate the locator at
//    alpha^-i for their positions i (Chien search) and flip the bits of the
//    roots that fall in the message.
// Field multiplications use log / antilog tables (global memory, L1-cached).
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "internal.h"

namespace gf2c {

static constexpr int kBchMaxT = 12;
static constexpr int kBchWarps = 8;  // frames per CTA at a time

struct BchDev {
  int n, k, t, r, N, words_n, words_k, rw;  // rw = 32-bit words of a parity row
  const uint16_t* exp;   // [2N]
  const uint16_t* log;   // [N + 1]
  const uint16_t* stab;  // [t][8][256]: odd j = 2s+1, byte position p
  const uint32_t* erow;  // [k][rw]: x^(r + d) mod g in parity-bit order
};

__device__ __forceinline__ uint16_t gf_mul(const BchDev& B, uint16_t a, uint16_t b) {
  if (!a || !b) return 0;
  return __ldg(&B.exp[__ldg(&B.log[a]) + __ldg(&B.log[b])]);
}
// a * alpha^e, 0 <= e < N
__device__ __forceinline__ uint16_t gf_mul_pow(const BchDev& B, uint16_t a, int e) {
  if (!a) return 0;
  return __ldg(&B.exp[__ldg(&B.log[a]) + e]);
}

__global__ void __launch_bounds__(kBchWarps * 32) bch_encode_kernel(const BchDev B, const uint64_t* __restrict__ msg,
                                                                    long long frames, uint64_t* __restrict__ cw) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * kBchWarps;
  for (long long f = (long long)blockIdx.x * kBchWarps + (threadIdx.x >> 5); f < frames; f += warps) {
    const uint64_t* m = msg + f * B.words_k;
    uint32_t acc[6] = {0, 0, 0, 0, 0, 0};
    for (int w = lane; w < B.words_k; w += 32) {
      uint64_t bits = m[w];
      if (w == B.words_k - 1 && (B.k & 63)) bits &= (1ull << (B.k & 63)) - 1ull;
      while (bits) {
        const int e = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        const uint32_t* row = B.erow + (size_t)(B.k - 1 - (64 * w + e)) * B.rw;
#pragma unroll
        for (int q = 0; q < 6; q++)
          if (q < B.rw) acc[q] ^= __ldg(&row[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] ^= __shfl_xor_sync(0xffffffffu, acc[q], o);
    // codeword word w = message bits (< k) | parity bits (k .. n-1)
    uint64_t* c = cw + f * B.words_n;
    for (int w = lane; w < B.words_n; w += 32) {
      const int b0 = 64 * w;
      uint64_t word = 0;
      if (b0 < B.k) {
        word = m[w];
        if (b0 + 64 > B.k) word &= (1ull << (B.k - b0)) - 1ull;
      }
      for (int e = max(0, B.k - b0); e < 64 && b0 + e < B.n; e++) {
        const int q = b0 + e - B.k;
        word |= (uint64_t)((acc[q >> 5] >> (q & 31)) & 1u) << e;
      }
      c[w] = word;
    }
  }
}

__global__ void __launch_bounds__(kBchWarps * 32) bch_decode_kernel(const BchDev B, const uint64_t* __restrict__ cw,
                                                                    long long frames, uint64_t* __restrict__ msg,
                                                                    int32_t* __restrict__ nflips,
                                                                    uint16_t* __restrict__ synd_out) {
  extern __shared__ uint16_t s_tab[];  // [t][8][256]
  for (int i = threadIdx.x; i < B.t * 8 * 256; i += blockDim.x) s_tab[i] = B.stab[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * kBchWarps;
  for (long long f = (long long)blockIdx.x * kBchWarps + (threadIdx.x >> 5); f < frames; f += warps) {
    const uint64_t* c = cw + f * B.words_n;
    // odd syndromes (partial sums of this lane's words)
    uint16_t so[kBchMaxT];
#pragma unroll
    for (int s = 0; s < kBchMaxT; s++) so[s] = 0;
    for (int w = lane; w < B.words_n; w += 32) {
      uint64_t word = c[w];
      if (w == B.words_n - 1 && (B.n & 63)) word &= (1ull << (B.n & 63)) - 1ull;
      if (!word) continue;
#pragma unroll
      for (int s = 0; s < kBchMaxT; s++) {
        if (s < B.t) {
          const uint16_t* T = s_tab + s * 2048;
          uint16_t q = 0;
#pragma unroll
          for (int p = 0; p < 8; p++) q ^= T[p * 256 + (int)((word >> (8 * p)) & 0xff)];
          // * beta^(64 w), beta = alpha^-(2s+1)
          const long long e = (long long)(B.N - ((64LL * w * (2 * s + 1)) % B.N)) % B.N;
          so[s] ^= gf_mul_pow(B, q, (int)e);
        }
      }
    }
    uint32_t any = 0;
#pragma unroll
    for (int s = 0; s < kBchMaxT; s++) {
      uint32_t v = so[s];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v ^= __shfl_xor_sync(0xffffffffu, v, o);
      // * alpha^(j (n-1))
      so[s] = (s < B.t) ? gf_mul_pow(B, (uint16_t)v, (int)(((long long)(2 * s + 1) * (B.n - 1)) % B.N)) : 0;
      any |= so[s];
    }
    // message bits as received
    uint64_t* mo = msg + f * B.words_k;
    for (int w = lane; w < B.words_k; w += 32) {
      uint64_t word = c[w];
      if (w == B.words_k - 1 && (B.k & 63)) word &= (1ull << (B.k & 63)) - 1ull;
      mo[w] = word;
    }
    __syncwarp();  // the copies are visible to the lanes that flip bits below
    if (synd_out || any) {
      uint16_t S[2 * kBchMaxT];  // S[j-1] = S_j
#pragma unroll
      for (int j = 1; j <= 2 * kBchMaxT; j++) {
        if (j & 1) S[j - 1] = so[(j - 1) >> 1];
        else S[j - 1] = gf_mul(B, S[j / 2 - 1], S[j / 2 - 1]);
      }
      if (synd_out && lane == 0)
        for (int j = 0; j < 2 * B.t; j++) synd_out[f * 2 * B.t + j] = S[j];
      if (!any) {
        if (lane == 0 && nflips) nflips[f] = 0;
        continue;
      }
      // Berlekamp-Massey (BchDecoder::berlekamp_massey), on lane 0
      uint16_t lam[2 * kBchMaxT + 2];
      int deg = 0;
      if (lane == 0) {
        uint16_t bb[2 * kBchMaxT + 2], tt[2 * kBchMaxT + 2];
        for (int i = 0; i < 2 * kBchMaxT + 2; i++) lam[i] = bb[i] = 0;
        lam[0] = bb[0] = 1;
        int l = 0, m = 1, dl = 0, db = 0;
        for (int nn = 0; nn < 2 * B.t; nn++) {
          uint16_t delta = S[nn];
          for (int i = 1; i <= l; i++)
            if (i <= dl && nn >= i) delta ^= gf_mul(B, lam[i], S[nn - i]);
          if (delta == 0) {
            m += 1;
            continue;
          }
          for (int i = 0; i <= dl; i++) tt[i] = lam[i];
          const int dt = dl;
          for (int i = 0; i <= db && m + i < 2 * kBchMaxT + 2; i++) lam[m + i] ^= gf_mul(B, delta, bb[i]);
          dl = 0;
          for (int i = 2 * kBchMaxT + 1; i > 0; i--)
            if (lam[i]) {
              dl = i;
              break;
            }
          if (2 * l <= nn) {
            l = nn + 1 - l;
            const uint16_t di = __ldg(&B.exp[(B.N - __ldg(&B.log[delta])) % B.N]);
            for (int i = 0; i < 2 * kBchMaxT + 2; i++) bb[i] = 0;
            db = 0;
            for (int i = 0; i <= dt; i++) {
              bb[i] = gf_mul(B, tt[i], di);
              if (bb[i]) db = i;
            }
            m = 1;
          } else {
            m += 1;
          }
        }
        deg = dl;
      }
      deg = __shfl_sync(0xffffffffu, deg, 0);
      // Chien search: lambda(alpha^-i) for degrees i = lane + 32 s
      int L[2 * kBchMaxT + 2], stepv[2 * kBchMaxT + 2];
      int roots = 0;
      if (deg > 0) {
        for (int j = 0; j <= deg; j++) {
          const uint32_t lj = __shfl_sync(0xffffffffu, (uint32_t)lam[j], 0);
          L[j] = lj ? (int)__ldg(&B.log[lj]) : -1;
          // exponent of the term at i = lane: log(lambda_j) - j * lane (mod N)
          if (L[j] >= 0) L[j] = (int)(((long long)L[j] - (long long)j * lane % B.N + B.N) % B.N);
          stepv[j] = (int)((32LL * j) % B.N);
        }
        for (int i = lane; i < B.n; i += 32) {
          uint32_t e = 0;
          for (int j = 0; j <= deg; j++) {
            if (L[j] >= 0) {
              e ^= __ldg(&B.exp[L[j]]);
              L[j] -= stepv[j];
              if (L[j] < 0) L[j] += B.N;
            }
          }
          if (e == 0) {
            roots++;
            const int bit = B.n - 1 - i;
            if (bit < B.k) atomicXor((unsigned long long*)&mo[bit >> 6], 1ull << (bit & 63));
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(0xffffffffu, roots, o);
      if (lane == 0 && nflips) nflips[f] = roots;
    } else if (lane == 0 && nflips) {
      nflips[f] = 0;
    }
  }
}

}  // namespace gf2c

using namespace gf2c;

struct gf2c_bch {
  int frame = 0, rate = 0, dev = -1;
  BchDev d{};
  std::vector<uint16_t> h_exp, h_log, h_stab;
  std::vector<uint32_t> h_erow;
  std::vector<uint8_t> g;
  std::vector<void*> allocs;
  void* stage[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[4] = {0, 0, 0, 0};
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

int bch_upload(gf2c_bch* b) {
  int dev = 0;
  GF2C_CUDA(cudaGetDevice(&dev));
  if (b->dev == dev) return GF2C_OK;
  if (b->dev >= 0) return set_error(GF2C_ERR_UNSUPPORTED, "BCH code already bound to another device");
  int rc;
  if ((rc = dev_upload(b, b->h_exp, &b->d.exp)) || (rc = dev_upload(b, b->h_log, &b->d.log)) ||
      (rc = dev_upload(b, b->h_stab, &b->d.stab)) || (rc = dev_upload(b, b->h_erow, &b->d.erow)))
    return rc;
  b->dev = dev;
  return GF2C_OK;
}

int bch_grid(long long frames) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (frames + kBchWarps - 1) / kBchWarps;
  return (int)std::max<long long>(1, std::min<long long>(want, (long long)sms * 8));
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
  const int mf = shortf ? 14 : 16;
  const uint32_t prim = shortf ? 0b100000000101011u : 0b10000000000101101u;
  const int q = 1 << mf;
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
  auto apow = [&](long long e) { return b->h_exp[((e % d.N) + d.N) % d.N]; };
  // generator g = g_1 ... g_t (binary)
  std::vector<uint8_t> g{1};
  for (int i = 0; i < d.t; i++) {
    std::vector<uint8_t> fct(mf + 1, 0);
    for (int j = 0; ; j++) {
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
  if ((int)g.size() - 1 != d.r) return set_error(GF2C_ERR_KERNEL, "internal: BCH generator degree mismatch");
  b->g = g;
  // encoder rows: rem_d = x^(r + d) mod g, parity bit q = coefficient of degree r-1-q
  b->h_erow.assign((size_t)d.k * d.rw, 0);
  std::vector<uint8_t> rem(d.r, 0);
  for (int e = 0; e < d.r; e++) rem[e] = g[e];  // x^r mod g = lower part of g (binary)
  for (int dd = 0; dd < d.k; dd++) {
    uint32_t* row = &b->h_erow[(size_t)dd * d.rw];
    for (int qb = 0; qb < d.r; qb++)
      if (rem[d.r - 1 - qb]) row[qb >> 5] |= 1u << (qb & 31);
    const uint8_t top = rem[d.r - 1];  // multiply by x modulo g
    for (int e = d.r - 1; e > 0; e--) rem[e] = rem[e - 1] ^ (top & g[e]);
    rem[0] = top & g[0];
  }
  // syndrome tables: odd j = 2s+1, beta = alpha^-j, T[s][p][v] = sum_e v_e beta^(8p + e)
  b->h_stab.assign((size_t)d.t * 8 * 256, 0);
  for (int s = 0; s < d.t; s++) {
    const int j = 2 * s + 1;
    for (int p = 0; p < 8; p++) {
      uint16_t unit[8];
      for (int e = 0; e < 8; e++) unit[e] = apow(-(long long)j * (8 * p + e));
      for (int v = 0; v < 256; v++) {
        uint16_t acc = 0;
        for (int e = 0; e < 8; e++)
          if ((v >> e) & 1) acc ^= unit[e];
        b->h_stab[((size_t)s * 8 + p) * 256 + v] = acc;
      }
    }
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
  if (field_m) *field_m = bch->frame == 1 ? 14 : 16;
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
  bch_encode_kernel<<<bch_grid(frames), kBchWarps * 32, 0, st>>>(d, in, frames, out);
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
  const uint64_t* in = cw_bits;
  uint64_t* out = msg_bits;
  int32_t* cor = corrected;
  uint16_t* syn = syndromes;
  if (mem == GF2C_MEM_HOST) {
    if ((rc = bch->ensure_stage(0, bin)) || (rc = bch->ensure_stage(1, bout)) || (rc = bch->ensure_stage(2, bc)) ||
        (rc = bch->ensure_stage(3, bs)))
      return rc;
    GF2C_CUDA(cudaMemcpyAsync(bch->stage[0], cw_bits, bin, cudaMemcpyHostToDevice, st));
    in = (const uint64_t*)bch->stage[0];
    out = (uint64_t*)bch->stage[1];
    cor = corrected ? (int32_t*)bch->stage[2] : nullptr;
    syn = syndromes ? (uint16_t*)bch->stage[3] : nullptr;
  }
  const size_t smem = (size_t)d.t * 8 * 256 * sizeof(uint16_t);
  GF2C_CUDA(cudaFuncSetAttribute(bch_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  bch_decode_kernel<<<bch_grid(frames), kBchWarps * 32, smem, st>>>(d, in, frames, out, cor, syn);
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
