// gf2cuda dense-parity LDPC encoder (sm_100a): encodes with the parity part P
// of a systematic generator [I_k | P], as stored in the gf2 encoder cache
// (RuEncodingMatrices::encode, crates/gf2-coding/src/ldpc/encoding/
// richardson_urbanke.rs:263-290: parity = P^T message, message bits in
// columns [0, k), parity bit j in column k + j).
//
// P is k x r bits, row i = the parity of message bit i, rows of S = ceil(r/64)
// words (the BitMatrix layout).  parity(f) = XOR of the rows i with message bit
// i set.  A CTA computes 64 frames x 32 parity words: for every 64 message bits
// it builds, in shared memory, the 16 XOR combinations of each group of 4 rows
// (sixteen 4-row tables, 64 KB), then every frame adds one table entry per 4
// message bits.  A warp covers the 32 words of one frame, so its table reads
// are 32 consecutive 8-byte entries.  A second kernel assembles the codeword
// words [message | parity].
#include <algorithm>
#include <vector>

#include "internal.h"

namespace gf2c {

static constexpr int kDfFrames = 64;  // frames per CTA
static constexpr int kDfWords = 32;   // parity words per CTA
static constexpr size_t kDfSmem = (size_t)(16 * 16 * kDfWords + kDfFrames) * 8;  // tables + message words

__global__ void __launch_bounds__(256) dense_parity_kernel(const uint64_t* __restrict__ P, long long k, int S,
                                                           const uint64_t* __restrict__ msg, int wk, long long frames,
                                                           uint64_t* __restrict__ par) {
  extern __shared__ __align__(16) uint64_t dsm[];
  uint64_t (*T)[16][kDfWords] = reinterpret_cast<uint64_t (*)[16][kDfWords]>(dsm);  // [row group][nibble][word]
  uint64_t* sm = dsm + 16 * 16 * kDfWords;  // message word of each frame of the tile
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const long long f0 = (long long)blockIdx.x * kDfFrames;
  const int w = blockIdx.y * kDfWords + lane;
  const bool wok = w < S;
  uint64_t acc[8];
#pragma unroll
  for (int j = 0; j < 8; j++) acc[j] = 0;
  for (int c = 0; c < wk; c++) {
    if (threadIdx.x < kDfFrames) {
      const long long f = f0 + threadIdx.x;
      uint64_t m = f < frames ? msg[f * wk + c] : 0ull;
      if (c == wk - 1 && (k & 63)) m &= (1ull << (k & 63)) - 1ull;
      sm[threadIdx.x] = m;
    }
    // tables of row groups q = g and g + 8 (rows 64 c + 4 q .. + 3)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int q = g + 8 * h;
      uint64_t v[4];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const long long row = 64LL * c + 4 * q + b;
        v[b] = (wok && row < k) ? __ldg(&P[row * S + w]) : 0ull;
      }
      uint64_t t[16];
      t[0] = 0;
#pragma unroll
      for (int x = 1; x < 16; x++) t[x] = t[x & (x - 1)] ^ v[__ffs(x) - 1];
#pragma unroll
      for (int x = 0; x < 16; x++) T[q][x][lane] = t[x];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint64_t m = sm[g + 8 * j];
#pragma unroll
      for (int q = 0; q < 16; q++) acc[j] ^= T[q][(m >> (4 * q)) & 15u][lane];
    }
    __syncthreads();
  }
  if (wok)
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const long long f = f0 + g + 8 * j;
      if (f < frames) par[f * S + w] = acc[j];
    }
}

// codeword word w of frame f: message bits below k, parity bit j at k + j
__global__ void dense_assemble_kernel(const uint64_t* __restrict__ msg, const uint64_t* __restrict__ par,
                                      long long frames, long long k, long long n, int wk, int wn, int S,
                                      uint64_t* __restrict__ cw) {
  const long long total = frames * wn;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / wn;
    const int w = (int)(i - f * wn);
    const long long b0 = 64LL * w;
    const uint64_t* pf = par + f * S;
    uint64_t word;
    if (b0 + 64 <= k) {
      word = msg[f * wk + w];
    } else if (b0 >= k) {
      const long long o = b0 - k;
      const int q = (int)(o >> 6), sh = (int)(o & 63);
      word = pf[q] >> sh;
      if (sh && q + 1 < S) word |= pf[q + 1] << (64 - sh);
    } else {
      const int sh = (int)(k - b0);  // 1..63
      word = (msg[f * wk + w] & ((1ull << sh) - 1ull)) | (pf[0] << sh);
    }
    if (w == wn - 1 && (n & 63)) word &= (1ull << (n & 63)) - 1ull;
    cw[i] = word;
  }
}

}  // namespace gf2c

using namespace gf2c;

struct gf2c_dense_encoder {
  int64_t k = 0, n = 0, r = 0;
  int S = 0, wk = 0, wn = 0, dev = -1;
  std::vector<uint64_t> hp;
  uint64_t* P = nullptr;
  void* stage[3] = {nullptr, nullptr, nullptr};
  size_t stage_bytes[3] = {0, 0, 0};
  ~gf2c_dense_encoder() {
    if (P) cudaFree(P);
    for (void* p : stage)
      if (p) cudaFree(p);
  }
  int ensure(int i, size_t bytes) {
    if (bytes <= stage_bytes[i]) return GF2C_OK;
    if (stage[i]) cudaFree(stage[i]);
    stage[i] = nullptr;
    stage_bytes[i] = 0;
    GF2C_CUDA(cudaMalloc(&stage[i], std::max(bytes, (size_t)256)));
    stage_bytes[i] = std::max(bytes, (size_t)256);
    return GF2C_OK;
  }
};

extern "C" {

int gf2c_dense_encoder_create(const uint64_t* parity_words, int64_t k, int64_t n, gf2c_dense_encoder** out) {
  if (!out) return set_error(GF2C_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (k <= 0 || n <= k || !parity_words) return set_error(GF2C_ERR_INVALID_ARG, "dense encoder needs 0 < k < n and P");
  if (k > (1LL << 40) || (n - k + 63) / 64 > (1 << 30)) return set_error(GF2C_ERR_UNSUPPORTED, "dense encoder: too large");
  std::unique_ptr<gf2c_dense_encoder> e(new (std::nothrow) gf2c_dense_encoder());
  if (!e) return set_error(GF2C_ERR_NOMEM, "out of host memory");
  e->k = k;
  e->n = n;
  e->r = n - k;
  e->S = (int)((e->r + 63) / 64);
  e->wk = (int)((k + 63) / 64);
  e->wn = (int)((n + 63) / 64);
  e->hp.assign(parity_words, parity_words + (size_t)k * e->S);
  if (e->r & 63)
    for (int64_t i = 0; i < k; i++) e->hp[(size_t)i * e->S + e->S - 1] &= (1ull << (e->r & 63)) - 1ull;
  *out = e.release();
  return GF2C_OK;
}

int gf2c_dense_encoder_destroy(gf2c_dense_encoder* enc) {
  delete enc;
  return GF2C_OK;
}

int gf2c_dense_encode_batch(gf2c_dense_encoder* enc, const uint64_t* msg_bits, int64_t frames, uint64_t* cw_bits,
                            int32_t mem, void* stream) {
  if (!enc || frames < 0 || (frames > 0 && (!msg_bits || !cw_bits)) || (mem != GF2C_MEM_HOST && mem != GF2C_MEM_DEVICE))
    return set_error(GF2C_ERR_INVALID_ARG, "bad arguments");
  if (frames == 0) return GF2C_OK;
  int dev = 0;
  GF2C_CUDA(cudaGetDevice(&dev));
  if (enc->dev != dev) {
    if (enc->dev >= 0) return set_error(GF2C_ERR_UNSUPPORTED, "dense encoder already bound to another device");
    GF2C_CUDA(cudaMalloc(&enc->P, enc->hp.size() * 8));
    GF2C_CUDA(cudaMemcpy(enc->P, enc->hp.data(), enc->hp.size() * 8, cudaMemcpyHostToDevice));
    GF2C_CUDA(cudaFuncSetAttribute(dense_parity_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDfSmem));
    enc->dev = dev;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bin = (size_t)frames * enc->wk * 8, bout = (size_t)frames * enc->wn * 8;
  int rc;
  if ((rc = enc->ensure(2, (size_t)frames * enc->S * 8))) return rc;
  const uint64_t* in = msg_bits;
  uint64_t* out = cw_bits;
  if (mem == GF2C_MEM_HOST) {
    if ((rc = enc->ensure(0, bin)) || (rc = enc->ensure(1, bout))) return rc;
    GF2C_CUDA(cudaMemcpyAsync(enc->stage[0], msg_bits, bin, cudaMemcpyHostToDevice, st));
    in = (const uint64_t*)enc->stage[0];
    out = (uint64_t*)enc->stage[1];
  }
  uint64_t* par = (uint64_t*)enc->stage[2];
  const dim3 grid((unsigned)((frames + kDfFrames - 1) / kDfFrames), (unsigned)((enc->S + kDfWords - 1) / kDfWords));
  if (grid.x > 0x7fffffffu || grid.y > 65535u) return set_error(GF2C_ERR_UNSUPPORTED, "dense encoder: batch too large");
  dense_parity_kernel<<<grid, 256, kDfSmem, st>>>(enc->P, enc->k, enc->S, in, enc->wk, frames, par);
  GF2C_CUDA(cudaGetLastError());
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  dense_assemble_kernel<<<sms * 8, 256, 0, st>>>(in, par, frames, enc->k, enc->n, enc->wk, enc->wn, enc->S, out);
  GF2C_CUDA(cudaGetLastError());
  if (mem == GF2C_MEM_HOST) {
    GF2C_CUDA(cudaMemcpyAsync(cw_bits, out, bout, cudaMemcpyDeviceToHost, st));
    GF2C_CUDA(cudaStreamSynchronize(st));
  }
  return GF2C_OK;
}

}  // extern "C"
