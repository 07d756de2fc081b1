/* CPU oracle for the LDPC belief-propagation path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is a C++ restatement of the erankavija/gf2 `gf2-coding` LDPC
 * path (code construction, flooding min-sum decoder, syndrome, systematic
 * encoder, AWGN channel) plus the CPU judges for the decoder variants the GPU
 * library adds (sum-product, layered schedule, FP16 message storage, learned
 * normalised/offset min-sum).  It is used only by the tests, by the smoke
 * check and by the CPU-baseline leg of the benchmark, always as the checker
 * or the timed CPU baseline, never as the product.
 *
 * Parity pins: the reference is Rust and cannot be built in this image, so the
 * restatement is pinned by the reference's own known-answer tests (restated in
 * tests/test_oracle_kat.py) and by the structural statistics of the 12
 * DVB-T2 codes.  The AWGN noise of the reference comes from `rand_distr`
 * (unpinned, no Cargo.lock): that RNG boundary is replaced by a seeded
 * Philox4x32-10 stream shared with the GPU, and both sides decode the same
 * LLR buffer.
 *
 * Every function is plain C ABI (for ctypes).  Bits are passed one per byte
 * unless a name says "packed" (u64 words, LSB first, the BitVec convention of
 * crates/gf2-core/src/lib.rs:15-17).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_code or_code;

/* ---- code construction (restates ldpc/core.rs, dvb_t2/builder.rs, sparse.rs) ---- */
or_code* or_code_dvbt2(int frame /*0 normal, 1 short*/, int rate /*0..5*/);
or_code* or_code_qc(const int32_t* base, int mb, int nb, int z);
or_code* or_code_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count);
void or_code_free(or_code* c);
/* n, m, k = max(n-m,0), nnz */
void or_code_dims(const or_code* c, int64_t* out4);
/* CSR export: indptr (m+1), indices (nnz); CSC export: indptr (n+1), indices */
void or_code_csr(const or_code* c, int64_t* indptr, int64_t* indices);
void or_code_csc(const or_code* c, int64_t* indptr, int64_t* indices);
const char* or_last_error(void);

/* s = H c over GF(2); returns popcount of s */
int64_t or_syndrome(const or_code* c, const uint8_t* cw, uint8_t* synd /*nullable*/);

/* ---- decoders ----
 * llr: frames x n f32.  Outputs (each nullable): msg frames x k bytes,
 * iters/conv/synd_ok per frame, beliefs frames x n f32 (final posteriors).
 * threads <= 0 means all hardware threads.
 */
/* Reference-faithful flooding min-sum: the data structures and the loop of
 * LdpcDecoder::decode_iterative (core.rs:889-938), neighbour lists with linear
 * position searches (core.rs:841-856), one decoder per frame as in
 * decode_batch (core.rs:729-756), AVX2 min-sum emulation
 * (gf2-kernels-simd/src/llr.rs:117-180). */
int or_decode_minsum_faithful(const or_code* c, const float* llr, int64_t frames,
                              int max_iter, int threads, uint8_t* msg, int32_t* iters,
                              uint8_t* conv, uint8_t* synd_ok, float* beliefs);

/* Generic flooding/layered decoder with edge-indexed messages (fast oracle).
 * algo: 0 min-sum (reference arithmetic, sign = x < 0), 1 sum-product FP32
 * (library numeric spec), 2 sum-product FP64 (judge), 3 normalised/offset
 * min-sum with weights alpha[t*L + l], beta[t*L + l] (L = layers, t = iteration,
 * t clamped to n_wt_iters-1).
 * sched: 0 flooding, 1 layered (row groups of the QC structure).
 * msg16: 1 = messages stored as IEEE binary16 (round to nearest even).
 */
int or_decode(const or_code* c, const float* llr, int64_t frames, int max_iter,
              int algo, int sched, int msg16, const float* alpha, const float* beta,
              int n_wt_iters, int threads, uint8_t* msg, int32_t* iters, uint8_t* conv,
              uint8_t* synd_ok, float* beliefs);

/* FP64 variant of or_decode for algo 2 that also returns final posteriors as
 * f64 (frames x n).  Used as the FER judge and for LLR deviation reports. */
int or_decode_spa64(const or_code* c, const float* llr, int64_t frames, int max_iter,
                    int sched, int threads, uint8_t* msg, int32_t* iters, uint8_t* conv,
                    uint8_t* synd_ok, double* beliefs);

/* Number of layers of the layered schedule (row groups), 0 if none. */
int or_code_layers(const or_code* c);
/* Layer of each check (m entries). */
void or_code_check_layer(const or_code* c, int32_t* layer);

/* ---- encoder ---- */
/* Systematic encode: msg frames x k bytes -> cw frames x n bytes.  DVB-T2
 * codes use the staircase accumulator; other codes the right-greedy pivot
 * encoder of RuEncodingMatrices (richardson_urbanke.rs:158-289). */
int or_encode(const or_code* c, const uint8_t* msg, int64_t frames, uint8_t* cw);
/* parity (pivot) columns of the generic encoder, m entries; message columns k */
int or_encoder_columns(const or_code* c, int64_t* msg_cols, int64_t* par_cols);

/* ---- channel ---- */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* seeded frames: info bits (frames x k bytes), codeword, LLR (frames x n f32)
 * with per-frame Eb/N0 in dB (ebn0 has `frames` entries). rate = k/n. */
int or_channel_frames(const or_code* c, uint64_t seed, uint64_t frame0, int64_t frames,
                      const double* ebn0_db, uint8_t* info, uint8_t* cw, float* llr);
double or_sigma2(double ebn0_db, double rate);
double or_own_log(double x);
void or_own_sincos2pi(double u, double* s, double* c);
double or_shannon_limit(double rate);

/* ---- learned normalised/offset min-sum (flooding, T unrolled iterations) ----
 * c2v = sign * alpha[t,l] * max(min|v2c| - beta[t,l], 0), layer l of the check.
 * loss = mean over frames and all n bits of softplus(-(1-2b) * L_T).
 * Returns loss; fills grad_alpha/grad_beta (T*L each).  FP64 throughout. */
double or_nms_loss_grad(const or_code* c, const float* llr, const uint8_t* cw,
                        int64_t frames, int T, const double* alpha, const double* beta,
                        double* grad_alpha, double* grad_beta, double* out_llr);

/* The same with the layered schedule (row groups in order, posterior updated
 * after each row group, weights per iteration and row group); NaN and an error
 * message for codes without row groups. */
double or_nms_layered_loss_grad(const or_code* c, const float* llr, const uint8_t* cw,
                                int64_t frames, int T, const double* alpha, const double* beta,
                                double* grad_alpha, double* grad_beta, double* out_llr);

/* IEEE binary16 round-to-nearest-even conversion, for message storage */
uint16_t or_f32_to_f16(float x);
float or_f16_to_f32(uint16_t h);

/* ---- DVB-T2 outer BCH code (bch.cpp) ----
 * Codewords are [message (k) | parity (n-k)], bit i at polynomial degree n-1-i.
 * out5 = {n, k, t, field degree m, generator degree}.  Syndromes S_1..S_2t as
 * GF(2^m) elements (polynomial basis of the DVB-T2 primitive polynomial).
 * or_bch_decode writes the k message bits and, per frame, the number of bits
 * it flipped (the Chien-search roots). */
typedef struct or_bch or_bch;
or_bch* or_bch_dvbt2(int frame, int rate);
void or_bch_free(or_bch* b);
void or_bch_dims(const or_bch* b, int64_t* out5);
void or_bch_generator(const or_bch* b, uint8_t* coeffs /* degree + 1, x^d at [d] */);
void or_bch_encode(const or_bch* b, const uint8_t* msg, int64_t frames, uint8_t* cw);
void or_bch_syndromes(const or_bch* b, const uint8_t* cw, int64_t frames, uint16_t* synd);
int or_bch_berlekamp_massey(const or_bch* b, const uint16_t* synd, uint16_t* lambda /* 2t+1 */);
void or_bch_decode(const or_bch* b, const uint8_t* cw, int64_t frames, uint8_t* msg, int32_t* nflips);

#ifdef __cplusplus
}
#endif
