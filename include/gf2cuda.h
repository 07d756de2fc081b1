/* gf2cuda -- B200-native (sm_100a) batched LDPC encoder / decoder.
 *
 * C ABI of the library.  It replaces the belief-propagation path of the
 * erankavija/gf2 `gf2-coding` crate (all paths below are relative to
 * crates/gf2-coding/src/ of that project):
 *
 *   LdpcCode::{dvb_t2_normal, dvb_t2_short}     ldpc/core.rs:197-262
 *   LdpcCode::from_quasi_cyclic                 ldpc/core.rs:168-173
 *   LdpcCode::from_edges                        ldpc/core.rs:96-104
 *   LdpcCode::{n, m, k, rate}                   ldpc/core.rs:107-124
 *   LdpcCode::{syndrome, is_valid_codeword}     ldpc/core.rs:129-138
 *   LdpcDecoder::new                            ldpc/core.rs:653-697
 *   LdpcDecoder::decode_batch                   ldpc/core.rs:729-756
 *   IterativeSoftDecoder::decode_iterative      traits.rs:335, ldpc/core.rs:889-938
 *   LdpcEncoder::{encode, encode_batch}         ldpc/core.rs:1106-1132, traits.rs:206
 *   AwgnChannel / BpskModulator                 channel.rs:51-218
 *
 * Conventions
 *   - Every function returns an int status (GF2C_OK = 0); nothing aborts or
 *     panics.  gf2c_last_error() gives a message for the calling thread.
 *   - Bit vectors are packed in uint64_t words, bit i of a vector in word i/64
 *     at bit position i%64 (the gf2-core BitVec layout), unused tail bits 0.
 *     A batch of F vectors of length L occupies F * ceil(L/64) words.
 *   - LLRs are IEEE f32, positive = bit 0 more likely (llr.rs:73-75).
 *   - `mem` selects where the array arguments of one call live:
 *     GF2C_MEM_HOST (pageable or pinned host memory; the library stages the
 *     copies on `stream`) or GF2C_MEM_DEVICE (device pointers on the current
 *     device).  `stream` is a cudaStream_t (NULL = legacy default stream).
 *     gf2c_decode_batch splits host-memory batches of 64 MB of LLRs and more
 *     into chunks that alternate between `stream` and a second stream of the
 *     decoder (its own workspace), so that copies overlap decoding; pinned
 *     host memory lets the copies run asynchronously.  A host-memory call
 *     stages the whole batch in device memory (GF2C_ERR_NOMEM when it does
 *     not fit: split such a batch into several calls).
 *     Host-memory calls return after the results are in host memory;
 *     device-memory calls are asynchronous on `stream`.
 *   - Code handles are immutable after creation and may be shared by threads.
 *     A decoder handle owns device workspace and must not be used by two
 *     host threads at once.
 */
#ifndef GF2CUDA_H
#define GF2CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define GF2C_OK 0
#define GF2C_ERR_INVALID_ARG 1   /* bad pointer, size or enum value */
#define GF2C_ERR_CUDA 2          /* a CUDA runtime call failed */
#define GF2C_ERR_UNSUPPORTED 3   /* option not available for this code */
#define GF2C_ERR_NOMEM 4         /* device or host allocation failed */
#define GF2C_ERR_RANK 5          /* parity-check matrix is rank deficient */
#define GF2C_ERR_KERNEL 6        /* a kernel reported an internal error */

#define GF2C_MEM_HOST 0
#define GF2C_MEM_DEVICE 1

/* DvbParams::for_code (ldpc/dvb_t2/params.rs:56-85) */
#define GF2C_DVBT2_NORMAL 0      /* n = 64800 */
#define GF2C_DVBT2_SHORT 1       /* n = 16200 */
#define GF2C_RATE_1_2 0
#define GF2C_RATE_3_5 1
#define GF2C_RATE_2_3 2
#define GF2C_RATE_3_4 3
#define GF2C_RATE_4_5 4
#define GF2C_RATE_5_6 5

/* Check-node rule of a decoder. */
#define GF2C_ALGO_MINSUM 0  /* the reference's decoder: plain min-sum (core.rs:790-814),
                               results bit-identical to LdpcDecoder up to the sign of zero */
#define GF2C_ALGO_SPA 1     /* sum-product 2 atanh(prod tanh(x/2)) (core.rs:762-787,
                               llr.rs:210-215), FP32, |extrinsic product| <= 1 - 2^-23 */
#define GF2C_ALGO_NMS 2     /* normalised + offset min-sum (llr.rs:352-399) with one
                               (alpha, beta) per iteration and row group */
#define GF2C_ALGO_SPA_FAST 3 /* sum-product evaluated with the SFU (ex2/lg2/rcp approximations):
                               2 atanh(prod tanh) through products of 1 -/+ e^-|x|; judged by
                               FER and LLR deviation against the FP64 sum-product, not bit-exact */
#define GF2C_SCHED_FLOODING 0  /* decode_iterative's schedule (core.rs:909-924) */
#define GF2C_SCHED_LAYERED 1   /* row-group layered schedule (QC and DVB-T2 codes) */
#define GF2C_MSG_F32 0
#define GF2C_MSG_F16 1         /* messages stored as binary16, arithmetic in f32 */

typedef struct gf2c_code gf2c_code;
typedef struct gf2c_decoder gf2c_decoder;

typedef struct {
  int32_t algorithm;        /* GF2C_ALGO_* */
  int32_t schedule;         /* GF2C_SCHED_* */
  int32_t msg_dtype;        /* GF2C_MSG_* */
  int32_t early_stop;       /* 1 = stop a frame when its syndrome is zero (the reference
                               always does); 0 = run every frame for max_iter iterations */
  const float* nms_alpha;   /* GF2C_ALGO_NMS: host array [nms_iters][layers] */
  const float* nms_beta;    /* GF2C_ALGO_NMS: host array [nms_iters][layers] */
  int32_t nms_iters;        /* rows of the weight arrays; iteration t uses row min(t, nms_iters-1) */
  int32_t threads_per_block;/* 0 = library choice (autotuned when a tuning entry exists) */
  int32_t blocks_per_sm;    /* 0 = library choice */
} gf2c_decoder_opts;

/* Fills opts with the reference behaviour: min-sum, flooding, f32, early stop. */
void gf2c_decoder_opts_default(gf2c_decoder_opts* opts);

const char* gf2c_last_error(void);
const char* gf2c_version(void);

/* ---- codes ---- */
/* LdpcCode::dvb_t2_normal / dvb_t2_short (core.rs:197-262). */
int gf2c_code_create_dvbt2(int32_t frame_size, int32_t rate, gf2c_code** out);
/* LdpcCode::from_quasi_cyclic (core.rs:168-173, 578-605): base is mb x nb row-major,
 * -1 = zero block, otherwise a right shift in [0, z). */
int gf2c_code_create_qc(const int32_t* base, int32_t mb, int32_t nb, int32_t z, gf2c_code** out);
/* LdpcCode::from_edges (core.rs:96-104): pairs = count (check, variable) pairs;
 * repeated pairs cancel in pairs (GF(2) XOR, sparse.rs:166-203). */
int gf2c_code_create_edges(int64_t m, int64_t n, const int64_t* pairs, int64_t count,
                           gf2c_code** out);
int gf2c_code_destroy(gf2c_code* code);
/* n, m, k = max(n - m, 0), nonzeros of H, row groups usable by the layered schedule
 * (0 when the code has none).  Any output pointer may be NULL. */
int gf2c_code_dims(const gf2c_code* code, int64_t* n, int64_t* m, int64_t* k, int64_t* nnz,
                   int32_t* layers);
/* H as CSR in the reference's order (rows ascending, columns ascending): indptr
 * has m+1 entries, indices nnz. */
int gf2c_code_csr(const gf2c_code* code, int64_t* indptr, int64_t* indices);

/* LdpcCode::syndrome over a batch (core.rs:129-133): synd = H cw, packed m bits per
 * frame; weight (nullable) = popcount per frame (0 = valid codeword, core.rs:135-138). */
int gf2c_syndrome_batch(const gf2c_code* code, const uint64_t* cw_bits, int64_t frames,
                        uint64_t* synd_bits, int32_t* weight, int32_t mem, void* stream);

/* ---- encoder ---- */
/* LdpcEncoder::encode_batch (core.rs:1106-1132): systematic codewords.  The message
 * bits occupy the non-pivot columns of a right-to-left RREF of H in ascending order
 * and the parity bits the pivot columns (richardson_urbanke.rs:158-289); for DVB-T2
 * codes that is [message | parity] with the staircase accumulator. */
int gf2c_encode_batch(const gf2c_code* code, const uint64_t* msg_bits, int64_t frames,
                      uint64_t* cw_bits, int32_t mem, void* stream);

/* ---- channel ---- */
/* Seeded synthetic frames: uniform info bits (Philox4x32-10, key = seed, counter
 * = (block, frame0 + f, 1, 0)), systematic encoding, BPSK 0 -> +1 / 1 -> -1
 * (channel.rs:51-57), AWGN with variance sigma2[f] (Box-Muller, counter
 * (pair, frame0 + f, 2, 0)) and LLR = (f32)(2 y / sigma2[f]) (channel.rs:100-102).
 * Any of info_bits / cw_bits / llr may be NULL.  sigma2 has `frames` entries, in
 * the same memory space as the outputs. */
int gf2c_channel_awgn(const gf2c_code* code, uint64_t seed, uint64_t frame0, int64_t frames,
                      const double* sigma2, uint64_t* info_bits, uint64_t* cw_bits, float* llr,
                      int32_t mem, void* stream);
/* AwgnChannel::from_eb_n0_db (channel.rs:153-158): 1 / (2 rate 10^(ebn0/10)). */
double gf2c_sigma2_from_ebn0(double ebn0_db, double rate);

/* ---- decoder ---- */
/* LdpcDecoder::new (core.rs:653-697).  One decoder may serve several codes (a mixed
 * batch): gf2c_decoder_create_multi takes ncodes code handles, which must outlive it. */
int gf2c_decoder_create(const gf2c_code* code, const gf2c_decoder_opts* opts,
                        gf2c_decoder** out);
int gf2c_decoder_create_multi(const gf2c_code* const* codes, int32_t ncodes,
                              const gf2c_decoder_opts* opts, gf2c_decoder** out);
int gf2c_decoder_destroy(gf2c_decoder* dec);

/* LdpcDecoder::decode_batch (core.rs:729-756) over `frames` frames of the decoder's
 * (first) code, each decoded as IterativeSoftDecoder::decode_iterative (core.rs:889-938):
 *   llr         frames x n f32, frame-major
 *   max_iter    iteration budget (>= 0; 0 returns the all-zero word, like a fresh
 *               reference decoder)
 *   msg_bits    frames x ceil(k/64) words: hard decisions of the first k bits
 *               (core.rs:930-935)                                   (nullable)
 *   iterations  frames int32: DecoderResult::iterations            (nullable)
 *   converged   frames uint8: DecoderResult::converged             (nullable)
 *   syndrome_ok frames uint8: DecoderResult::syndrome_check_passed (nullable)
 *   beliefs     frames x n f32 final posterior LLRs                (nullable)
 * frames == 0 is a no-op.  Each frame's results depend on that frame only; a batch
 * of more frames than the decoder runs at once (up to 16384) is decoded hardest
 * frames first (two small kernels order the frames by their sum of |LLR|), so
 * the device-memory path launches 1 or 3 kernels (gf2c_decoder_last_launches). */
int gf2c_decode_batch(gf2c_decoder* dec, const float* llr, int64_t frames, int32_t max_iter,
                      uint64_t* msg_bits, int32_t* iterations, uint8_t* converged,
                      uint8_t* syndrome_ok, float* beliefs, int32_t mem, void* stream);

/* A decoder with a fallback, on the device -- no counterpart in the reference
 * (its decode_batch, core.rs:729-756, runs one decoder).  `primary` (e.g. the
 * learned min-sum decoder) decodes every frame with max_iter_primary
 * iterations; a small kernel lists the frames whose syndrome still fails, and
 * `fallback` (e.g. sum-product, layered schedule) decodes those frames again
 * from their LLRs with max_iter_fallback iterations, its results replacing
 * theirs (iterations = max_iter_primary + the fallback's count).  The list
 * and its length stay on the device: no host synchronisation between the
 * passes.  fallback_count (nullable, int64): frames re-decoded.
 * Both decoders must decode the same code.
 *   mem == GF2C_MEM_DEVICE: every pointer is device memory (fallback_count
 *     too); asynchronous on `stream`; 3 or 5 kernel launches.
 *   mem == GF2C_MEM_HOST: every pointer is host memory (pinned memory copies
 *     fastest); the batch is copied in, decoded and copied out, large batches
 *     in chunks on two streams so that copies overlap decoding (the fallback
 *     passes and output copies on a third stream of the primary decoder, one
 *     per group of chunks); returns when the results are in host memory. */
int gf2c_decode_batch_fallback(gf2c_decoder* primary, gf2c_decoder* fallback, const float* llr, int64_t frames,
                               int32_t max_iter_primary, int32_t max_iter_fallback, uint64_t* msg_bits,
                               int32_t* iterations, uint8_t* converged, uint8_t* syndrome_ok,
                               int64_t* fallback_count, int32_t mem, void* stream);

/* Mixed batch in one persistent launch: frame f uses code code_id[f] (index into the
 * codes given at creation), reads n[code] LLRs at llr + llr_offset[f], writes
 * ceil(k/64) words at msg_bits + msg_offset[f] (both in elements), and has its own
 * budget max_iter[f].  Per-frame outputs as in gf2c_decode_batch.  A decoder of
 * several codes first runs a small ordering kernel, so that the persistent launch
 * decodes the frames code by code (longest codes first); a frame's results do not
 * depend on the order.  With mem ==
 * GF2C_MEM_DEVICE and use_graph = 1 the launch sequence is captured once per
 * (frames, pointers) shape into a CUDA graph and replayed.  With mem ==
 * GF2C_MEM_HOST a large batch of several codes goes in chunks of frames in
 * memory order (the frame order of each chunk made on the host), whose copies
 * overlap the decoding of earlier chunks; use_graph is ignored. */
int gf2c_decode_mixed(gf2c_decoder* dec, const float* llr, const int64_t* llr_offset,
                      const int32_t* code_id, const int32_t* max_iter, int64_t frames,
                      uint64_t* msg_bits, const int64_t* msg_offset, int32_t* iterations,
                      uint8_t* converged, uint8_t* syndrome_ok, int32_t use_graph,
                      int32_t mem, void* stream);

/* Decoding without any device allocation -- no counterpart in the reference (its
 * decoder is host code).  For callers that cannot call cudaMalloc: work being
 * captured into a CUDA graph, processes whose device memory belongs to a pool or
 * budget the library must not grow, real-time paths that forbid the allocator.
 * Decodes `frames` frames of `code` exactly like gf2c_decode_batch with the
 * default options (reference min-sum, flooding, f32, early stop); all pointers
 * are device memory, asynchronous on `stream`.  Its scratch (the code's tables,
 * the frame counter and the per-CTA workspace) is a 64 MiB static device array
 * that every GPU loading the library holds until exit; codes whose tables plus
 * one frame's workspace exceed it are rejected with GF2C_ERR_UNSUPPORTED.  The
 * first call on a device looks up the array's device address and should come
 * before any stream capture.  All calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller. */
int gf2c_decode_batch_noalloc(const gf2c_code* code, const float* llr, int64_t frames, int32_t max_iter,
                              uint64_t* msg_bits, int32_t* iterations, uint8_t* converged,
                              uint8_t* syndrome_ok, void* stream);

/* FP64 sum-product judge -- no counterpart in the reference, whose sum-product
 * (check_node_update_spa + Llr::boxplus_n, core.rs:762-787, llr.rs:210-215) is
 * FP32 and unused.  The precision reference that the FP32 / FP16 decoders are
 * stated against: 2 atanh(prod tanh(x/2)) with FP64 tanh / atanh, FP64
 * messages and posteriors, |extrinsic product| <= 1 - 2^-50, flooding
 * (core.rs:909-924) or layered schedule, syndrome early stop after every
 * iteration.  Outputs as in gf2c_decode_batch except beliefs, which are FP64
 * (frames x n, natural order).  Device memory only, asynchronous on `stream`;
 * DVB-T2 and QC codes only (GF2C_ERR_UNSUPPORTED otherwise).  It keeps its own
 * workspace per host thread (allocated on first use). */
int gf2c_judge_spa64(const gf2c_code* code, int32_t schedule, const float* llr, int64_t frames, int32_t max_iter,
                     uint64_t* msg_bits, int32_t* iterations, uint8_t* converged, uint8_t* syndrome_ok,
                     double* beliefs, void* stream);

/* Number of kernel launches issued by the last decode call of `dec`. */
int gf2c_decoder_last_launches(const gf2c_decoder* dec, int32_t* launches);

/* ---- learned normalised / offset min-sum (no reference counterpart: the
 * reference only offers the fixed-weight rules Llr::boxplus_normalized_minsum_n
 * and boxplus_offset_minsum_n, llr.rs:352-399) ----
 * c2v = sign * alpha[t][l] * max(min|v2c| - beta[t][l], 0) for unrolled flooding
 * iteration t < iterations and row group l < layers (layers = 1 for codes
 * without row groups).  The trained weights decode with GF2C_ALGO_NMS. */
typedef struct gf2c_nms_trainer gf2c_nms_trainer;
int gf2c_nms_trainer_create(const gf2c_code* code, int32_t iterations, int64_t max_frames,
                            gf2c_nms_trainer** out);
int gf2c_nms_trainer_destroy(gf2c_nms_trainer* tr);
int gf2c_nms_trainer_layers(const gf2c_nms_trainer* tr, int32_t* layers);
/* Schedule of the unrolled decoder the trainer differentiates: GF2C_SCHED_FLOODING
 * (the default, decode_iterative's schedule) or GF2C_SCHED_LAYERED (row groups
 * in order, the posterior updated after each; weights per iteration and row
 * group; the forward equals the layered GF2C_ALGO_NMS decoder with FP32
 * messages bit for bit).  GF2C_ERR_UNSUPPORTED for codes without row groups. */
int gf2c_nms_trainer_set_schedule(gf2c_nms_trainer* tr, int32_t schedule);
/* Forward (iterations steps of the trainer's schedule, no early stop) and backward over a device
 * batch: llr [frames][n] f32, cw_bits [frames][ceil(n/64)] transmitted codewords,
 * alpha / beta [iterations][layers].  Writes the mean binary cross-entropy of
 * sigmoid(final LLR) against the codeword bits to *loss and its gradients to
 * grad_alpha / grad_beta (overwritten); soft_out [frames][n] (nullable) receives
 * the final LLRs.  All pointers are device memory; asynchronous on `stream`. */
int gf2c_nms_loss_grad(gf2c_nms_trainer* tr, const float* llr, const uint64_t* cw_bits, int64_t frames,
                       const float* alpha, const float* beta, float* grad_alpha, float* grad_beta,
                       float* loss, float* soft_out, void* stream);
/* Frame / bit error counters of a Monte Carlo point (device memory): compares
 * two packed batches of `words` words per frame; totals[0] += frames with an
 * error, totals[1] += bit errors; bit_errors (nullable) receives the per-frame
 * counts.  The reference only has an uncoded BER runner (SimulationRunner,
 * simulation.rs:140-193); its coded FER loop lives in examples/ldpc_awgn.rs:121-175. */
int gf2c_count_errors(const uint64_t* ref_bits, const uint64_t* test_bits, int64_t frames, int32_t words,
                      int32_t* bit_errors, uint64_t* totals, void* stream);
/* One Adam step (bias-corrected, step >= 1) on device arrays of `count` floats;
 * parameters are clamped to [lo, hi]. */
int gf2c_adam_step(float* params, const float* grads, float* m, float* v, int64_t count, float lr,
                   float beta1, float beta2, float eps, int32_t step, float lo, float hi, void* stream);

/* ---- DVB-T2 outer BCH code (the step after LDPC decoding) ----
 * A BCH code handle holds one of the 12 DVB-T2 outer codes: n = k_ldpc of the
 * matching LDPC code, k = Kbch, t = 12 (10 for normal 2/3 and 5/6), GF(2^14)
 * for short and GF(2^16) for normal frames.  Codewords are [message | parity]
 * with bit i the coefficient of degree n-1-i (the reference's convention), in
 * the packed BitVec layout. */
typedef struct gf2c_bch gf2c_bch;
/* BchCode::dvb_t2 (crates/gf2-coding/src/bch/dvb_t2/mod.rs:62-78,
 * params.rs:56-85, generators.rs:14-62); frame_size / rate as for the LDPC codes. */
int gf2c_bch_create_dvbt2(int32_t frame_size, int32_t rate, gf2c_bch** out);
int gf2c_bch_destroy(gf2c_bch* bch);
/* BchCode::{n, k, t} (bch/core.rs:235-247) and the field degree m. */
int gf2c_bch_dims(const gf2c_bch* bch, int64_t* n, int64_t* k, int32_t* t, int32_t* field_m);
/* BchCode::generator (bch/core.rs:255): n-k+1 binary coefficients, x^d at [d]. */
int gf2c_bch_generator(const gf2c_bch* bch, uint8_t* coeffs);
/* BchEncoder::{encode, encode_batch} (bch/core.rs:396-480): frames x ceil(k/64)
 * message words in, frames x ceil(n/64) codeword words out. */
int gf2c_bch_encode_batch(gf2c_bch* bch, const uint64_t* msg_bits, int64_t frames, uint64_t* cw_bits,
                          int32_t mem, void* stream);
/* BchDecoder::{decode, decode_batch} (bch/core.rs:542-665): frames x ceil(n/64)
 * codeword words in, frames x ceil(k/64) message words out, bit-identical to
 * the reference (syndromes, Berlekamp-Massey, Chien search, no check of the
 * root count).  corrected (nullable): bits flipped per frame (the number of
 * roots found); syndromes (nullable): frames x 2t elements S_1..S_2t of
 * BchDecoder::compute_syndromes (bch/core.rs:562-617). */
int gf2c_bch_decode_batch(gf2c_bch* bch, const uint64_t* cw_bits, int64_t frames, uint64_t* msg_bits,
                          int32_t* corrected, uint16_t* syndromes, int32_t mem, void* stream);

/* ------------------------------------------------------------------------
 * gf2 file formats and the LDPC encoder cache (host side).
 * Binary "GF2DATA" files (crates/gf2-core/src/io/format.rs:1-16,
 * header.rs:6-82): 32-byte header, compact JSON metadata, little-endian payload;
 * type tags 1 BitVec (io/bitvec.rs), 2 BitMatrix (io/matrix.rs),
 * 3 SpBitMatrix (COO pairs, io/sparse.rs), 4 SpBitMatrixDual (CSR + CSC).
 * format: 0 binary, 1 text, 2 hex (io/formats.rs); -1 on input = detect as
 * SerializationFormat::detect does.  Bits are packed BitVec words; a
 * BitMatrix is rows x ceil(cols/64) words, row-major.
 * ------------------------------------------------------------------------ */
/* SerializationFormat::detect + the header / metadata: type tag (1..4), format,
 * dims3 = {len_bits} (BitVec), {rows, cols} (BitMatrix), {rows, cols, nnz}. */
int gf2c_io_probe(const char* path, int32_t* type_tag, int32_t* format, int64_t* dims3);
/* BitVec::save_to_file_with_format / load_from_file (auto-detect) (io/bitvec.rs). */
int gf2c_io_write_bitvec(const char* path, const uint64_t* words, int64_t len_bits, int32_t format);
int gf2c_io_read_bitvec(const char* path, uint64_t* words, int64_t cap_words, int64_t* len_bits);
/* BitMatrix::save_to_file_with_format / load_from_file_with_format (io/matrix.rs). */
int gf2c_io_write_bitmatrix(const char* path, const uint64_t* words, int64_t rows, int64_t cols, int32_t format);
int gf2c_io_read_bitmatrix(const char* path, int32_t format, uint64_t* words, int64_t cap_words, int64_t* rows,
                           int64_t* cols);
/* SpBitMatrix (type 3) / SpBitMatrixDual (type 4) save (binary or text) and
 * load (io/sparse.rs): CSR with ascending columns; loading a COO file sorts
 * and removes repeated edges (SpBitMatrix::from_coo_deduplicated).  Pass
 * row_ptr / col_idx NULL to query rows / cols / nnz first. */
int gf2c_io_write_sparse(const char* path, int32_t type_tag, int64_t rows, int64_t cols, const int64_t* row_ptr,
                         const int64_t* col_idx, int32_t format);
int gf2c_io_read_sparse(const char* path, int32_t format, int64_t* rows, int64_t* cols, int64_t* nnz,
                        int64_t* row_ptr, int64_t* col_idx, int64_t cap_nnz);
/* LdpcCode from / to a parity-check matrix file (type 3 or 4). */
int gf2c_code_create_file(const char* path, gf2c_code** out);
int gf2c_io_write_code(const char* path, const gf2c_code* code, int32_t type_tag, int32_t format);
/* SipHash-1-3 (the algorithm of Rust's DefaultHasher; zero keys there). */
int gf2c_siphash13(const void* data, int64_t len, uint64_t k0, uint64_t k1, uint64_t* out);
/* CacheKey::from_params (ldpc/encoding/cache.rs:84-90, 461-487): the
 * structural hash of H that names the cache file "n{n}_k{k}_h{hash:x}.gf2". */
int gf2c_code_cache_hash(const gf2c_code* code, uint64_t* hash);
/* RuEncodingMatrices::parity_part (richardson_urbanke.rs:372): P, k x
 * ceil((n-k)/64) words, row i = the parity bits of message bit i, for the
 * systematic form with the message in columns [0, k) (what the cache files
 * hold); GF2C_ERR_UNSUPPORTED for a code whose systematic columns differ. */
int gf2c_code_parity_part(const gf2c_code* code, uint64_t* words);
/* Encoding with a dense parity part (RuEncodingMatrices::encode /
 * encode_batch, richardson_urbanke.rs:263-330, as reconstructed by
 * EncodingCache::from_directory, cache.rs:347-433): codeword = [message |
 * P^T message].  P is copied at creation (host words). */
typedef struct gf2c_dense_encoder gf2c_dense_encoder;
int gf2c_dense_encoder_create(const uint64_t* parity_words, int64_t k, int64_t n, gf2c_dense_encoder** out);
int gf2c_dense_encoder_destroy(gf2c_dense_encoder* enc);
int gf2c_dense_encode_batch(gf2c_dense_encoder* enc, const uint64_t* msg_bits, int64_t frames, uint64_t* cw_bits,
                            int32_t mem, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GF2CUDA_H */
