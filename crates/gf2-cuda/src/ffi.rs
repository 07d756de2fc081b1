//! Raw declarations of the gf2cuda C ABI (`include/gf2cuda.h`), one `extern "C"`
//! item per C function with the same argument order and types.  Every function
//! returns a status code (`GF2C_OK` = 0) unless its C declaration says otherwise;
//! `gf2c_last_error` gives the calling thread's message.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_void};

pub const GF2C_OK: i32 = 0;
pub const GF2C_ERR_INVALID_ARG: i32 = 1;
pub const GF2C_ERR_CUDA: i32 = 2;
pub const GF2C_ERR_UNSUPPORTED: i32 = 3;
pub const GF2C_ERR_NOMEM: i32 = 4;
pub const GF2C_ERR_RANK: i32 = 5;
pub const GF2C_ERR_KERNEL: i32 = 6;

pub const GF2C_MEM_HOST: i32 = 0;
pub const GF2C_MEM_DEVICE: i32 = 1;

pub const GF2C_DVBT2_NORMAL: i32 = 0;
pub const GF2C_DVBT2_SHORT: i32 = 1;

pub const GF2C_ALGO_MINSUM: i32 = 0;
pub const GF2C_ALGO_SPA: i32 = 1;
pub const GF2C_ALGO_NMS: i32 = 2;
pub const GF2C_ALGO_SPA_FAST: i32 = 3;
pub const GF2C_SCHED_FLOODING: i32 = 0;
pub const GF2C_SCHED_LAYERED: i32 = 1;
pub const GF2C_MSG_F32: i32 = 0;
pub const GF2C_MSG_F16: i32 = 1;

#[repr(C)]
pub struct gf2c_code {
    _p: [u8; 0],
}
#[repr(C)]
pub struct gf2c_decoder {
    _p: [u8; 0],
}
#[repr(C)]
pub struct gf2c_nms_trainer {
    _p: [u8; 0],
}
#[repr(C)]
pub struct gf2c_bch {
    _p: [u8; 0],
}
#[repr(C)]
pub struct gf2c_dense_encoder {
    _p: [u8; 0],
}

/// `gf2c_decoder_opts`: field order and types as in the C struct.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct gf2c_decoder_opts {
    pub algorithm: i32,
    pub schedule: i32,
    pub msg_dtype: i32,
    pub early_stop: i32,
    pub nms_alpha: *const f32,
    pub nms_beta: *const f32,
    pub nms_iters: i32,
    pub threads_per_block: i32,
    pub blocks_per_sm: i32,
}

extern "C" {
    // ---- library ----
    pub fn gf2c_decoder_opts_default(opts: *mut gf2c_decoder_opts);
    pub fn gf2c_last_error() -> *const c_char;
    pub fn gf2c_version() -> *const c_char;

    // ---- codes ----
    pub fn gf2c_code_create_dvbt2(frame_size: i32, rate: i32, out: *mut *mut gf2c_code) -> i32;
    pub fn gf2c_code_create_qc(base: *const i32, mb: i32, nb: i32, z: i32, out: *mut *mut gf2c_code) -> i32;
    pub fn gf2c_code_create_edges(m: i64, n: i64, pairs: *const i64, count: i64, out: *mut *mut gf2c_code) -> i32;
    pub fn gf2c_code_destroy(code: *mut gf2c_code) -> i32;
    pub fn gf2c_code_dims(code: *const gf2c_code, n: *mut i64, m: *mut i64, k: *mut i64, nnz: *mut i64,
                          layers: *mut i32) -> i32;
    pub fn gf2c_code_csr(code: *const gf2c_code, indptr: *mut i64, indices: *mut i64) -> i32;
    pub fn gf2c_syndrome_batch(code: *const gf2c_code, cw_bits: *const u64, frames: i64, synd_bits: *mut u64,
                               weight: *mut i32, mem: i32, stream: *mut c_void) -> i32;

    // ---- encoder and channel ----
    pub fn gf2c_encode_batch(code: *const gf2c_code, msg_bits: *const u64, frames: i64, cw_bits: *mut u64,
                             mem: i32, stream: *mut c_void) -> i32;
    pub fn gf2c_channel_awgn(code: *const gf2c_code, seed: u64, frame0: u64, frames: i64, sigma2: *const f64,
                             info_bits: *mut u64, cw_bits: *mut u64, llr: *mut f32, mem: i32,
                             stream: *mut c_void) -> i32;
    pub fn gf2c_sigma2_from_ebn0(ebn0_db: f64, rate: f64) -> f64;

    // ---- decoder ----
    pub fn gf2c_decoder_create(code: *const gf2c_code, opts: *const gf2c_decoder_opts,
                               out: *mut *mut gf2c_decoder) -> i32;
    pub fn gf2c_decoder_create_multi(codes: *const *const gf2c_code, ncodes: i32, opts: *const gf2c_decoder_opts,
                                     out: *mut *mut gf2c_decoder) -> i32;
    pub fn gf2c_decoder_destroy(dec: *mut gf2c_decoder) -> i32;
    pub fn gf2c_decode_batch(dec: *mut gf2c_decoder, llr: *const f32, frames: i64, max_iter: i32,
                             msg_bits: *mut u64, iterations: *mut i32, converged: *mut u8, syndrome_ok: *mut u8,
                             beliefs: *mut f32, mem: i32, stream: *mut c_void) -> i32;
    pub fn gf2c_decode_batch_fallback(primary: *mut gf2c_decoder, fallback: *mut gf2c_decoder, llr: *const f32,
                                      frames: i64, max_iter_primary: i32, max_iter_fallback: i32,
                                      msg_bits: *mut u64, iterations: *mut i32, converged: *mut u8,
                                      syndrome_ok: *mut u8, fallback_count: *mut i64, mem: i32,
                                      stream: *mut c_void) -> i32;
    pub fn gf2c_decode_mixed(dec: *mut gf2c_decoder, llr: *const f32, llr_offset: *const i64, code_id: *const i32,
                             max_iter: *const i32, frames: i64, msg_bits: *mut u64, msg_offset: *const i64,
                             iterations: *mut i32, converged: *mut u8, syndrome_ok: *mut u8, use_graph: i32,
                             mem: i32, stream: *mut c_void) -> i32;
    pub fn gf2c_decode_batch_noalloc(code: *const gf2c_code, llr: *const f32, frames: i64, max_iter: i32,
                                     msg_bits: *mut u64, iterations: *mut i32, converged: *mut u8,
                                     syndrome_ok: *mut u8, stream: *mut c_void) -> i32;
    pub fn gf2c_judge_spa64(code: *const gf2c_code, schedule: i32, llr: *const f32, frames: i64, max_iter: i32,
                            msg_bits: *mut u64, iterations: *mut i32, converged: *mut u8, syndrome_ok: *mut u8,
                            beliefs: *mut f64, stream: *mut c_void) -> i32;
    pub fn gf2c_decoder_last_launches(dec: *const gf2c_decoder, launches: *mut i32) -> i32;

    // ---- learned normalised / offset min-sum ----
    pub fn gf2c_nms_trainer_create(code: *const gf2c_code, iterations: i32, max_frames: i64,
                                   out: *mut *mut gf2c_nms_trainer) -> i32;
    pub fn gf2c_nms_trainer_destroy(tr: *mut gf2c_nms_trainer) -> i32;
    pub fn gf2c_nms_trainer_set_schedule(tr: *mut gf2c_nms_trainer, schedule: i32) -> i32;
    pub fn gf2c_nms_trainer_layers(tr: *const gf2c_nms_trainer, layers: *mut i32) -> i32;
    pub fn gf2c_nms_loss_grad(tr: *mut gf2c_nms_trainer, llr: *const f32, cw_bits: *const u64, frames: i64,
                              alpha: *const f32, beta: *const f32, grad_alpha: *mut f32, grad_beta: *mut f32,
                              loss: *mut f32, soft_out: *mut f32, stream: *mut c_void) -> i32;
    pub fn gf2c_count_errors(ref_bits: *const u64, test_bits: *const u64, frames: i64, words: i32,
                             bit_errors: *mut i32, totals: *mut u64, stream: *mut c_void) -> i32;
    pub fn gf2c_adam_step(params: *mut f32, grads: *const f32, m: *mut f32, v: *mut f32, count: i64, lr: f32,
                          beta1: f32, beta2: f32, eps: f32, step: i32, lo: f32, hi: f32,
                          stream: *mut c_void) -> i32;

    // ---- DVB-T2 outer BCH code ----
    pub fn gf2c_bch_create_dvbt2(frame_size: i32, rate: i32, out: *mut *mut gf2c_bch) -> i32;
    pub fn gf2c_bch_destroy(bch: *mut gf2c_bch) -> i32;
    pub fn gf2c_bch_dims(bch: *const gf2c_bch, n: *mut i64, k: *mut i64, t: *mut i32, field_m: *mut i32) -> i32;
    pub fn gf2c_bch_generator(bch: *const gf2c_bch, coeffs: *mut u8) -> i32;
    pub fn gf2c_bch_encode_batch(bch: *mut gf2c_bch, msg_bits: *const u64, frames: i64, cw_bits: *mut u64,
                                 mem: i32, stream: *mut c_void) -> i32;
    pub fn gf2c_bch_decode_batch(bch: *mut gf2c_bch, cw_bits: *const u64, frames: i64, msg_bits: *mut u64,
                                 corrected: *mut i32, syndromes: *mut u16, mem: i32, stream: *mut c_void) -> i32;

    // ---- gf2 files and the encoder cache ----
    pub fn gf2c_io_probe(path: *const c_char, type_tag: *mut i32, format: *mut i32, dims3: *mut i64) -> i32;
    pub fn gf2c_io_write_bitvec(path: *const c_char, words: *const u64, len_bits: i64, format: i32) -> i32;
    pub fn gf2c_io_read_bitvec(path: *const c_char, words: *mut u64, cap_words: i64, len_bits: *mut i64) -> i32;
    pub fn gf2c_io_write_bitmatrix(path: *const c_char, words: *const u64, rows: i64, cols: i64,
                                   format: i32) -> i32;
    pub fn gf2c_io_read_bitmatrix(path: *const c_char, format: i32, words: *mut u64, cap_words: i64,
                                  rows: *mut i64, cols: *mut i64) -> i32;
    pub fn gf2c_io_write_sparse(path: *const c_char, type_tag: i32, rows: i64, cols: i64, row_ptr: *const i64,
                                col_idx: *const i64, format: i32) -> i32;
    pub fn gf2c_io_read_sparse(path: *const c_char, format: i32, rows: *mut i64, cols: *mut i64, nnz: *mut i64,
                               row_ptr: *mut i64, col_idx: *mut i64, cap_nnz: i64) -> i32;
    pub fn gf2c_code_create_file(path: *const c_char, out: *mut *mut gf2c_code) -> i32;
    pub fn gf2c_io_write_code(path: *const c_char, code: *const gf2c_code, type_tag: i32, format: i32) -> i32;
    pub fn gf2c_siphash13(data: *const c_void, len: i64, k0: u64, k1: u64, out: *mut u64) -> i32;
    pub fn gf2c_code_cache_hash(code: *const gf2c_code, hash: *mut u64) -> i32;
    pub fn gf2c_code_parity_part(code: *const gf2c_code, words: *mut u64) -> i32;
    pub fn gf2c_dense_encoder_create(parity_words: *const u64, k: i64, n: i64,
                                     out: *mut *mut gf2c_dense_encoder) -> i32;
    pub fn gf2c_dense_encoder_destroy(enc: *mut gf2c_dense_encoder) -> i32;
    pub fn gf2c_dense_encode_batch(enc: *mut gf2c_dense_encoder, msg_bits: *const u64, frames: i64,
                                   cw_bits: *mut u64, mem: i32, stream: *mut c_void) -> i32;
}
