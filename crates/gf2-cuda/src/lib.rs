//! gf2-cuda: the gf2-coding LDPC belief-propagation path on an NVIDIA B200,
//! behind the reference crate's own decoder and encoder traits.
//!
//! What each type replaces (paths under crates/gf2-coding/src/):
//!   `CudaLdpcCode`            `LdpcCode::{dvb_t2_normal, dvb_t2_short, from_edges,
//!                              from_quasi_cyclic, n, m, k, rate, syndrome,
//!                              is_valid_codeword}`                ldpc/core.rs:96-262
//!   `CudaLdpcDecoder`         `LdpcDecoder::new` + `IterativeSoftDecoder` +
//!                             `SoftDecoder`                       ldpc/core.rs:653-938,
//!                                                                  traits.rs:242-347
//!   `decode_batch`            `LdpcDecoder::decode_batch`          ldpc/core.rs:729-756
//!   `CudaLdpcEncoder`         `LdpcEncoder::{encode, encode_batch}` ldpc/core.rs:1106-1132
//!
//! Every call goes through the C ABI in `ffi`; bad input panics, as the
//! reference's `assert_eq!` checks do.  The default decoder options are the
//! reference's: plain min-sum, flooding schedule, FP32 messages, syndrome
//! early stop; its results are bit-identical to `LdpcDecoder`'s (a message that
//! is exactly zero may carry the other sign of zero).
#![cfg(feature = "cuda")]

pub mod ffi;

use std::ffi::CStr;
use std::ptr;

use gf2_coding::llr::Llr;
use gf2_coding::traits::{BlockEncoder, DecoderResult, IterativeSoftDecoder, SoftDecoder};
use gf2_core::BitVec;

fn check(rc: i32) {
    if rc != ffi::GF2C_OK {
        let msg = unsafe { CStr::from_ptr(ffi::gf2c_last_error()) };
        panic!("gf2cuda error {rc}: {}", msg.to_string_lossy());
    }
}

fn words(bits: usize) -> usize {
    (bits + 63) / 64
}

/// Code rate index of the DVB-T2 constructors (the order of `CodeRate`).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum DvbRate {
    R1_2 = 0,
    R3_5 = 1,
    R2_3 = 2,
    R3_4 = 3,
    R4_5 = 4,
    R5_6 = 5,
}

/// An LDPC code uploaded to the library (immutable, shareable by threads).
pub struct CudaLdpcCode {
    raw: *mut ffi::gf2c_code,
    n: usize,
    m: usize,
    k: usize,
}

unsafe impl Send for CudaLdpcCode {}
unsafe impl Sync for CudaLdpcCode {}

impl CudaLdpcCode {
    /// `LdpcCode::dvb_t2_normal` (n = 64800).
    pub fn dvb_t2_normal(rate: DvbRate) -> Self {
        Self::dvb_t2(ffi::GF2C_DVBT2_NORMAL, rate)
    }

    /// `LdpcCode::dvb_t2_short` (n = 16200).
    pub fn dvb_t2_short(rate: DvbRate) -> Self {
        Self::dvb_t2(ffi::GF2C_DVBT2_SHORT, rate)
    }

    fn dvb_t2(frame: i32, rate: DvbRate) -> Self {
        let mut raw = ptr::null_mut();
        check(unsafe { ffi::gf2c_code_create_dvbt2(frame, rate as i32, &mut raw) });
        Self::wrap(raw)
    }

    /// `LdpcCode::from_edges`: (check, variable) pairs; a repeated pair cancels (GF(2)).
    pub fn from_edges(m: usize, n: usize, edges: &[(usize, usize)]) -> Self {
        let flat: Vec<i64> = edges.iter().flat_map(|&(r, c)| [r as i64, c as i64]).collect();
        let mut raw = ptr::null_mut();
        check(unsafe { ffi::gf2c_code_create_edges(m as i64, n as i64, flat.as_ptr(), edges.len() as i64, &mut raw) });
        Self::wrap(raw)
    }

    /// `LdpcCode::from_quasi_cyclic`: base matrix rows of circulant shifts, -1 = zero block.
    pub fn from_quasi_cyclic(base: &[Vec<i32>], z: usize) -> Self {
        let mb = base.len();
        let nb = base.first().map_or(0, |r| r.len());
        let flat: Vec<i32> = base
            .iter()
            .flat_map(|r| {
                assert_eq!(r.len(), nb, "base matrix rows must have equal length");
                r.iter().copied()
            })
            .collect();
        let mut raw = ptr::null_mut();
        check(unsafe { ffi::gf2c_code_create_qc(flat.as_ptr(), mb as i32, nb as i32, z as i32, &mut raw) });
        Self::wrap(raw)
    }

    fn wrap(raw: *mut ffi::gf2c_code) -> Self {
        let (mut n, mut m, mut k, mut nnz, mut layers) = (0i64, 0i64, 0i64, 0i64, 0i32);
        check(unsafe { ffi::gf2c_code_dims(raw, &mut n, &mut m, &mut k, &mut nnz, &mut layers) });
        Self { raw, n: n as usize, m: m as usize, k: k as usize }
    }

    pub fn n(&self) -> usize {
        self.n
    }
    pub fn m(&self) -> usize {
        self.m
    }
    pub fn k(&self) -> usize {
        self.k
    }
    /// `LdpcCode::rate` = k / n.
    pub fn rate(&self) -> f64 {
        self.k as f64 / self.n as f64
    }

    /// `LdpcCode::syndrome`: H c over GF(2), m bits.
    pub fn syndrome(&self, codeword: &BitVec) -> BitVec {
        assert_eq!(codeword.len(), self.n, "codeword length must equal n");
        let mut synd = vec![0u64; words(self.m)];
        let mut weight = 0i32;
        check(unsafe {
            ffi::gf2c_syndrome_batch(self.raw, codeword.words().as_ptr(), 1, synd.as_mut_ptr(), &mut weight,
                                     ffi::GF2C_MEM_HOST, ptr::null_mut())
        });
        BitVec::from_words(synd, self.m)
    }

    /// `LdpcCode::is_valid_codeword`: the syndrome is zero.
    pub fn is_valid_codeword(&self, codeword: &BitVec) -> bool {
        self.syndrome(codeword).count_ones() == 0
    }
}

impl Drop for CudaLdpcCode {
    fn drop(&mut self) {
        unsafe {
            ffi::gf2c_code_destroy(self.raw);
        }
    }
}

/// Decoder options beyond the reference's (min-sum, flooding, FP32): the
/// library's sum-product, layered schedule, FP16 message storage and learned
/// normalised / offset min-sum weights (alpha, beta of [iterations][row groups]).
pub struct DecoderOptions {
    pub algorithm: i32,
    pub schedule: i32,
    pub msg_dtype: i32,
    pub early_stop: bool,
    pub nms_weights: Option<(Vec<f32>, Vec<f32>, usize)>,
}

impl Default for DecoderOptions {
    fn default() -> Self {
        Self {
            algorithm: ffi::GF2C_ALGO_MINSUM,
            schedule: ffi::GF2C_SCHED_FLOODING,
            msg_dtype: ffi::GF2C_MSG_F32,
            early_stop: true,
            nms_weights: None,
        }
    }
}

/// `LdpcDecoder` on the GPU.  Owns device workspace; `&mut self` keeps it to
/// one thread at a time, as the reference's decoder does.
pub struct CudaLdpcDecoder {
    code: CudaLdpcCode,
    raw: *mut ffi::gf2c_decoder,
    last_iterations: usize,
}

unsafe impl Send for CudaLdpcDecoder {}

impl CudaLdpcDecoder {
    /// `LdpcDecoder::new(code)`: the reference's decoder (bit-identical results).
    pub fn new(code: CudaLdpcCode) -> Self {
        Self::with_options(code, DecoderOptions::default())
    }

    pub fn with_options(code: CudaLdpcCode, o: DecoderOptions) -> Self {
        let mut opts = std::mem::MaybeUninit::<ffi::gf2c_decoder_opts>::uninit();
        let mut raw = ptr::null_mut();
        unsafe {
            ffi::gf2c_decoder_opts_default(opts.as_mut_ptr());
            let mut opts = opts.assume_init();
            opts.algorithm = o.algorithm;
            opts.schedule = o.schedule;
            opts.msg_dtype = o.msg_dtype;
            opts.early_stop = o.early_stop as i32;
            if let Some((a, b, iters)) = &o.nms_weights {
                assert_eq!(a.len(), b.len(), "alpha and beta must have the same shape");
                opts.nms_alpha = a.as_ptr();
                opts.nms_beta = b.as_ptr();
                opts.nms_iters = *iters as i32;
            }
            // the weights are copied to the device inside gf2c_decoder_create
            check(ffi::gf2c_decoder_create(code.raw, &opts, &mut raw));
        }
        Self { code, raw, last_iterations: 0 }
    }

    pub fn code(&self) -> &CudaLdpcCode {
        &self.code
    }

    /// `LdpcDecoder::decode_batch`: all frames in one call (one persistent launch).
    pub fn decode_batch(&mut self, llr_blocks: &[Vec<Llr>], max_iterations: usize) -> Vec<DecoderResult> {
        let (n, k, f) = (self.code.n, self.code.k, llr_blocks.len());
        if f == 0 {
            return Vec::new();
        }
        // Llr is a plain struct Llr(f32) without repr(transparent): copy the values
        let mut llr = Vec::with_capacity(f * n);
        for b in llr_blocks {
            assert_eq!(b.len(), n, "LLR length must equal n");
            llr.extend(b.iter().map(|l| l.value()));
        }
        let wk = words(k);
        let mut bits = vec![0u64; f * wk];
        let mut iters = vec![0i32; f];
        let (mut conv, mut synd) = (vec![0u8; f], vec![0u8; f]);
        check(unsafe {
            ffi::gf2c_decode_batch(self.raw, llr.as_ptr(), f as i64, max_iterations as i32, bits.as_mut_ptr(),
                                   iters.as_mut_ptr(), conv.as_mut_ptr(), synd.as_mut_ptr(), ptr::null_mut(),
                                   ffi::GF2C_MEM_HOST, ptr::null_mut())
        });
        (0..f)
            .map(|i| {
                DecoderResult::new(BitVec::from_words(bits[i * wk..(i + 1) * wk].to_vec(), k), iters[i] as usize,
                                   conv[i] != 0, synd[i] != 0)
            })
            .collect()
    }

    /// `decode_batch` with a fallback decoder (no counterpart in the
    /// reference): this decoder on every frame, then `fallback` (a layered
    /// decoder of the same code, e.g. sum-product) on the frames whose
    /// syndrome still fails, the list kept on the device.  Returns the results
    /// and the number of frames re-decoded.
    pub fn decode_batch_with_fallback(&mut self, fallback: &mut CudaLdpcDecoder, llr_blocks: &[Vec<Llr>],
                                      max_iterations: usize, fallback_iterations: usize)
                                      -> (Vec<DecoderResult>, usize) {
        let (n, k, f) = (self.code.n, self.code.k, llr_blocks.len());
        if f == 0 {
            return (Vec::new(), 0);
        }
        let mut llr = Vec::with_capacity(f * n);
        for b in llr_blocks {
            assert_eq!(b.len(), n, "LLR length must equal n");
            llr.extend(b.iter().map(|l| l.value()));
        }
        let wk = words(k);
        let mut bits = vec![0u64; f * wk];
        let mut iters = vec![0i32; f];
        let (mut conv, mut synd) = (vec![0u8; f], vec![0u8; f]);
        let mut redecoded = 0i64;
        check(unsafe {
            ffi::gf2c_decode_batch_fallback(self.raw, fallback.raw, llr.as_ptr(), f as i64, max_iterations as i32,
                                            fallback_iterations as i32, bits.as_mut_ptr(), iters.as_mut_ptr(),
                                            conv.as_mut_ptr(), synd.as_mut_ptr(), &mut redecoded,
                                            ffi::GF2C_MEM_HOST, ptr::null_mut())
        });
        let results = (0..f)
            .map(|i| {
                DecoderResult::new(BitVec::from_words(bits[i * wk..(i + 1) * wk].to_vec(), k), iters[i] as usize,
                                   conv[i] != 0, synd[i] != 0)
            })
            .collect();
        (results, redecoded as usize)
    }
}

impl Drop for CudaLdpcDecoder {
    fn drop(&mut self) {
        unsafe {
            ffi::gf2c_decoder_destroy(self.raw);
        }
    }
}

impl SoftDecoder for CudaLdpcDecoder {
    fn k(&self) -> usize {
        self.code.k
    }
    fn n(&self) -> usize {
        self.code.n
    }
    /// The reference's `decode_soft` is a hard decision on each of the n input
    /// LLRs (core.rs:877-885, Llr::hard_decision llr.rs:73-75).
    fn decode_soft(&self, llrs: &[Llr]) -> BitVec {
        assert_eq!(llrs.len(), self.code.n, "LLR length must equal n");
        let mut out = BitVec::with_capacity(self.code.n);
        for &l in llrs {
            out.push_bit(l.hard_decision());
        }
        out
    }
}

impl IterativeSoftDecoder for CudaLdpcDecoder {
    fn decode_iterative(&mut self, llrs: &[Llr], max_iterations: usize) -> DecoderResult {
        let r = self.decode_batch(&[llrs.to_vec()], max_iterations).pop().expect("one frame in, one result out");
        self.last_iterations = r.iterations;
        r
    }
    fn last_iteration_count(&self) -> usize {
        self.last_iterations
    }
    /// Every call decodes from the channel LLRs alone; no state carries over.
    fn reset(&mut self) {
        self.last_iterations = 0;
    }
}

/// `LdpcDecoder::decode_batch(code, llr_blocks, max_iterations)` as a free
/// function with the reference's signature.
pub fn decode_batch(code: CudaLdpcCode, llr_blocks: &[Vec<Llr>], max_iterations: usize) -> Vec<DecoderResult> {
    CudaLdpcDecoder::new(code).decode_batch(llr_blocks, max_iterations)
}

/// `LdpcEncoder`: systematic codewords [message | parity].
pub struct CudaLdpcEncoder<'a> {
    code: &'a CudaLdpcCode,
}

impl<'a> CudaLdpcEncoder<'a> {
    pub fn new(code: &'a CudaLdpcCode) -> Self {
        Self { code }
    }

    /// `LdpcEncoder::encode_batch` (core.rs:1106-1132).
    pub fn encode_batch(&self, messages: &[BitVec]) -> Vec<BitVec> {
        let (n, k, f) = (self.code.n, self.code.k, messages.len());
        if f == 0 {
            return Vec::new();
        }
        let (wk, wn) = (words(k), words(n));
        let mut msg = Vec::with_capacity(f * wk);
        for m in messages {
            assert_eq!(m.len(), k, "message length must equal k");
            msg.extend_from_slice(m.words());
        }
        let mut cw = vec![0u64; f * wn];
        check(unsafe {
            ffi::gf2c_encode_batch(self.code.raw, msg.as_ptr(), f as i64, cw.as_mut_ptr(), ffi::GF2C_MEM_HOST,
                                   ptr::null_mut())
        });
        cw.chunks(wn).map(|w| BitVec::from_words(w.to_vec(), n)).collect()
    }
}

impl BlockEncoder for CudaLdpcEncoder<'_> {
    fn k(&self) -> usize {
        self.code.k
    }
    fn n(&self) -> usize {
        self.code.n
    }
    fn encode(&self, message: &BitVec) -> BitVec {
        self.encode_batch(std::slice::from_ref(message)).pop().expect("one message in, one codeword out")
    }
}

/// DVB-T2 outer BCH code (`BchCode::dvb_t2`, crates/gf2-coding/src/bch/dvb_t2/mod.rs:62-78)
/// with batch encode / decode (`BchEncoder::encode_batch`, `BchDecoder::decode_batch`,
/// bch/core.rs:396-665): n of the BCH code is k of the matching LDPC code, so an
/// LDPC decode's message bits are a BCH codeword.
pub struct CudaBchCode {
    raw: *mut ffi::gf2c_bch,
    n: usize,
    k: usize,
}

unsafe impl Send for CudaBchCode {}

impl CudaBchCode {
    pub fn dvb_t2(frame: i32, rate: DvbRate) -> Self {
        let mut raw = ptr::null_mut();
        check(unsafe { ffi::gf2c_bch_create_dvbt2(frame, rate as i32, &mut raw) });
        let (mut n, mut k, mut t, mut m) = (0i64, 0i64, 0i32, 0i32);
        check(unsafe { ffi::gf2c_bch_dims(raw, &mut n, &mut k, &mut t, &mut m) });
        Self { raw, n: n as usize, k: k as usize }
    }

    pub fn n(&self) -> usize {
        self.n
    }
    pub fn k(&self) -> usize {
        self.k
    }

    /// Systematic codewords [message | parity] of a batch of messages.
    pub fn encode_batch(&mut self, messages: &[BitVec]) -> Vec<BitVec> {
        let (wk, wn, f) = (words(self.k), words(self.n), messages.len());
        if f == 0 {
            return Vec::new();
        }
        let mut msg = Vec::with_capacity(f * wk);
        for m in messages {
            assert_eq!(m.len(), self.k, "message length must equal k");
            msg.extend_from_slice(m.words());
        }
        let mut cw = vec![0u64; f * wn];
        check(unsafe {
            ffi::gf2c_bch_encode_batch(self.raw, msg.as_ptr(), f as i64, cw.as_mut_ptr(), ffi::GF2C_MEM_HOST,
                                       ptr::null_mut())
        });
        cw.chunks(wn).map(|w| BitVec::from_words(w.to_vec(), self.n)).collect()
    }

    /// Hard-decision decode of a batch of received words (bit-identical to
    /// `BchDecoder::decode`, including its behaviour beyond t errors).
    pub fn decode_batch(&mut self, received: &[BitVec]) -> Vec<BitVec> {
        let (wk, wn, f) = (words(self.k), words(self.n), received.len());
        if f == 0 {
            return Vec::new();
        }
        let mut cw = Vec::with_capacity(f * wn);
        for r in received {
            assert_eq!(r.len(), self.n, "received word length must equal n");
            cw.extend_from_slice(r.words());
        }
        let mut msg = vec![0u64; f * wk];
        check(unsafe {
            ffi::gf2c_bch_decode_batch(self.raw, cw.as_ptr(), f as i64, msg.as_mut_ptr(), ptr::null_mut(),
                                       ptr::null_mut(), ffi::GF2C_MEM_HOST, ptr::null_mut())
        });
        msg.chunks(wk).map(|w| BitVec::from_words(w.to_vec(), self.k)).collect()
    }
}

impl Drop for CudaBchCode {
    fn drop(&mut self) {
        unsafe {
            ffi::gf2c_bch_destroy(self.raw);
        }
    }
}
