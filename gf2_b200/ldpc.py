"""Host-side mirror of the gf2-coding LDPC API, backed by the sm_100a library.

Names, argument meaning and error behaviour follow erankavija/gf2
(crates/gf2-coding/src/): LdpcCode (ldpc/core.rs:59-262), QuasiCyclicLdpc and
CirculantMatrix (ldpc/core.rs:404-606), LdpcDecoder (ldpc/core.rs:632-960),
LdpcEncoder (ldpc/core.rs:984-1133), DecoderResult (traits.rs:115-177), Llr
(llr.rs:40-399), AwgnChannel / BpskModulator (channel.rs:51-295).

Bit vectors are numpy uint8 arrays holding one bit per element (the reference's
BitVec); the packed uint64 form of the C ABI is produced by pack_bits().  Where
the reference panics (assert_eq! on lengths, invalid shifts) this module raises
ValueError.  Every decode / encode call runs on the GPU through the C ABI;
there is no CPU path.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _capi as C


# ----------------------------------------------------------------------------
# bit packing (gf2-core BitVec: u64 words, bit i in word i/64 at position i%64)
# ----------------------------------------------------------------------------
def words(nbits):
    return (nbits + 63) // 64


def pack_bits(bits, nbits=None):
    b = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8))
    if b.ndim == 1:
        b = b[None, :]
    L = b.shape[1] if nbits is None else nbits
    W = words(L)
    pad = np.zeros((b.shape[0], W * 64), np.uint8)
    pad[:, :L] = b[:, :L] & 1
    return np.packbits(pad.reshape(b.shape[0], W, 64), axis=2, bitorder="little").view(np.uint64).reshape(
        b.shape[0], W)


def unpack_bits(packed, nbits):
    p = np.ascontiguousarray(np.asarray(packed, dtype=np.uint64))
    if p.ndim == 1:
        p = p[None, :]
    u = np.unpackbits(p.view(np.uint8).reshape(p.shape[0], -1), axis=1, bitorder="little")
    return u[:, :nbits]


# Bound at import time: object finalisers may run after module globals are
# cleared at interpreter exit.
_CODE_DESTROY = C.lib.gf2c_code_destroy
_DECODER_DESTROY = C.lib.gf2c_decoder_destroy


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream_ptr(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(stream)


class CodeRate:
    """bch::CodeRate (crates/gf2-coding/src/bch/mod.rs)."""
    Rate1_2 = 0
    Rate3_5 = 1
    Rate2_3 = 2
    Rate3_4 = 3
    Rate4_5 = 4
    Rate5_6 = 5


class FrameSize:
    Normal = 0
    Short = 1


# ----------------------------------------------------------------------------
# LLR and channel
# ----------------------------------------------------------------------------
class Llr:
    """Llr(f32) newtype (llr.rs:40-41); positive = bit 0 more likely."""

    __slots__ = ("_v",)

    def __init__(self, value):
        self._v = float(np.float32(value))

    def value(self):
        return self._v

    def hard_decision(self):
        return self._v < 0.0

    def magnitude(self):
        return abs(self._v)

    @staticmethod
    def zero():
        return Llr(0.0)

    @staticmethod
    def infinity():
        return Llr(np.inf)

    @staticmethod
    def neg_infinity():
        return Llr(-np.inf)

    def saturate(self, mx):
        return Llr(min(max(self._v, -mx), mx))

    def __repr__(self):
        return f"Llr({self._v})"


def _llr_array(llrs, n=None):
    if isinstance(llrs, np.ndarray):
        a = np.ascontiguousarray(llrs, dtype=np.float32)
    else:
        a = np.ascontiguousarray([x.value() if isinstance(x, Llr) else x for x in llrs], dtype=np.float32)
    if n is not None and a.shape[-1] != n:
        raise ValueError("LLR length must equal n")
    return a


class BpskModulator:
    """channel.rs:40-103."""

    @staticmethod
    def modulate(bit):
        return -1.0 if bit else 1.0

    @staticmethod
    def modulate_bits(bits):
        return [BpskModulator.modulate(b) for b in bits]

    @staticmethod
    def demodulate_hard(symbol):
        return symbol < 0.0

    @staticmethod
    def to_llr(received, sigma_squared):
        return Llr(np.float32(2.0 * received / sigma_squared))


class AwgnChannel:
    """AWGN channel (channel.rs:105-218).  Noise for GPU frames comes from the
    library's seeded Philox stream; the host-side transmit() uses numpy."""

    def __init__(self, sigma_squared):
        if not sigma_squared > 0.0:
            raise ValueError("Noise variance must be positive")
        self.sigma_squared = float(sigma_squared)

    @classmethod
    def from_variance(cls, sigma_squared):
        return cls(sigma_squared)

    @classmethod
    def from_eb_n0_db(cls, eb_n0_db, rate):
        if not (0.0 < rate <= 1.0):
            raise ValueError("Code rate must be in (0, 1]")
        return cls(C.lib.gf2c_sigma2_from_ebn0(float(eb_n0_db), float(rate)))

    def variance(self):
        return self.sigma_squared

    def transmit_symbols(self, symbols, rng):
        s = np.asarray(symbols, np.float64)
        return s + rng.normal(0.0, np.sqrt(self.sigma_squared), size=s.shape)

    def to_llrs(self, received):
        r = np.asarray(received, np.float64)
        return ((2.0 * r) / self.sigma_squared).astype(np.float32)


# ----------------------------------------------------------------------------
# codes
# ----------------------------------------------------------------------------
class CirculantMatrix:
    """ldpc/core.rs:381-448: row i has its 1 in column (i + shift) mod size."""

    def __init__(self, shift, size):
        self._shift, self._size = int(shift), int(size)

    def shift(self):
        return self._shift

    def size(self):
        return self._size

    def to_edges(self, base_row, base_col):
        z = self._size
        return [(base_row * z + i, base_col * z + (i + self._shift) % z) for i in range(z)]


class QuasiCyclicLdpc:
    """ldpc/core.rs:450-606."""

    def __init__(self, base_matrix, expansion_factor):
        if len(base_matrix) == 0:
            raise ValueError("Base matrix must have at least one row")
        if expansion_factor <= 0:
            raise ValueError("Expansion factor must be positive")
        cols = len(base_matrix[0])
        if any(len(r) != cols for r in base_matrix):
            raise ValueError("All rows in base matrix must have the same length")
        self.base_matrix = [list(map(int, r)) for r in base_matrix]
        self._z = int(expansion_factor)

    def base_rows(self):
        return len(self.base_matrix)

    def base_cols(self):
        return len(self.base_matrix[0])

    def expansion_factor(self):
        return self._z

    def expanded_rows(self):
        return self.base_rows() * self._z

    def expanded_cols(self):
        return self.base_cols() * self._z

    def to_edges(self):
        out = []
        for r, row in enumerate(self.base_matrix):
            for c, s in enumerate(row):
                if s == -1:
                    continue
                if not (0 <= s < self._z):
                    raise ValueError(f"Shift value {s} at position ({r},{c}) must be -1 or in range [0,{self._z})")
                out.extend(CirculantMatrix(s, self._z).to_edges(r, c))
        return out


class LdpcCode:
    """An LDPC code (parity-check matrix H), built by the library exactly as the
    reference builds it (same CSR/CSC neighbour orders)."""

    def __init__(self, handle):
        self._h = handle
        n, m, k, nnz = C._i64(), C._i64(), C._i64(), C._i64()
        lay = C._i32()
        C.check(C.lib.gf2c_code_dims(self._h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(k),
                                     ctypes.byref(nnz), ctypes.byref(lay)))
        self._n, self._m, self._k, self._nnz, self._layers = n.value, m.value, k.value, nnz.value, lay.value

    def __del__(self, _destroy=_CODE_DESTROY):  # bound now: module globals may be gone at exit
        h = getattr(self, "_h", None)
        if h:
            _destroy(h)
            self._h = None

    @classmethod
    def _create(cls, fn, *args):
        h = ctypes.c_void_p()
        rc = fn(*args, ctypes.byref(h))
        if rc == C.ERR_INVALID_ARG:
            raise ValueError(C.lib.gf2c_last_error().decode())
        C.check(rc)
        return cls(h)

    @classmethod
    def dvb_t2_short(cls, rate):
        return cls._create(C.lib.gf2c_code_create_dvbt2, FrameSize.Short, int(rate))

    @classmethod
    def dvb_t2_normal(cls, rate):
        return cls._create(C.lib.gf2c_code_create_dvbt2, FrameSize.Normal, int(rate))

    @classmethod
    def from_edges(cls, m, n, edges):
        a = np.ascontiguousarray(np.asarray(edges, dtype=np.int64).reshape(-1, 2))
        return cls._create(C.lib.gf2c_code_create_edges, int(m), int(n), _ptr(a), a.shape[0])

    @classmethod
    def from_quasi_cyclic(cls, qc):
        qc.to_edges()  # the reference's shift validation and panics
        b = np.ascontiguousarray(np.asarray(qc.base_matrix, dtype=np.int32))
        return cls._create(C.lib.gf2c_code_create_qc, _ptr(b), b.shape[0], b.shape[1], qc.expansion_factor())

    def n(self):
        return self._n

    def m(self):
        return self._m

    def k(self):
        return self._k

    def nnz(self):
        return self._nnz

    def layers(self):
        return self._layers

    def rate(self):
        return self._k / self._n

    @property
    def handle(self):
        return self._h

    def csr(self):
        ip = np.zeros(self._m + 1, np.int64)
        ix = np.zeros(max(self._nnz, 1), np.int64)
        C.check(C.lib.gf2c_code_csr(self._h, _ptr(ip), _ptr(ix)))
        return ip, ix[: self._nnz]

    # -- GPU batch operations on numpy / torch arrays --
    def syndrome_batch(self, cw_bits_packed, stream=None):
        """LdpcCode::syndrome over packed codewords [F, words(n)] -> (synd [F, words(m)], weight [F])."""
        if hasattr(cw_bits_packed, "data_ptr"):
            import torch
            F = cw_bits_packed.shape[0]
            s = torch.zeros((F, words(self._m)), dtype=torch.int64, device=cw_bits_packed.device)
            w = torch.zeros(F, dtype=torch.int32, device=cw_bits_packed.device)
            C.check(C.lib.gf2c_syndrome_batch(self._h, _ptr(cw_bits_packed), F, _ptr(s), _ptr(w), C.MEM_DEVICE,
                                              _stream_ptr(stream or torch.cuda.current_stream())))
            return s, w
        cw = np.ascontiguousarray(cw_bits_packed, np.uint64)
        F = cw.shape[0]
        s = np.zeros((F, words(self._m)), np.uint64)
        w = np.zeros(F, np.int32)
        C.check(C.lib.gf2c_syndrome_batch(self._h, _ptr(cw), F, _ptr(s), _ptr(w), C.MEM_HOST, None))
        return s, w

    def syndrome(self, codeword):
        """LdpcCode::syndrome (core.rs:129-133): s = H c over GF(2), as bits."""
        cw = np.asarray(codeword, np.uint8)
        if cw.shape[-1] != self._n:
            raise ValueError("Codeword length must equal n")
        s, _ = self.syndrome_batch(pack_bits(cw, self._n))
        return unpack_bits(s, self._m)[0]

    def is_valid_codeword(self, codeword):
        cw = np.asarray(codeword, np.uint8)
        if cw.shape[-1] != self._n:
            raise ValueError("Codeword length must equal n")
        _, w = self.syndrome_batch(pack_bits(cw, self._n))
        return int(w[0]) == 0


# ----------------------------------------------------------------------------
# decoder
# ----------------------------------------------------------------------------
@dataclass
class DecoderResult:
    """traits.rs:115-177."""
    decoded_bits: np.ndarray
    iterations: int
    converged: bool
    syndrome_check_passed: bool


def _opts(algorithm=C.ALGO_MINSUM, schedule=C.SCHED_FLOODING, msg_dtype=C.MSG_F32, early_stop=True,
          nms_alpha=None, nms_beta=None, threads_per_block=0, blocks_per_sm=0):
    o = C.DecoderOpts()
    C.lib.gf2c_decoder_opts_default(ctypes.byref(o))
    o.algorithm = algorithm
    o.schedule = schedule
    o.msg_dtype = msg_dtype
    o.early_stop = 1 if early_stop else 0
    o.threads_per_block = threads_per_block
    o.blocks_per_sm = blocks_per_sm
    keep = []
    if nms_alpha is not None:
        a = np.ascontiguousarray(nms_alpha, np.float32)
        b = np.ascontiguousarray(nms_beta, np.float32)
        if a.shape != b.shape or a.ndim != 2:
            raise ValueError("nms_alpha / nms_beta must be [iterations, layers]")
        o.nms_alpha = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        o.nms_beta = b.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        o.nms_iters = a.shape[0]
        keep = [a, b]
    return o, keep


class LdpcDecoder:
    """Belief-propagation decoder (ldpc/core.rs:632-960).

    The defaults reproduce the reference decoder: flooding plain min-sum with
    syndrome early stop.  algorithm / schedule / msg_dtype select the library's
    other decoders (sum-product, layered, FP16 message storage, learned
    normalised/offset min-sum)."""

    def __init__(self, code, algorithm=C.ALGO_MINSUM, schedule=C.SCHED_FLOODING, msg_dtype=C.MSG_F32,
                 early_stop=True, nms_alpha=None, nms_beta=None, threads_per_block=0, blocks_per_sm=0,
                 codes=None):
        self.code = code
        self.codes = list(codes) if codes is not None else [code]
        o, keep = _opts(algorithm, schedule, msg_dtype, early_stop, nms_alpha, nms_beta, threads_per_block,
                        blocks_per_sm)
        h = ctypes.c_void_p()
        arr = (ctypes.c_void_p * len(self.codes))(*[c.handle for c in self.codes])
        rc = C.lib.gf2c_decoder_create_multi(arr, len(self.codes), ctypes.byref(o), ctypes.byref(h))
        if rc == C.ERR_INVALID_ARG:
            raise ValueError(C.lib.gf2c_last_error().decode())
        C.check(rc)
        self._h = h
        self._last_iterations = 0
        del keep

    def __del__(self, _destroy=_DECODER_DESTROY):  # bound now: module globals may be gone at exit
        h = getattr(self, "_h", None)
        if h:
            _destroy(h)
            self._h = None

    def k(self):
        return self.code.k()

    def n(self):
        return self.code.n()

    def last_iteration_count(self):
        return self._last_iterations

    def reset(self):
        self._last_iterations = 0

    def last_launches(self):
        v = ctypes.c_int32()
        C.check(C.lib.gf2c_decoder_last_launches(self._h, ctypes.byref(v)))
        return v.value

    def decode_soft(self, llrs):
        """SoftDecoder::decode_soft (core.rs:877-885): hard decisions of the input."""
        a = _llr_array(llrs, self.n())
        return (a < 0).astype(np.uint8)

    def decode_arrays(self, llr, max_iterations, beliefs=False):
        """Decode a host batch llr [F, n] f32.  Returns dict of numpy arrays:
        msg (packed [F, words(k)]), iters, conv, synd_ok, beliefs (optional)."""
        a = _llr_array(llr)
        if a.ndim == 1:
            a = a[None, :]
        if a.shape[1] != self.n():
            raise ValueError("LLR length must equal n")
        if max_iterations < 0:
            raise ValueError("max_iterations must be >= 0")
        F = a.shape[0]
        msg = np.zeros((F, words(self.k())), np.uint64)
        it = np.zeros(F, np.int32)
        cv = np.zeros(F, np.uint8)
        so = np.zeros(F, np.uint8)
        bel = np.zeros((F, self.n()), np.float32) if beliefs else None
        C.check(C.lib.gf2c_decode_batch(self._h, _ptr(a), F, int(max_iterations), _ptr(msg), _ptr(it), _ptr(cv),
                                        _ptr(so), _ptr(bel), C.MEM_HOST, None))
        out = dict(msg=msg, iters=it, conv=cv.astype(bool), synd_ok=so.astype(bool))
        if beliefs:
            out["beliefs"] = bel
        return out

    def decode_tensors(self, llr, max_iterations, out=None, beliefs=False, stream=None):
        """Decode a device batch (torch CUDA tensor [F, n] f32), asynchronously on
        `stream`.  Returns a dict of device tensors."""
        import torch
        if llr.dtype != torch.float32 or not llr.is_cuda or llr.dim() != 2 or llr.shape[1] != self.n():
            raise ValueError("llr must be a CUDA float32 tensor [frames, n]")
        llr = llr.contiguous()
        F = llr.shape[0]
        dev = llr.device
        if out is None:
            out = dict(msg=torch.zeros((F, words(self.k())), dtype=torch.int64, device=dev),
                       iters=torch.zeros(F, dtype=torch.int32, device=dev),
                       conv=torch.zeros(F, dtype=torch.uint8, device=dev),
                       synd_ok=torch.zeros(F, dtype=torch.uint8, device=dev))
            if beliefs:
                out["beliefs"] = torch.zeros((F, self.n()), dtype=torch.float32, device=dev)
        st = stream or torch.cuda.current_stream(dev)
        C.check(C.lib.gf2c_decode_batch(self._h, _ptr(llr), F, int(max_iterations), _ptr(out["msg"]),
                                        _ptr(out["iters"]), _ptr(out["conv"]), _ptr(out["synd_ok"]),
                                        _ptr(out.get("beliefs")), C.MEM_DEVICE, _stream_ptr(st)))
        return out

    def decode_with_fallback(self, fallback, llr, max_iterations, fallback_iterations, out=None, stream=None):
        """This decoder on every frame of a batch, then `fallback` (a layered
        decoder of the same code) on the frames whose syndrome still fails,
        the list of those frames kept on the device
        (gf2c_decode_batch_fallback).
        Device batch (CUDA tensor [F, n] f32): asynchronous on `stream`; returns
        a dict of device tensors, fallback_count [1] int64 = frames re-decoded.
        Host batch (CPU tensor or numpy array [F, n] f32; pinned tensors copy
        fastest): copied in, decoded (large batches in chunks whose copies
        overlap decoding) and copied out before the call returns; returns CPU
        tensors (numpy arrays for numpy input) and fallback_count as an int."""
        import torch
        host_np = isinstance(llr, np.ndarray)
        if host_np:
            llr = torch.from_numpy(np.ascontiguousarray(llr, dtype=np.float32))
        if llr.dtype != torch.float32 or llr.dim() != 2 or llr.shape[1] != self.n():
            raise ValueError("llr must be a float32 tensor / array [frames, n]")
        llr = llr.contiguous()
        F, dev = llr.shape[0], llr.device
        if not llr.is_cuda:
            if out is None:
                pin = llr.is_pinned()
                out = dict(msg=torch.zeros((F, words(self.k())), dtype=torch.int64, pin_memory=pin),
                           iters=torch.zeros(F, dtype=torch.int32, pin_memory=pin),
                           conv=torch.zeros(F, dtype=torch.uint8, pin_memory=pin),
                           synd_ok=torch.zeros(F, dtype=torch.uint8, pin_memory=pin))
            want = dict(msg=torch.int64, iters=torch.int32, conv=torch.uint8, synd_ok=torch.uint8)
            for k, dt in want.items():
                if out[k].is_cuda or not out[k].is_contiguous() or out[k].shape[0] != F or out[k].dtype != dt:
                    raise ValueError("host outputs must be contiguous CPU tensors of the batch's frames "
                                     "(msg int64 [F, words(k)], iters int32, conv / synd_ok uint8)")
            if out["msg"].dim() != 2 or out["msg"].shape[1] != words(self.k()):
                raise ValueError("msg must be int64 [frames, words(k)]")
            cnt = np.zeros(1, np.int64)
            C.check(C.lib.gf2c_decode_batch_fallback(self._h, fallback._h, _ptr(llr), F, int(max_iterations),
                                                     int(fallback_iterations), _ptr(out["msg"]), _ptr(out["iters"]),
                                                     _ptr(out["conv"]), _ptr(out["synd_ok"]), _ptr(cnt),
                                                     C.MEM_HOST, None))
            out["fallback_count"] = int(cnt[0])
            if host_np:
                out = {k: (v.numpy() if hasattr(v, "numpy") else v) for k, v in out.items()}
            return out
        if out is None:
            out = dict(msg=torch.zeros((F, words(self.k())), dtype=torch.int64, device=dev),
                       iters=torch.zeros(F, dtype=torch.int32, device=dev),
                       conv=torch.zeros(F, dtype=torch.uint8, device=dev),
                       synd_ok=torch.zeros(F, dtype=torch.uint8, device=dev),
                       fallback_count=torch.zeros(1, dtype=torch.int64, device=dev))
        st = stream or torch.cuda.current_stream(dev)
        C.check(C.lib.gf2c_decode_batch_fallback(self._h, fallback._h, _ptr(llr), F, int(max_iterations),
                                                 int(fallback_iterations), _ptr(out["msg"]), _ptr(out["iters"]),
                                                 _ptr(out["conv"]), _ptr(out["synd_ok"]),
                                                 _ptr(out["fallback_count"]), C.MEM_DEVICE, _stream_ptr(st)))
        return out

    def decode_iterative(self, llrs, max_iterations):
        """IterativeSoftDecoder::decode_iterative (traits.rs:335, core.rs:889-938)."""
        a = _llr_array(llrs, self.n())
        r = self.decode_arrays(a[None, :], max_iterations)
        self._last_iterations = int(r["iters"][0])
        return DecoderResult(unpack_bits(r["msg"], self.k())[0], int(r["iters"][0]), bool(r["conv"][0]),
                             bool(r["synd_ok"][0]))

    @staticmethod
    def decode_batch(code, llr_blocks, max_iterations, **kw):
        """LdpcDecoder::decode_batch (core.rs:729-756) -> list of DecoderResult."""
        if len(llr_blocks) == 0:
            return []
        a = np.stack([_llr_array(b, code.n()) for b in llr_blocks])
        dec = LdpcDecoder(code, **kw)
        r = dec.decode_arrays(a, max_iterations)
        bits = unpack_bits(r["msg"], code.k())
        return [DecoderResult(bits[i], int(r["iters"][i]), bool(r["conv"][i]), bool(r["synd_ok"][i]))
                for i in range(a.shape[0])]

    def decode_mixed_tensors(self, llr, llr_offset, code_id, max_iter, msg, msg_offset, iters, conv, synd_ok,
                             use_graph=True, stream=None):
        """Mixed-code batch in one persistent launch (device tensors)."""
        import torch
        st = stream or torch.cuda.current_stream(llr.device)
        C.check(C.lib.gf2c_decode_mixed(self._h, _ptr(llr), _ptr(llr_offset), _ptr(code_id), _ptr(max_iter),
                                        int(code_id.shape[0]), _ptr(msg), _ptr(msg_offset), _ptr(iters),
                                        _ptr(conv), _ptr(synd_ok), 1 if use_graph else 0, C.MEM_DEVICE,
                                        _stream_ptr(st)))

    def decode_mixed_arrays(self, llr, llr_offset, code_id, max_iter, msg_offset):
        """Mixed-code batch from host arrays; returns dict of numpy arrays."""
        llr = np.ascontiguousarray(llr, np.float32)
        lo = np.ascontiguousarray(llr_offset, np.int64)
        cid = np.ascontiguousarray(code_id, np.int32)
        mit = np.ascontiguousarray(max_iter, np.int32)
        mo = np.ascontiguousarray(msg_offset, np.int64)
        F = cid.shape[0]
        total = int(max((mo[f] + words(self.codes[cid[f]].k()) for f in range(F)), default=1))
        msg = np.zeros(total, np.uint64)
        it = np.zeros(F, np.int32)
        cv = np.zeros(F, np.uint8)
        so = np.zeros(F, np.uint8)
        C.check(C.lib.gf2c_decode_mixed(self._h, _ptr(llr), _ptr(lo), _ptr(cid), _ptr(mit), F, _ptr(msg), _ptr(mo),
                                        _ptr(it), _ptr(cv), _ptr(so), 0, C.MEM_HOST, None))
        return dict(msg=msg, iters=it, conv=cv.astype(bool), synd_ok=so.astype(bool))


# ----------------------------------------------------------------------------
# encoder and channel
# ----------------------------------------------------------------------------
class LdpcEncoder:
    """Systematic encoder (ldpc/core.rs:984-1133)."""

    def __init__(self, code):
        self.code = code

    def k(self):
        return self.code.k()

    def n(self):
        return self.code.n()

    def encode_packed(self, msg_packed, stream=None):
        if hasattr(msg_packed, "data_ptr"):
            import torch
            F = msg_packed.shape[0]
            cw = torch.zeros((F, words(self.n())), dtype=torch.int64, device=msg_packed.device)
            C.check(C.lib.gf2c_encode_batch(self.code.handle, _ptr(msg_packed), F, _ptr(cw), C.MEM_DEVICE,
                                            _stream_ptr(stream or torch.cuda.current_stream())))
            return cw
        m = np.ascontiguousarray(msg_packed, np.uint64)
        cw = np.zeros((m.shape[0], words(self.n())), np.uint64)
        rc = C.lib.gf2c_encode_batch(self.code.handle, _ptr(m), m.shape[0], _ptr(cw), C.MEM_HOST, None)
        if rc == C.ERR_RANK:
            raise ValueError(C.lib.gf2c_last_error().decode())
        C.check(rc)
        return cw

    def encode(self, message):
        """BlockEncoder::encode (traits.rs:206): k bits -> n bits."""
        msg = np.asarray(message, np.uint8)
        if msg.shape[-1] != self.k():
            raise ValueError(f"Message length must be k = {self.k()}")
        return unpack_bits(self.encode_packed(pack_bits(msg, self.k())), self.n())[0]

    def encode_batch(self, messages):
        """LdpcEncoder::encode_batch (core.rs:1106-1120)."""
        if len(messages) == 0:
            return []
        m = np.stack([np.asarray(x, np.uint8) for x in messages])
        if m.shape[1] != self.k():
            raise ValueError(f"Message length must be k = {self.k()}")
        cw = unpack_bits(self.encode_packed(pack_bits(m, self.k())), self.n())
        return [cw[i] for i in range(cw.shape[0])]


def awgn_frames(code, seed, frame0, frames, sigma2, device=None, want_info=True, want_cw=True, stream=None):
    """Seeded synthetic frames on the GPU: info bits, codewords, LLRs.

    sigma2: scalar or per-frame array.  With device=None the results are numpy
    arrays (host path of the C ABI); with a torch device they are CUDA tensors."""
    if device is None:
        s2 = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma2, np.float64), (frames,)))
        info = np.zeros((frames, words(code.k())), np.uint64) if want_info else None
        cw = np.zeros((frames, words(code.n())), np.uint64) if want_cw else None
        llr = np.zeros((frames, code.n()), np.float32)
        C.check(C.lib.gf2c_channel_awgn(code.handle, int(seed), int(frame0), int(frames), _ptr(s2), _ptr(info),
                                        _ptr(cw), _ptr(llr), C.MEM_HOST, None))
        return info, cw, llr
    import torch
    s2 = torch.as_tensor(np.broadcast_to(np.asarray(sigma2, np.float64), (frames,)).copy(), device=device)
    info = torch.zeros((frames, words(code.k())), dtype=torch.int64, device=device) if want_info else None
    cw = torch.zeros((frames, words(code.n())), dtype=torch.int64, device=device) if want_cw else None
    llr = torch.empty((frames, code.n()), dtype=torch.float32, device=device)
    C.check(C.lib.gf2c_channel_awgn(code.handle, int(seed), int(frame0), int(frames), _ptr(s2), _ptr(info),
                                    _ptr(cw), _ptr(llr), C.MEM_DEVICE,
                                    _stream_ptr(stream or torch.cuda.current_stream(device))))
    return info, cw, llr


def judge_spa64(code, llr, max_iterations, schedule=C.SCHED_LAYERED, beliefs=False, stream=None):
    """FP64 sum-product judge on the GPU (gf2c_judge_spa64): the precision
    reference the FP32 / FP16 decoders are stated against.  llr: CUDA float32
    tensor [F, n].  Returns a dict of device tensors like
    LdpcDecoder.decode_tensors; beliefs are float64."""
    import torch
    if llr.dtype != torch.float32 or not llr.is_cuda or llr.dim() != 2 or llr.shape[1] != code.n():
        raise ValueError("llr must be a CUDA float32 tensor [frames, n]")
    llr = llr.contiguous()
    F, dev = llr.shape[0], llr.device
    out = dict(msg=torch.zeros((F, words(code.k())), dtype=torch.int64, device=dev),
               iters=torch.zeros(F, dtype=torch.int32, device=dev),
               conv=torch.zeros(F, dtype=torch.uint8, device=dev),
               synd_ok=torch.zeros(F, dtype=torch.uint8, device=dev))
    if beliefs:
        out["beliefs"] = torch.zeros((F, code.n()), dtype=torch.float64, device=dev)
    st = stream or torch.cuda.current_stream(dev)
    C.check(C.lib.gf2c_judge_spa64(code.handle, int(schedule), _ptr(llr), F, int(max_iterations), _ptr(out["msg"]),
                                   _ptr(out["iters"]), _ptr(out["conv"]), _ptr(out["synd_ok"]),
                                   _ptr(out.get("beliefs")), _stream_ptr(st)))
    return out


def sigma2_from_ebn0(ebn0_db, rate):
    return C.lib.gf2c_sigma2_from_ebn0(float(ebn0_db), float(rate))
