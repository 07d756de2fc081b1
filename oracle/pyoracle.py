"""ctypes bindings of the CPU oracle (test infrastructure only).

Imported by the tests, by the smoke check and by the CPU-baseline leg of the
benchmark.  Bits are numpy uint8 arrays (one bit per byte).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)


def build():
    """Compile liboracle.so with its Makefile (idempotent)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.or_code_dvbt2.restype = ctypes.c_void_p
        L.or_code_dvbt2.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_code_qc.restype = ctypes.c_void_p
        L.or_code_qc.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_code_edges.restype = ctypes.c_void_p
        L.or_code_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, _i64p, ctypes.c_int64]
        L.or_code_free.argtypes = [ctypes.c_void_p]
        L.or_code_dims.argtypes = [ctypes.c_void_p, _i64p]
        L.or_code_csr.argtypes = [ctypes.c_void_p, _i64p, _i64p]
        L.or_code_csc.argtypes = [ctypes.c_void_p, _i64p, _i64p]
        L.or_last_error.restype = ctypes.c_char_p
        L.or_syndrome.restype = ctypes.c_int64
        L.or_syndrome.argtypes = [ctypes.c_void_p, _u8p, _u8p]
        L.or_decode_minsum_faithful.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, ctypes.c_int,
                                                ctypes.c_int, _u8p, _i32p, _u8p, _u8p, _f32p]
        L.or_decode.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
                                _u8p, _i32p, _u8p, _u8p, _f32p]
        L.or_decode_spa64.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_int64, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, _u8p, _i32p, _u8p, _u8p, _f64p]
        L.or_code_layers.argtypes = [ctypes.c_void_p]
        L.or_code_check_layer.argtypes = [ctypes.c_void_p, _i32p]
        L.or_encode.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _u8p]
        L.or_encoder_columns.argtypes = [ctypes.c_void_p, _i64p, _i64p]
        L.or_philox4x32.argtypes = [_u32p, _u32p, _u32p]
        L.or_channel_frames.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_int64, _f64p, _u8p, _u8p, _f32p]
        L.or_sigma2.restype = ctypes.c_double
        L.or_sigma2.argtypes = [ctypes.c_double, ctypes.c_double]
        L.or_own_log.restype = ctypes.c_double
        L.or_own_log.argtypes = [ctypes.c_double]
        L.or_own_sincos2pi.argtypes = [ctypes.c_double, _f64p, _f64p]
        L.or_shannon_limit.restype = ctypes.c_double
        L.or_shannon_limit.argtypes = [ctypes.c_double]
        L.or_nms_layered_loss_grad.restype = ctypes.c_double
        L.or_nms_layered_loss_grad.argtypes = [ctypes.c_void_p, _f32p, _u8p, ctypes.c_int64, ctypes.c_int,
                                               _f64p, _f64p, _f64p, _f64p, _f64p]
        L.or_nms_loss_grad.restype = ctypes.c_double
        L.or_nms_loss_grad.argtypes = [ctypes.c_void_p, _f32p, _u8p, ctypes.c_int64, ctypes.c_int,
                                       _f64p, _f64p, _f64p, _f64p, _f64p]
        L.or_f32_to_f16.restype = ctypes.c_uint16
        L.or_f32_to_f16.argtypes = [ctypes.c_float]
        L.or_f16_to_f32.restype = ctypes.c_float
        L.or_f16_to_f32.argtypes = [ctypes.c_uint16]
        _u16p = ctypes.POINTER(ctypes.c_uint16)
        L.or_bch_dvbt2.restype = ctypes.c_void_p
        L.or_bch_dvbt2.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_bch_free.argtypes = [ctypes.c_void_p]
        L.or_bch_dims.argtypes = [ctypes.c_void_p, _i64p]
        L.or_bch_generator.argtypes = [ctypes.c_void_p, _u8p]
        L.or_bch_encode.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _u8p]
        L.or_bch_syndromes.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _u16p]
        L.or_bch_berlekamp_massey.restype = ctypes.c_int
        L.or_bch_berlekamp_massey.argtypes = [ctypes.c_void_p, _u16p, _u16p]
        L.or_bch_decode.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _u8p, _i32p]
        _LIB = L
    return _LIB


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


class OracleError(RuntimeError):
    pass


class Code:
    """A parity-check matrix built the way the reference builds it."""

    def __init__(self, handle):
        if not handle:
            raise OracleError(lib().or_last_error().decode())
        self.h = handle
        d = np.zeros(4, np.int64)
        lib().or_code_dims(self.h, _p(d, _i64p))
        self.n, self.m, self.k, self.nnz = (int(x) for x in d)
        self.layers = int(lib().or_code_layers(self.h))

    @classmethod
    def dvbt2(cls, frame, rate):
        return cls(lib().or_code_dvbt2(frame, rate))

    @classmethod
    def qc(cls, base, z):
        b = np.ascontiguousarray(np.asarray(base, np.int32))
        return cls(lib().or_code_qc(_p(b, _i32p), b.shape[0], b.shape[1], z))

    @classmethod
    def edges(cls, m, n, pairs):
        a = np.ascontiguousarray(np.asarray(pairs, np.int64).reshape(-1, 2))
        return cls(lib().or_code_edges(m, n, _p(a, _i64p), a.shape[0]))

    def __del__(self):
        try:
            lib().or_code_free(self.h)
        except Exception:
            pass

    @property
    def rate(self):
        return self.k / self.n

    def csr(self):
        ip = np.zeros(self.m + 1, np.int64)
        ix = np.zeros(self.nnz, np.int64)
        lib().or_code_csr(self.h, _p(ip, _i64p), _p(ix, _i64p))
        return ip, ix

    def csc(self):
        ip = np.zeros(self.n + 1, np.int64)
        ix = np.zeros(self.nnz, np.int64)
        lib().or_code_csc(self.h, _p(ip, _i64p), _p(ix, _i64p))
        return ip, ix

    def check_layer(self):
        a = np.zeros(self.m, np.int32)
        lib().or_code_check_layer(self.h, _p(a, _i32p))
        return a

    def syndrome(self, cw):
        cw = np.ascontiguousarray(cw, np.uint8)
        s = np.zeros(self.m, np.uint8)
        lib().or_syndrome(self.h, _p(cw, _u8p), _p(s, _u8p))
        return s

    # ---- decoders ----
    def _outs(self, frames):
        return (np.zeros((frames, self.k), np.uint8), np.zeros(frames, np.int32),
                np.zeros(frames, np.uint8), np.zeros(frames, np.uint8),
                np.zeros((frames, self.n), np.float32))

    def decode_faithful(self, llr, max_iter, threads=0):
        llr = np.ascontiguousarray(llr, np.float32).reshape(-1, self.n)
        F = llr.shape[0]
        msg, it, cv, so, bel = self._outs(F)
        rc = lib().or_decode_minsum_faithful(self.h, _p(llr, _f32p), F, max_iter, threads,
                                             _p(msg, _u8p), _p(it, _i32p), _p(cv, _u8p),
                                             _p(so, _u8p), _p(bel, _f32p))
        if rc:
            raise OracleError(lib().or_last_error().decode())
        return dict(msg=msg, iters=it, conv=cv.astype(bool), synd_ok=so.astype(bool), beliefs=bel)

    def decode(self, llr, max_iter, algo=0, sched=0, msg16=False, alpha=None, beta=None,
               threads=0):
        llr = np.ascontiguousarray(llr, np.float32).reshape(-1, self.n)
        F = llr.shape[0]
        msg, it, cv, so, bel = self._outs(F)
        nw = 0
        if alpha is not None:
            alpha = np.ascontiguousarray(alpha, np.float32)
            beta = np.ascontiguousarray(beta, np.float32)
            nw = alpha.size // max(self.layers, 1)
        rc = lib().or_decode(self.h, _p(llr, _f32p), F, max_iter, algo, sched, int(msg16),
                             _p(alpha, _f32p), _p(beta, _f32p), nw, threads, _p(msg, _u8p),
                             _p(it, _i32p), _p(cv, _u8p), _p(so, _u8p), _p(bel, _f32p))
        if rc:
            raise OracleError(lib().or_last_error().decode())
        return dict(msg=msg, iters=it, conv=cv.astype(bool), synd_ok=so.astype(bool), beliefs=bel)

    def decode_spa64(self, llr, max_iter, sched=0, threads=0):
        llr = np.ascontiguousarray(llr, np.float32).reshape(-1, self.n)
        F = llr.shape[0]
        msg, it, cv, so, _ = self._outs(F)
        bel = np.zeros((F, self.n), np.float64)
        rc = lib().or_decode_spa64(self.h, _p(llr, _f32p), F, max_iter, sched, threads,
                                   _p(msg, _u8p), _p(it, _i32p), _p(cv, _u8p), _p(so, _u8p),
                                   _p(bel, _f64p))
        if rc:
            raise OracleError(lib().or_last_error().decode())
        return dict(msg=msg, iters=it, conv=cv.astype(bool), synd_ok=so.astype(bool), beliefs=bel)

    # ---- encoder / channel ----
    def encode(self, msg):
        msg = np.ascontiguousarray(msg, np.uint8).reshape(-1, self.k)
        cw = np.zeros((msg.shape[0], self.n), np.uint8)
        if lib().or_encode(self.h, _p(msg, _u8p), msg.shape[0], _p(cw, _u8p)):
            raise OracleError(lib().or_last_error().decode())
        return cw

    def encoder_columns(self):
        mc = np.zeros(self.k, np.int64)
        pc = np.zeros(self.m, np.int64)
        if lib().or_encoder_columns(self.h, _p(mc, _i64p), _p(pc, _i64p)):
            raise OracleError(lib().or_last_error().decode())
        return mc, pc

    def channel(self, seed, frame0, frames, ebn0_db):
        eb = np.ascontiguousarray(np.broadcast_to(np.asarray(ebn0_db, np.float64), (frames,)))
        info = np.zeros((frames, self.k), np.uint8)
        cw = np.zeros((frames, self.n), np.uint8)
        llr = np.zeros((frames, self.n), np.float32)
        if lib().or_channel_frames(self.h, seed, frame0, frames, _p(eb, _f64p), _p(info, _u8p),
                                   _p(cw, _u8p), _p(llr, _f32p)):
            raise OracleError(lib().or_last_error().decode())
        return info, cw, llr

    def nms_loss_grad(self, llr, cw, T, alpha, beta, layered=False):
        llr = np.ascontiguousarray(llr, np.float32).reshape(-1, self.n)
        cw = np.ascontiguousarray(cw, np.uint8).reshape(-1, self.n)
        a = np.ascontiguousarray(alpha, np.float64)
        b = np.ascontiguousarray(beta, np.float64)
        ga = np.zeros_like(a)
        gb = np.zeros_like(b)
        out = np.zeros(llr.shape, np.float64)
        fn = lib().or_nms_layered_loss_grad if layered else lib().or_nms_loss_grad
        loss = fn(self.h, _p(llr, _f32p), _p(cw, _u8p), llr.shape[0], T,
                  _p(a, _f64p), _p(b, _f64p), _p(ga, _f64p), _p(gb, _f64p), _p(out, _f64p))
        if loss != loss:
            raise OracleError(lib().or_last_error().decode())
        return loss, ga, gb, out


def philox4x32(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().or_philox4x32(_p(c, _u32p), _p(k, _u32p), _p(o, _u32p))
    return o


def sigma2(ebn0_db, rate):
    return lib().or_sigma2(ebn0_db, rate)


def shannon_limit(rate):
    return lib().or_shannon_limit(rate)


def f32_to_f16_bits(x):
    return lib().or_f32_to_f16(x)


class Bch:
    """DVB-T2 outer BCH code (bch.cpp): BchCode::dvb_t2, encode, syndromes,
    Berlekamp-Massey, decode (bits one per byte)."""

    def __init__(self, frame, rate):
        self.h = lib().or_bch_dvbt2(frame, rate)
        if not self.h:
            raise OracleError("bad DVB-T2 BCH frame / rate")
        d = np.zeros(5, np.int64)
        lib().or_bch_dims(self.h, _p(d, _i64p))
        self.n, self.k, self.t, self.field_m, self.gen_degree = (int(x) for x in d)

    def __del__(self):
        try:
            lib().or_bch_free(self.h)
        except Exception:
            pass

    def generator(self):
        g = np.zeros(self.gen_degree + 1, np.uint8)
        lib().or_bch_generator(self.h, _p(g, _u8p))
        return g

    def encode(self, msg):
        m = np.ascontiguousarray(msg, np.uint8).reshape(-1, self.k)
        cw = np.zeros((m.shape[0], self.n), np.uint8)
        lib().or_bch_encode(self.h, _p(m, _u8p), m.shape[0], _p(cw, _u8p))
        return cw

    def syndromes(self, cw):
        c = np.ascontiguousarray(cw, np.uint8).reshape(-1, self.n)
        s = np.zeros((c.shape[0], 2 * self.t), np.uint16)
        lib().or_bch_syndromes(self.h, _p(c, _u8p), c.shape[0], _p(s, ctypes.POINTER(ctypes.c_uint16)))
        return s

    def berlekamp_massey(self, synd):
        s = np.ascontiguousarray(synd, np.uint16)
        lam = np.zeros(2 * self.t + 1, np.uint16)
        deg = lib().or_bch_berlekamp_massey(self.h, _p(s, ctypes.POINTER(ctypes.c_uint16)),
                                            _p(lam, ctypes.POINTER(ctypes.c_uint16)))
        return lam[:deg + 1]

    def decode(self, cw):
        c = np.ascontiguousarray(cw, np.uint8).reshape(-1, self.n)
        msg = np.zeros((c.shape[0], self.k), np.uint8)
        flips = np.zeros(c.shape[0], np.int32)
        lib().or_bch_decode(self.h, _p(c, _u8p), c.shape[0], _p(msg, _u8p), _p(flips, _i32p))
        return msg, flips
