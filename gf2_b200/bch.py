"""DVB-T2 outer BCH code on the GPU: the reference's BchCode / BchEncoder /
BchDecoder (crates/gf2-coding/src/bch) over the library's C ABI.

Codewords are [message (k) | parity (n - k)], bit i the coefficient of degree
n-1-i; n equals k of the matching LDPC code, so the message bits an LDPC
decoder returns are a BCH codeword.  Bits are numpy uint8 arrays (one bit per
byte) or packed uint64 words (the BitVec layout, `pack_bits`).
"""
import ctypes

import numpy as np

from . import _capi as C
from .ldpc import _ptr, _stream_ptr, pack_bits, unpack_bits, words

_BCH_DESTROY = C.lib.gf2c_bch_destroy


class BchCode:
    """BchCode::dvb_t2 (bch/dvb_t2/mod.rs:62-78)."""

    def __init__(self, handle):
        self.handle = handle
        n, k = ctypes.c_int64(), ctypes.c_int64()
        t, m = ctypes.c_int32(), ctypes.c_int32()
        C.check(C.lib.gf2c_bch_dims(handle, ctypes.byref(n), ctypes.byref(k), ctypes.byref(t), ctypes.byref(m)))
        self._n, self._k, self._t, self.field_m = n.value, k.value, t.value, m.value

    @classmethod
    def dvb_t2(cls, frame_size, rate):
        h = ctypes.c_void_p()
        rc = C.lib.gf2c_bch_create_dvbt2(int(frame_size), int(rate), ctypes.byref(h))
        if rc == C.ERR_INVALID_ARG:
            raise ValueError(C.lib.gf2c_last_error().decode())
        C.check(rc)
        return cls(h)

    def __del__(self, _destroy=_BCH_DESTROY):  # bound now: module globals may be gone at exit
        h = getattr(self, "handle", None)
        if h:
            _destroy(h)
            self.handle = None

    def n(self):
        return self._n

    def k(self):
        return self._k

    def t(self):
        return self._t

    def designed_distance(self):
        return 2 * self._t + 1

    def generator(self):
        """Binary coefficients of g(x), x^d at index d."""
        g = np.zeros(self._n - self._k + 1, np.uint8)
        C.check(C.lib.gf2c_bch_generator(self.handle, _ptr(g)))
        return g


class BchEncoder:
    """BchEncoder (bch/core.rs:347-480)."""

    def __init__(self, code):
        self.code = code

    def k(self):
        return self.code.k()

    def n(self):
        return self.code.n()

    def encode_words(self, msg_words, stream=None):
        """Packed messages [F, ceil(k/64)] (numpy or CUDA tensor) -> packed codewords."""
        c = self.code
        if hasattr(msg_words, "data_ptr"):
            import torch
            F = msg_words.shape[0]
            out = torch.zeros((F, words(c.n())), dtype=torch.int64, device=msg_words.device)
            st = stream or torch.cuda.current_stream(msg_words.device)
            C.check(C.lib.gf2c_bch_encode_batch(c.handle, _ptr(msg_words.contiguous()), F, _ptr(out), C.MEM_DEVICE,
                                                _stream_ptr(st)))
            return out
        m = np.ascontiguousarray(msg_words, np.uint64).reshape(-1, words(c.k()))
        out = np.zeros((m.shape[0], words(c.n())), np.uint64)
        C.check(C.lib.gf2c_bch_encode_batch(c.handle, _ptr(m), m.shape[0], _ptr(out), C.MEM_HOST, None))
        return out

    def encode(self, message):
        """BlockEncoder::encode: k bits -> n bits."""
        return self.encode_batch([message])[0]

    def encode_batch(self, messages):
        m = np.asarray(messages, np.uint8).reshape(-1, self.code.k())
        return unpack_bits(self.encode_words(pack_bits(m, self.code.k())), self.code.n())


class BchDecoder:
    """BchDecoder (bch/core.rs:486-818)."""

    def __init__(self, code):
        self.code = code

    def decode_words(self, cw_words, syndromes=False, stream=None):
        """Packed codewords [F, ceil(n/64)] -> dict(msg packed [F, ceil(k/64)],
        corrected [F] bits flipped, syndromes [F, 2t] when asked)."""
        c = self.code
        if hasattr(cw_words, "data_ptr"):
            import torch
            F = cw_words.shape[0]
            dev = cw_words.device
            out = dict(msg=torch.zeros((F, words(c.k())), dtype=torch.int64, device=dev),
                       corrected=torch.zeros(F, dtype=torch.int32, device=dev))
            if syndromes:
                out["syndromes"] = torch.zeros((F, 2 * c.t()), dtype=torch.int16, device=dev)
            st = stream or torch.cuda.current_stream(dev)
            C.check(C.lib.gf2c_bch_decode_batch(c.handle, _ptr(cw_words.contiguous()), F, _ptr(out["msg"]),
                                                _ptr(out["corrected"]), _ptr(out.get("syndromes")), C.MEM_DEVICE,
                                                _stream_ptr(st)))
            return out
        w = np.ascontiguousarray(cw_words, np.uint64).reshape(-1, words(c.n()))
        F = w.shape[0]
        out = dict(msg=np.zeros((F, words(c.k())), np.uint64), corrected=np.zeros(F, np.int32))
        if syndromes:
            out["syndromes"] = np.zeros((F, 2 * c.t()), np.uint16)
        C.check(C.lib.gf2c_bch_decode_batch(c.handle, _ptr(w), F, _ptr(out["msg"]), _ptr(out["corrected"]),
                                            _ptr(out.get("syndromes")), C.MEM_HOST, None))
        return out

    def compute_syndromes(self, received):
        """BchDecoder::compute_syndromes: S_1..S_2t of one received word."""
        r = self.decode_words(pack_bits(np.asarray(received, np.uint8), self.code.n()), syndromes=True)
        return r["syndromes"][0]

    def decode(self, received):
        """HardDecisionDecoder::decode: n bits -> k message bits."""
        return self.decode_batch([received])[0]

    def decode_batch(self, received):
        r = np.asarray(received, np.uint8).reshape(-1, self.code.n())
        out = self.decode_words(pack_bits(r, self.code.n()))
        return unpack_bits(out["msg"], self.code.k())
