"""gf2 file formats and the LDPC encoder cache, over the library's C ABI.

* BitVec / BitMatrix / SpBitMatrix / SpBitMatrixDual files in the reference's
  binary "GF2DATA", text and hex formats (crates/gf2-core/src/io): `save_bitvec`,
  `load_bitvec`, `save_bitmatrix`, `load_bitmatrix`, `save_sparse`,
  `load_sparse`, `probe`; LDPC codes from / to parity-check matrix files
  (`load_code`, `save_code`).
* `EncodingCache` (crates/gf2-coding/src/ldpc/encoding/cache.rs): dense
  parity parts P (k x r, row i = the parity of message bit i) keyed by
  (n, k, structural hash of H), saved as "n{n}_k{k}_h{hash:x}.gf2" BitMatrix
  files, and `DenseEncoder`, which encodes with such a P on the GPU.

Bits are numpy uint8 arrays (one bit per byte) or packed uint64 words.
"""
import ctypes
import os

import numpy as np

from . import _capi as C
from .ldpc import LdpcCode, _ptr, _stream_ptr, pack_bits, unpack_bits, words

BINARY, TEXT, HEX = 0, 1, 2
_FORMATS = {"binary": BINARY, "text": TEXT, "hex": HEX, BINARY: BINARY, TEXT: TEXT, HEX: HEX}
TYPE_BITVEC, TYPE_BITMATRIX, TYPE_SPBITMATRIX, TYPE_SPBITMATRIX_DUAL = 1, 2, 3, 4


def _fmt(format):
    if format is None:
        return -1
    try:
        return _FORMATS[format]
    except KeyError:
        raise ValueError(f"unknown format {format!r}") from None


def _path(p):
    return os.fsencode(p)


def _check(rc):
    if rc == C.ERR_INVALID_ARG:
        raise ValueError(C.lib.gf2c_last_error().decode())
    C.check(rc)


def probe(path):
    """(type tag, format, dims): SerializationFormat::detect plus the header."""
    tag, fmt = ctypes.c_int32(), ctypes.c_int32()
    dims = np.zeros(3, np.int64)
    _check(C.lib.gf2c_io_probe(_path(path), ctypes.byref(tag), ctypes.byref(fmt), _ptr(dims)))
    return tag.value, fmt.value, tuple(int(d) for d in dims)


# ---------------------------------------------------------------------------
# BitVec / BitMatrix
# ---------------------------------------------------------------------------
def save_bitvec(path, bits, format="binary", len_bits=None):
    """BitVec::save_to_file_with_format: `bits` one per byte, or packed words
    with `len_bits`."""
    a = np.asarray(bits)
    if len_bits is None:
        a = a.astype(np.uint8).reshape(-1)
        len_bits = a.size
        w = pack_bits(a, len_bits).reshape(-1) if len_bits else np.zeros(0, np.uint64)
    else:
        w = np.ascontiguousarray(a, np.uint64).reshape(-1)
    _check(C.lib.gf2c_io_write_bitvec(_path(path), _ptr(w) if w.size else None, int(len_bits), _fmt(format)))


def load_bitvec_words(path):
    """BitVec::load_from_file (format auto-detected): (packed words, len_bits)."""
    n = ctypes.c_int64()
    _check(C.lib.gf2c_io_read_bitvec(_path(path), None, 0, ctypes.byref(n)))
    w = np.zeros(words(n.value) if n.value else 0, np.uint64)
    _check(C.lib.gf2c_io_read_bitvec(_path(path), _ptr(w) if w.size else None, w.size, ctypes.byref(n)))
    return w, n.value


def load_bitvec(path):
    w, n = load_bitvec_words(path)
    return unpack_bits(w.reshape(1, -1), n)[0] if n else np.zeros(0, np.uint8)


def save_bitmatrix(path, matrix=None, format="binary", words_=None, rows=None, cols=None):
    """BitMatrix::save_to_file_with_format: a 0/1 array [rows, cols], or packed
    row words [rows, ceil(cols/64)] with rows / cols."""
    if words_ is None:
        m = np.asarray(matrix, np.uint8)
        rows, cols = m.shape
        w = pack_bits(m, cols) if rows and cols else np.zeros((rows, 0), np.uint64)
    else:
        w = np.ascontiguousarray(words_, np.uint64)
    _check(C.lib.gf2c_io_write_bitmatrix(_path(path), _ptr(w) if w.size else None, int(rows), int(cols), _fmt(format)))


def load_bitmatrix_words(path, format="binary"):
    """BitMatrix::load_from_file(_with_format): (row words [rows, stride], rows, cols)."""
    r, c = ctypes.c_int64(), ctypes.c_int64()
    f = _fmt(format)
    _check(C.lib.gf2c_io_read_bitmatrix(_path(path), f, None, 0, ctypes.byref(r), ctypes.byref(c)))
    S = words(c.value) if c.value else 0
    w = np.zeros((r.value, S), np.uint64)
    _check(C.lib.gf2c_io_read_bitmatrix(_path(path), f, _ptr(w) if w.size else None, w.size, ctypes.byref(r),
                                        ctypes.byref(c)))
    return w, r.value, c.value


def load_bitmatrix(path, format="binary"):
    w, r, c = load_bitmatrix_words(path, format)
    return unpack_bits(w, c) if r and c else np.zeros((r, c), np.uint8)


# ---------------------------------------------------------------------------
# sparse matrices and codes
# ---------------------------------------------------------------------------
def _csr_from_edges(rows, edges):
    e = np.asarray(edges, np.int64).reshape(-1, 2)
    ptr = np.zeros(rows + 1, np.int64)
    by_row = [sorted(set(int(c) for c in e[e[:, 0] == r, 1])) for r in range(rows)] if len(e) else [[]] * rows
    idx = np.array([c for row in by_row for c in row], np.int64)
    ptr[1:] = np.cumsum([len(row) for row in by_row])
    return ptr, idx


def save_sparse(path, rows, cols, row_ptr=None, col_idx=None, edges=None, dual=False, format="binary"):
    """SpBitMatrix (dual=False) / SpBitMatrixDual (dual=True)
    save_to_file_with_format, from CSR (ascending columns) or an edge list."""
    if edges is not None:
        row_ptr, col_idx = _csr_from_edges(rows, edges)
    ptr = np.ascontiguousarray(row_ptr, np.int64)
    idx = np.ascontiguousarray(col_idx, np.int64)
    _check(C.lib.gf2c_io_write_sparse(_path(path), TYPE_SPBITMATRIX_DUAL if dual else TYPE_SPBITMATRIX, int(rows),
                                      int(cols), _ptr(ptr), _ptr(idx) if idx.size else None, _fmt(format)))


def load_sparse(path, format=None):
    """SpBitMatrix / SpBitMatrixDual load: (rows, cols, row_ptr, col_idx)."""
    r, c, z = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    f = _fmt(format)
    _check(C.lib.gf2c_io_read_sparse(_path(path), f, ctypes.byref(r), ctypes.byref(c), ctypes.byref(z), None, None, 0))
    ptr = np.zeros(r.value + 1, np.int64)
    idx = np.zeros(max(z.value, 1), np.int64)
    _check(C.lib.gf2c_io_read_sparse(_path(path), f, ctypes.byref(r), ctypes.byref(c), ctypes.byref(z), _ptr(ptr),
                                     _ptr(idx), idx.size))
    return r.value, c.value, ptr, idx[: z.value]


def load_code(path):
    """An LdpcCode whose H is read from an SpBitMatrix / SpBitMatrixDual file."""
    return LdpcCode._create(C.lib.gf2c_code_create_file, _path(path))


def save_code(path, code, dual=True, format="binary"):
    """H of `code` as SpBitMatrixDual (default) or SpBitMatrix."""
    _check(C.lib.gf2c_io_write_code(_path(path), code.handle, TYPE_SPBITMATRIX_DUAL if dual else TYPE_SPBITMATRIX,
                                    _fmt(format)))


def siphash13(data, k0=0, k1=0):
    """SipHash-1-3 of `data` (bytes); Rust's DefaultHasher with its zero keys."""
    b = bytes(data)
    buf = ctypes.create_string_buffer(b, len(b)) if b else None
    out = ctypes.c_uint64()
    _check(C.lib.gf2c_siphash13(buf, len(b), k0, k1, ctypes.byref(out)))
    return out.value


# ---------------------------------------------------------------------------
# encoder cache
# ---------------------------------------------------------------------------
def cache_key(code):
    """CacheKey::from_params (cache.rs:84-90): (n, k, structural hash of H)."""
    h = ctypes.c_uint64()
    _check(C.lib.gf2c_code_cache_hash(code.handle, ctypes.byref(h)))
    return code.n(), code.k(), h.value


def cache_filename(key):
    n, k, h = key
    return f"n{n}_k{k}_h{h:x}.gf2"


def parse_cache_filename(name):
    """parse_cache_filename (cache.rs:490-502) on a file stem; None if malformed."""
    parts = name.split("_")
    if len(parts) != 3 or not (parts[0].startswith("n") and parts[1].startswith("k") and parts[2].startswith("h")):
        return None
    try:
        return int(parts[0][1:]), int(parts[1][1:]), int(parts[2][1:], 16)
    except ValueError:
        return None


def parity_part(code):
    """RuEncodingMatrices::parity_part: P words [k, ceil((n-k)/64)]."""
    k, r = code.k(), code.n() - code.k()
    P = np.zeros((k, words(r)), np.uint64)
    rc = C.lib.gf2c_code_parity_part(code.handle, _ptr(P))
    if rc == C.ERR_UNSUPPORTED:
        raise ValueError(C.lib.gf2c_last_error().decode())
    _check(rc)
    return P


_DENSE_DESTROY = C.lib.gf2c_dense_encoder_destroy


class DenseEncoder:
    """Encoder from a dense parity part (RuEncodingMatrices::encode /
    encode_batch): codeword = [message | P^T message], on the GPU."""

    def __init__(self, P, k, n):
        self.P = np.ascontiguousarray(P, np.uint64).reshape(k, words(n - k))
        self._k, self._n = int(k), int(n)
        h = ctypes.c_void_p()
        _check(C.lib.gf2c_dense_encoder_create(_ptr(self.P), self._k, self._n, ctypes.byref(h)))
        self.handle = h

    def __del__(self, _destroy=_DENSE_DESTROY):  # bound now: module globals may be gone at exit
        h = getattr(self, "handle", None)
        if h:
            _destroy(h)
            self.handle = None

    def k(self):
        return self._k

    def n(self):
        return self._n

    def encode_words(self, msg_words, stream=None):
        """Packed messages [F, ceil(k/64)] (numpy or CUDA tensor) -> packed codewords."""
        if hasattr(msg_words, "data_ptr"):
            import torch
            F = msg_words.shape[0]
            out = torch.zeros((F, words(self._n)), dtype=torch.int64, device=msg_words.device)
            st = stream or torch.cuda.current_stream(msg_words.device)
            _check(C.lib.gf2c_dense_encode_batch(self.handle, _ptr(msg_words.contiguous()), F, _ptr(out),
                                                 C.MEM_DEVICE, _stream_ptr(st)))
            return out
        m = np.ascontiguousarray(msg_words, np.uint64).reshape(-1, words(self._k))
        out = np.zeros((m.shape[0], words(self._n)), np.uint64)
        _check(C.lib.gf2c_dense_encode_batch(self.handle, _ptr(m), m.shape[0], _ptr(out), C.MEM_HOST, None))
        return out

    def encode(self, message):
        return self.encode_batch([message])[0]

    def encode_batch(self, messages):
        m = np.asarray(messages, np.uint8).reshape(-1, self._k)
        return unpack_bits(self.encode_words(pack_bits(m, self._k)), self._n)


class EncodingCache:
    """EncodingCache (cache.rs:141-438): parity parts keyed by CacheKey."""

    def __init__(self):
        self._entries = {}

    def get_or_compute(self, code):
        """The cached (or newly computed) parity part of `code`."""
        key = cache_key(code)
        if key not in self._entries:
            self._entries[key] = parity_part(code)
        return self._entries[key]

    def insert(self, key, P):
        n, k, _ = key
        self._entries[key] = np.ascontiguousarray(P, np.uint64).reshape(k, words(n - k))

    def get(self, code):
        return self._entries.get(cache_key(code))

    def encoder(self, code):
        """LdpcEncoder::with_cache: a DenseEncoder from the cached parity part."""
        return DenseEncoder(self.get_or_compute(code), code.k(), code.n())

    def precompute_dvb_t2(self):
        for frame in (0, 1):
            for rate in range(6):
                code = LdpcCode.dvb_t2_normal(rate) if frame == 0 else LdpcCode.dvb_t2_short(rate)
                self.get_or_compute(code)

    def stats(self):
        return {"entries": len(self._entries)}

    def clear(self):
        self._entries.clear()

    def keys(self):
        return list(self._entries)

    def save_to_directory(self, path):
        """save_to_directory (cache.rs:304-325): one BitMatrix file per entry."""
        os.makedirs(path, exist_ok=True)
        for key, P in self._entries.items():
            n, k, _ = key
            save_bitmatrix(os.path.join(path, cache_filename(key)), words_=P, rows=k, cols=n - k)

    @classmethod
    def from_directory(cls, path):
        """from_directory (cache.rs:347-433): every well-named .gf2 file."""
        if not os.path.isdir(path):
            raise FileNotFoundError(f"Directory does not exist: {path}")
        cache = cls()
        for name in sorted(os.listdir(path)):
            stem, ext = os.path.splitext(name)
            if ext != ".gf2":
                continue
            key = parse_cache_filename(stem)
            if key is None:
                continue
            n, k, _ = key
            P, rows, cols = load_bitmatrix_words(os.path.join(path, name))
            if rows != k or cols != n - k:
                raise ValueError(f"{name}: parity part is {rows} x {cols}, expected {k} x {n - k}")
            cache._entries[key] = P
        return cache
