"""CPU tests of the C ABI: the library loads, exports every declared symbol,
builds codes identical to the oracle's, and rejects bad arguments with status
codes (no GPU work is issued here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "gf2cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gf2c_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from gf2_b200 import _capi
    lib = ctypes.CDLL(_capi.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(_capi.EXPORTS) == syms


def test_codes_match_oracle(oracle):
    import gf2_b200 as g
    for idx in range(12):
        a = g.LdpcCode.dvb_t2_normal(idx) if idx < 6 else g.LdpcCode.dvb_t2_short(idx - 6)
        b = oracle.Code.dvbt2(idx // 6, idx % 6)
        ip, ix = a.csr()
        jp, jx = b.csr()
        assert (ip == jp).all() and (ix == jx).all()
        assert (a.n(), a.m(), a.k(), a.layers()) == (b.n, b.m, b.k, b.layers)
    base = [[0, 1, -1, 2], [3, -1, 0, 1]]
    a = g.LdpcCode.from_quasi_cyclic(g.QuasiCyclicLdpc(base, 5))
    b = oracle.Code.qc(base, 5)
    assert (a.csr()[1] == b.csr()[1]).all() and a.layers() == 2
    edges = [(0, 1), (0, 1), (1, 2), (1, 0), (2, 3)]
    a = g.LdpcCode.from_edges(3, 4, edges)
    b = oracle.Code.edges(3, 4, edges)
    assert (a.csr()[1] == b.csr()[1]).all() and a.nnz() == 3 and a.layers() == 0


def test_invalid_arguments_return_codes():
    import gf2_b200 as g
    with pytest.raises(ValueError):
        g.LdpcCode.from_edges(2, 3, [(5, 0)])
    with pytest.raises(ValueError):
        g.LdpcCode.from_quasi_cyclic(g.QuasiCyclicLdpc([[7]], 3))
    with pytest.raises(ValueError):
        g.QuasiCyclicLdpc([], 3)
    from gf2_b200 import _capi
    h = ctypes.c_void_p()
    assert _capi.lib.gf2c_code_create_dvbt2(2, 0, ctypes.byref(h)) == _capi.ERR_INVALID_ARG
    assert _capi.lib.gf2c_code_create_dvbt2(0, 6, ctypes.byref(h)) == _capi.ERR_INVALID_ARG
    assert _capi.lib.gf2c_code_create_qc(None, 1, 1, 3, ctypes.byref(h)) == _capi.ERR_INVALID_ARG
    assert b"frame" in _capi.lib.gf2c_last_error() or len(_capi.lib.gf2c_last_error()) > 0
    assert _capi.lib.gf2c_decode_batch(None, None, 1, 5, None, None, None, None, None, 0, None) == \
        _capi.ERR_INVALID_ARG
    assert _capi.lib.gf2c_decoder_create(None, None, ctypes.byref(h)) == _capi.ERR_INVALID_ARG


def test_bit_packing_roundtrip():
    import gf2_b200 as g
    rng = np.random.default_rng(0)
    for L in (1, 63, 64, 65, 7200, 16200):
        b = rng.integers(0, 2, (3, L), dtype=np.uint8)
        p = g.pack_bits(b, L)
        assert p.shape == (3, (L + 63) // 64)
        assert (g.unpack_bits(p, L) == b).all()
        # BitVec layout: bit i in word i // 64 at position i % 64
        i = L - 1
        assert ((int(p[0, i // 64]) >> (i % 64)) & 1) == b[0, i]


def test_llr_and_channel_helpers():
    import gf2_b200 as g
    assert g.Llr(3.5).hard_decision() is False and g.Llr(-2.0).hard_decision() is True
    assert g.Llr(0.0).hard_decision() is False
    assert g.Llr(100.0).saturate(10.0).value() == 10.0
    assert g.BpskModulator.modulate(False) == 1.0 and g.BpskModulator.modulate(True) == -1.0
    ch = g.AwgnChannel.from_eb_n0_db(1.0, 7200 / 16200)
    assert abs(ch.variance() - 1.0 / (2 * (7200 / 16200) * 10 ** 0.1)) < 1e-15
    with pytest.raises(ValueError):
        g.AwgnChannel.from_variance(0.0)
    assert g.CirculantMatrix(1, 4).to_edges(0, 0) == [(0, 1), (1, 2), (2, 3), (3, 0)]
