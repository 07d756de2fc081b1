"""Encoding with a dense parity part on the GPU (the encoder-cache path) against
the library's own encoders, which the oracle pins: the codewords must be
identical bit for bit."""
import numpy as np
import pytest

import gf2_b200 as g
from gf2_b200 import gf2io

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("frame,rate,frames", [(1, 0, 100), (1, 5, 3), (0, 1, 130)])
def test_dense_encoder_matches_encoder(gpu, frame, rate, frames):
    import torch
    code = g.LdpcCode.dvb_t2_normal(rate) if frame == 0 else g.LdpcCode.dvb_t2_short(rate)
    enc = g.LdpcEncoder(code)
    dense = gf2io.DenseEncoder(gf2io.parity_part(code), code.k(), code.n())
    rng = np.random.default_rng(frame * 10 + rate)
    msg = rng.integers(0, 2, (frames, code.k())).astype(np.uint8)
    mw = g.pack_bits(msg, code.k())
    want = enc.encode_packed(mw)
    assert (dense.encode_words(mw) == want).all()
    dev = torch.from_numpy(mw.view(np.int64)).to(gpu)
    got = dense.encode_words(dev)
    torch.cuda.synchronize()
    assert (got.cpu().numpy().view(np.uint64) == want).all()


def test_dense_encoder_qc_and_cache_directory(gpu, tmp_path):
    base = [[1, 2, 0, 0, -1, -1], [0, -1, 3, 0, 0, -1], [2, 1, -1, -1, 0, 0]]
    qc_code = g.LdpcCode.from_quasi_cyclic(g.QuasiCyclicLdpc(np.array(base), 100))
    dvb = g.LdpcCode.dvb_t2_short(2)
    cache = g.EncodingCache()
    for c in (qc_code, dvb):
        cache.get_or_compute(c)
    cache.save_to_directory(tmp_path)
    loaded = g.EncodingCache.from_directory(tmp_path)
    rng = np.random.default_rng(9)
    for c in (qc_code, dvb):
        msg = rng.integers(0, 2, (65, c.k())).astype(np.uint8)
        cw = loaded.encoder(c).encode_batch(msg)
        assert (cw == g.unpack_bits(g.LdpcEncoder(c).encode_packed(g.pack_bits(msg, c.k())), c.n())).all()
