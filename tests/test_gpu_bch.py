"""DVB-T2 outer BCH code on the GPU against the CPU oracle, bit for bit:
encoder, syndromes and decoder, with 0..t errors (corrected) and beyond t
(decoding failures, which must fail exactly like the reference's decoder)."""
import numpy as np
import pytest

import gf2_b200 as g

pytestmark = pytest.mark.gpu

CODES = [(f, r) for f in (1, 0) for r in range(6)]


@pytest.mark.parametrize("frame,rate", CODES)
def test_encode_matches_oracle(gpu, oracle, frame, rate):
    b = oracle.Bch(frame, rate)
    code = g.BchCode.dvb_t2(frame, rate)
    rng = np.random.default_rng(100 + 10 * frame + rate)
    msg = rng.integers(0, 2, (6, b.k)).astype(np.uint8)
    msg[0] = 1  # the reference's all-ones roundtrip message
    cw = g.BchEncoder(code).encode_batch(msg)
    assert (cw == b.encode(msg)).all()


@pytest.mark.parametrize("frame,rate", CODES)
def test_decode_matches_oracle(gpu, oracle, frame, rate):
    b = oracle.Bch(frame, rate)
    code = g.BchCode.dvb_t2(frame, rate)
    rng = np.random.default_rng(200 + 10 * frame + rate)
    errs = list(range(0, b.t + 5))  # 0..t corrected, t+1..t+4 beyond the design distance
    msg = rng.integers(0, 2, (len(errs), b.k)).astype(np.uint8)
    cw = b.encode(msg)
    for f, e in enumerate(errs):
        cw[f, rng.choice(b.n, size=e, replace=False)] ^= 1
    dec = g.BchDecoder(code)
    out = dec.decode_words(g.pack_bits(cw, b.n), syndromes=True)
    om, of = b.decode(cw)
    assert (g.unpack_bits(out["msg"], b.k) == om).all()
    assert (out["corrected"] == of).all()
    assert (out["syndromes"] == b.syndromes(cw)).all()
    for f, e in enumerate(errs[:b.t + 1]):
        assert out["corrected"][f] == e and (om[f] == msg[f]).all()


def test_device_path_and_ldpc_chain(gpu, oracle):
    """BCH on the message bits of the LDPC decoder, all on the device:
    info -> BCH encode -> LDPC encode -> AWGN -> LDPC decode -> BCH decode."""
    import torch
    frame, rate = 1, 2
    ldpc = g.LdpcCode.dvb_t2_short(rate)
    bch = g.BchCode.dvb_t2(frame, rate)
    assert bch.n() == ldpc.k()
    rng = np.random.default_rng(3)
    F = 64
    info = rng.integers(0, 2, (F, bch.k())).astype(np.uint8)
    dinfo = torch.from_numpy(g.pack_bits(info, bch.k()).view(np.int64)).to(gpu)
    bcw = g.BchEncoder(bch).encode_words(dinfo)
    torch.cuda.synchronize()
    host = g.BchEncoder(bch).encode_words(g.pack_bits(info, bch.k()))
    assert (bcw.cpu().numpy().view(np.uint64) == host).all()
    ocw = oracle.Code.dvbt2(frame, rate).encode(g.unpack_bits(host, bch.n()))
    llr = np.where(ocw == 1, -6.0, 6.0).astype(np.float32)
    flip = rng.random(llr.shape) < 0.004
    llr[flip] = -llr[flip]
    dec = g.LdpcDecoder(ldpc)
    r = dec.decode_tensors(torch.from_numpy(llr).to(gpu), 30)
    out = g.BchDecoder(bch).decode_words(r["msg"])
    torch.cuda.synchronize()
    assert (g.unpack_bits(out["msg"].cpu().numpy().view(np.uint64), bch.k()) == info).all()
