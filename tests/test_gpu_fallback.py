"""The device-side fallback path (gf2c_decode_batch_fallback): a learned-style
normalised min-sum decoder with 10 layered iterations on every frame, then
layered sum-product on the frames whose syndrome still fails -- the same
results as running the two decoders separately and merging on the host."""
import numpy as np
import pytest
import torch

import gf2_b200 as g

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ebn0", [2.1, 2.3])
def test_fallback_equals_two_separate_passes(gpu, ebn0):
    code = g.LdpcCode.dvb_t2_normal(g.CodeRate.Rate2_3)
    L, T = code.layers(), 10
    prim = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16,
                         nms_alpha=np.full((T, L), 0.8, np.float32), nms_beta=np.zeros((T, L), np.float32))
    fb = g.LdpcDecoder(code, algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    F = 600
    info, _, llr = g.awgn_frames(code, 41, 0, F, g.sigma2_from_ebn0(ebn0, code.rate()), device=gpu,
                                 want_cw=False)
    out = prim.decode_with_fallback(fb, llr, T, 50)
    torch.cuda.synchronize()
    p = prim.decode_tensors(llr, T)
    failed = torch.nonzero(p["synd_ok"] == 0).flatten()
    assert int(out["fallback_count"][0]) == failed.numel()
    if ebn0 < 2.2:
        assert failed.numel() > 5
    ok = p["synd_ok"] != 0
    assert torch.equal(out["msg"][ok], p["msg"][ok]) and torch.equal(out["iters"][ok], p["iters"][ok])
    if failed.numel():
        r = fb.decode_tensors(llr.index_select(0, failed), 50)
        assert torch.equal(out["msg"][failed], r["msg"])
        assert torch.equal(out["iters"][failed], r["iters"] + T)
        assert torch.equal(out["conv"][failed], r["conv"]) and torch.equal(out["synd_ok"][failed], r["synd_ok"])
    fe = int((out["msg"] != info).any(dim=1).sum())
    fe_p = int((p["msg"] != info).any(dim=1).sum())
    assert fe <= fe_p
    # a repeated call reuses the output buffers and gives the same results
    out2 = prim.decode_with_fallback(fb, llr, T, 50)
    assert torch.equal(out2["msg"], out["msg"]) and torch.equal(out2["iters"], out["iters"])


def test_fallback_argument_checks(gpu):
    a = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    b = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate3_5)
    da = g.LdpcDecoder(a, algorithm=g.ALGO_MINSUM, schedule=g.SCHED_LAYERED)
    db = g.LdpcDecoder(b, algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED)
    flood = g.LdpcDecoder(a)
    llr = torch.zeros((2, a.n()), dtype=torch.float32, device=gpu)
    with pytest.raises(g.Gf2cError):
        da.decode_with_fallback(db, llr, 5, 10)  # different codes
    with pytest.raises(g.Gf2cError):
        da.decode_with_fallback(flood, llr, 5, 10)  # fallback not layered


@pytest.mark.parametrize("frames", [40, 1000, 2800])
def test_fallback_host_memory_equals_device(gpu, frames):
    """The host-memory call gives the device call's results and count: 40
    frames in one piece; 1000 normal frames in three chunks on two streams,
    one fallback pass per chunk; 2800 in nine chunks whose fallback passes
    run per group of two chunks on the fallback stream."""
    code = g.LdpcCode.dvb_t2_normal(g.CodeRate.Rate2_3)
    L, T = code.layers(), 10
    prim = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16,
                         nms_alpha=np.full((T, L), 0.8, np.float32), nms_beta=np.zeros((T, L), np.float32))
    fb = g.LdpcDecoder(code, algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    s2 = np.array([g.sigma2_from_ebn0(2.0 + 0.1 * (f % 4), code.rate()) for f in range(frames)])
    _, _, llr = g.awgn_frames(code, 43, 0, frames, s2, device=gpu, want_info=False, want_cw=False)
    d = prim.decode_with_fallback(fb, llr, T, 50)
    torch.cuda.synchronize()
    assert int(d["fallback_count"][0]) > 0
    h_llr = llr.cpu().pin_memory()
    h = prim.decode_with_fallback(fb, h_llr, T, 50)
    assert h["fallback_count"] == int(d["fallback_count"][0])
    for k in ("msg", "iters", "conv", "synd_ok"):
        assert not h[k].is_cuda
        assert torch.equal(h[k], d[k].cpu()), k
    # numpy in, numpy out (pageable memory)
    hn = prim.decode_with_fallback(fb, llr.cpu().numpy(), T, 50)
    assert isinstance(hn["msg"], np.ndarray) and hn["fallback_count"] == h["fallback_count"]
    assert (hn["msg"] == d["msg"].cpu().numpy()).all() and (hn["iters"] == d["iters"].cpu().numpy()).all()


def test_fallback_same_decoder_host_pipeline(gpu):
    """One layered decoder as both the primary (8 iterations) and the fallback:
    on host memory each chunk's two passes stay on that chunk's stream and
    workspace (2800 normal frames, nine chunks on two streams); the results
    and the count equal the device call's."""
    code = g.LdpcCode.dvb_t2_normal(g.CodeRate.Rate2_3)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    F = 2800
    s2 = np.array([g.sigma2_from_ebn0(2.0 + 0.2 * (f % 6), code.rate()) for f in range(F)])
    _, _, llr = g.awgn_frames(code, 44, 0, F, s2, device=gpu, want_info=False, want_cw=False)
    d = dec.decode_with_fallback(dec, llr, 8, 50)
    torch.cuda.synchronize()
    assert 0 < int(d["fallback_count"][0]) < F
    h = dec.decode_with_fallback(dec, llr.cpu().pin_memory(), 8, 50)
    assert h["fallback_count"] == int(d["fallback_count"][0])
    for k in ("msg", "iters", "conv", "synd_ok"):
        assert torch.equal(h[k], d[k].cpu()), k
