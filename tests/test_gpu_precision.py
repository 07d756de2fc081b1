"""Precision of the FP32 / FP16 sum-product decoders against the FP64 judge.

Config 1 (short 1/2, 256 frames, 1.0 dB, flooding, exact FP32 sum-product):
every frame the FP64 judge decodes is decoded to the same message; the frame
error counts agree; the one-iteration posteriors agree within 1e-4 relative
where neither side is near the FP32 message clamp.

Config 2 (normal 3/5, layered, FP16 / FP32 message storage, exact and SFU
sum-product): one Eb/N0 point of the 0.6..1.4 dB sweep at 1024 frames through
gf2_b200.precision (the full sweep is `python -m gf2_b200.precision`):
decisions equal to the judge's on the frames it decodes, FER within the
judge's Wilson interval, bounded one- and five-iteration deviations.  A frame
that no decoder decodes oscillates chaotically, so decision agreement is
measured on the frames the judge decodes.
"""
import numpy as np
import pytest
import torch

import gf2_b200 as g
from gf2_b200 import precision

pytestmark = pytest.mark.gpu


def test_config1_fp32_sum_product_matches_fp64_judge(gpu):
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    s2 = g.sigma2_from_ebn0(1.0, code.rate())
    info, _, llr = g.awgn_frames(code, 1, 0, 256, s2, device=gpu, want_cw=False)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_SPA, schedule=g.SCHED_FLOODING)
    r = dec.decode_tensors(llr, 50)
    j = g.judge_spa64(code, llr, 50, schedule=g.SCHED_FLOODING)
    jc = j["conv"].bool()
    assert int(jc.sum()) > 64
    assert torch.equal(r["msg"][jc], j["msg"][jc]), "decisions differ on frames the judge decodes"
    assert torch.equal(r["conv"].bool()[jc], jc[jc])
    fe = int((r["msg"] != info).any(dim=1).sum())
    fej = int((j["msg"] != info).any(dim=1).sum())
    assert abs(fe - fej) <= 2, (fe, fej)
    r1 = dec.decode_tensors(llr, 1, beliefs=True)
    j1 = g.judge_spa64(code, llr, 1, schedule=g.SCHED_FLOODING, beliefs=True)
    L = j1["beliefs"]
    mask = L.abs() < 8.0
    rel = ((r1["beliefs"].double() - L).abs() / L.abs().clamp(min=1.0))[mask]
    assert float(rel.max()) <= 1e-4, float(rel.max())


def test_config2_precision_point(gpu):
    code = g.LdpcCode.dvb_t2_normal(g.CodeRate.Rate3_5)
    r = precision.precision_point(code, 1.2, 1024, seed=11, point=4)
    jf = r["judge_fp64"]
    lo, hi = jf["fer_ci"]
    for name, _, _ in precision.DECODERS:
        x = r[name]
        assert x["hd_bits"] > 0.999, (name, x)
        assert x["judge_decoded"] > 500 and x["hd_decoded"] >= 0.995, (name, x)
        assert lo <= x["fer"] <= hi, (name, x, jf)
    # one- and five-iteration posterior deviations (measured on this point:
    # FP32 storage ~2e-5 / 1.5e-4, FP16 storage ~3e-3 / 9e-3)
    for name in ("spa_exact_f32", "spa_fast_f32"):
        assert r[name]["dev_it1"] < 2e-4 and r[name]["dev_it5"] < 2e-3, r[name]
    for name in ("spa_exact_f16", "spa_fast_f16"):
        assert r[name]["dev_it1"] < 1e-2 and r[name]["dev_it5"] < 5e-2, r[name]
