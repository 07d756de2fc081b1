"""The GPU FP64 sum-product judge (gf2c_judge_spa64) against the CPU oracle's
FP64 sum-product on the same seeded LLRs.

Both evaluate 2 atanh(prod tanh(x/2)) in FP64 with the same product order and
clamp, with different tanh / atanh implementations (CUDA's and the host
libm's, each within a few ulp).  Bars: one-iteration posteriors within
1e-9 relative; after a full decode, the same iteration count, flags and
decisions on every frame, posteriors within 1e-6 relative.
"""
import numpy as np
import pytest
import torch

import gf2_b200 as g

pytestmark = pytest.mark.gpu


def dvb(idx):
    return g.LdpcCode.dvb_t2_normal(idx) if idx < 6 else g.LdpcCode.dvb_t2_short(idx - 6)


def run_judge(code, llr, max_iter, sched):
    t = torch.from_numpy(llr).cuda()
    r = g.judge_spa64(code, t, max_iter, schedule=sched, beliefs=True)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in r.items()}


@pytest.mark.parametrize("idx,sched,frames,ebn0", [(6, 1, 24, 1.0), (6, 0, 24, 1.0), (1, 1, 4, 1.2),
                                                   (5, 1, 3, 3.3), (9, 1, 12, 2.2)])
def test_judge_matches_cpu_fp64(gpu, oracle, idx, sched, frames, ebn0):
    """Normal 3/5 and 5/6 hold row groups with 3 and 4 circulants in one block
    (repeated variables in a layer)."""
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    _, _, llr = ocode.channel(31, 0, frames, ebn0)
    for it in (1, 2):
        r = run_judge(code, llr, it, sched)
        ref = ocode.decode_spa64(llr, it, sched=sched)
        assert (r["iters"] == ref["iters"]).all()
        dev = np.abs(r["beliefs"] - ref["beliefs"])
        assert (dev <= 1e-9 * np.maximum(np.abs(ref["beliefs"]), 1.0)).all(), dev.max()
    # Full decodes: a frame that converges does so at the same iteration with the
    # same decisions.  Frames that never converge keep oscillating for all 50
    # iterations, where ulp-level differences of the two tanh / atanh libraries
    # are amplified, so only their flags are compared.
    r = run_judge(code, llr, 50, sched)
    ref = ocode.decode_spa64(llr, 50, sched=sched)
    assert (r["conv"].astype(bool) == ref["conv"]).all()
    assert (r["synd_ok"].astype(bool) == ref["synd_ok"]).all()
    c = ref["conv"]
    assert (r["iters"][c] == ref["iters"][c]).all(), (r["iters"], ref["iters"])
    assert (r["iters"][~c] == 50).all()
    assert (g.unpack_bits(r["msg"].view(np.uint64), code.k())[c] == ref["msg"][c]).all()
    dev = np.abs(r["beliefs"][c] - ref["beliefs"][c])
    assert (dev <= 1e-6 * np.maximum(np.abs(ref["beliefs"][c]), 1.0)).all(), dev.max()


def test_judge_edge_cases(gpu, oracle):
    code = dvb(6)
    ocode = oracle.Code.dvbt2(1, 0)
    _, _, llr = ocode.channel(5, 0, 2, 1.0)
    r = run_judge(code, llr, 0, 1)
    assert (r["iters"] == 0).all() and (r["msg"] == 0).all() and (r["conv"] == 0).all()
    assert (r["synd_ok"] == 1).all() and (r["beliefs"] == 0).all()
    # zero frames: no-op; codes without the row-group plan: unsupported
    g.judge_spa64(code, torch.zeros((0, code.n()), dtype=torch.float32, device="cuda"), 5)
    edges = g.LdpcCode.from_edges(3, 6, [(0, 0), (0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (2, 5), (2, 0)])
    with pytest.raises(g.Gf2cError):
        g.judge_spa64(edges, torch.zeros((1, 6), dtype=torch.float32, device="cuda"), 5)
    # error-free +10 frames converge after one iteration with the zero word
    ones = np.full((3, code.n()), 10.0, np.float32)
    r = run_judge(code, ones, 50, 1)
    assert (r["iters"] == 1).all() and (r["conv"] == 1).all() and (r["msg"] == 0).all()
