"""The FER / BER Monte Carlo driver against a host recount and the oracle.

simulate_point runs channel kernel -> decoder -> error-count kernel per batch
and accumulates counters on the device.  Here the same seeded frames are
regenerated batch by batch (same frame indices), decoded by the CPU oracle
(the reference decoder's restatement: min-sum, bit-identical results), and
the frame errors, bit errors, the reference example's frame-error rule
(!converged || !syndrome_check_passed, examples/ldpc_awgn.rs:156-158),
undetected errors and the iteration histogram are recounted on the host.
"""
import numpy as np
import pytest

import gf2_b200 as g
from gf2_b200.montecarlo import shard_frame0, simulate_point

pytestmark = pytest.mark.gpu


def host_recount(code, ocode, ebn0, max_iter, batch, nbatches, seed, decode):
    k = code.k()
    tot = dict(fe=0, be=0, fr=0, ud=0, frames=0, hist=np.zeros(max_iter + 1, np.int64))
    s2 = g.sigma2_from_ebn0(ebn0, code.rate())
    for b in range(nbatches):
        info, _, llr = g.awgn_frames(code, seed, shard_frame0(b, batch, 0, 1), batch, s2)
        r = decode(llr)
        bits = r["msg_bits"]
        ref = g.unpack_bits(info.view(np.uint64), k)
        wrong = (bits != ref)
        tot["fe"] += int(wrong.any(axis=1).sum())
        tot["be"] += int(wrong.sum())
        failed = ~(r["conv"] & r["synd_ok"])
        tot["fr"] += int(failed.sum())
        tot["ud"] += int((wrong.any(axis=1) & r["synd_ok"]).sum())
        tot["frames"] += batch
        tot["hist"] += np.bincount(r["iters"], minlength=max_iter + 1)
    return tot


@pytest.mark.parametrize("ebn0", [1.1, 1.6])
def test_simulate_point_equals_oracle_recount(gpu, oracle, ebn0):
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    ocode = oracle.Code.dvbt2(1, 0)
    batch, nb, max_iter = 96, 3, 30
    res = simulate_point(g.LdpcDecoder(code), code, ebn0, max_iter, batch=batch, max_frames=batch * nb,
                         min_frame_errors=10 ** 9, seed=5, device=gpu)

    def dec(llr):
        r = ocode.decode(llr, max_iter)
        return dict(msg_bits=r["msg"], conv=r["conv"], synd_ok=r["synd_ok"], iters=r["iters"])
    t = host_recount(code, ocode, ebn0, max_iter, batch, nb, 5, dec)
    assert res["frames"] == t["frames"] == batch * nb
    assert res["frame_errors"] == t["fe"]
    assert res["bit_errors"] == t["be"]
    assert res["frame_errors_ref_rule"] == t["fr"]
    assert res["undetected_errors"] == t["ud"]
    assert res["iter_hist"] == t["hist"].tolist()
    if ebn0 < 1.5:
        assert t["fr"] > 0  # the point exercises both rules


def test_simulate_point_sum_product_host_recount(gpu):
    """A decoder that is not bit-exact against the oracle: recount the GPU's own
    decisions on the host."""
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    kw = dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    batch, nb, max_iter = 128, 2, 20
    res = simulate_point(g.LdpcDecoder(code, **kw), code, 0.9, max_iter, batch=batch, max_frames=batch * nb,
                         min_frame_errors=10 ** 9, seed=9, device=gpu)
    d = g.LdpcDecoder(code, **kw)

    def dec(llr):
        r = d.decode_arrays(llr, max_iter)
        return dict(msg_bits=g.unpack_bits(r["msg"], code.k()), conv=r["conv"], synd_ok=r["synd_ok"],
                    iters=r["iters"])
    t = host_recount(code, None, 0.9, max_iter, batch, nb, 9, dec)
    assert (res["frame_errors"], res["bit_errors"], res["frame_errors_ref_rule"], res["undetected_errors"]) == \
        (t["fe"], t["be"], t["fr"], t["ud"])
    lo, hi = res["fer_ci"]
    assert lo <= res["fer"] <= hi
