"""GPU tests of the learned normalised / offset min-sum decoder: the training
kernels' gradients against the FP64 oracle, the training forward against the
inference decoder, the gain of the trained weights over the method without
them, and checkpoint / resume."""
import numpy as np
import pytest

import gf2_b200 as g

pytestmark = pytest.mark.gpu


def _batch(oracle, idx, frames, ebn0, seed, device):
    import torch
    oc = oracle.Code.dvbt2(idx // 6, idx % 6)
    _, cw, llr = oc.channel(seed, 0, frames, ebn0)
    cwp = g.pack_bits(cw, oc.n).view(np.int64)
    return oc, cw, llr, torch.from_numpy(llr).to(device), torch.from_numpy(cwp).to(device)


def test_gradient_matches_fp64_oracle(gpu, oracle):
    from gf2_b200.learned import NmsTrainer
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate5_6)
    T = 4
    tr = NmsTrainer(code, iterations=T, batch=4, device=gpu)
    rng = np.random.default_rng(3)
    a = (0.7 + 0.3 * rng.random((T, tr.L))).astype(np.float32)
    b = (0.3 * rng.random((T, tr.L))).astype(np.float32)
    import torch
    tr.P[0].copy_(torch.from_numpy(a))
    tr.P[1].copy_(torch.from_numpy(b))
    oc, cw, llr, tl, tc = _batch(oracle, 11, 4, 3.0, 5, gpu)
    loss, G = tr.loss_grad(tl, tc)
    torch.cuda.synchronize()
    l64, ga, gb, _ = oc.nms_loss_grad(llr, cw, T, a.astype(np.float64).ravel(), b.astype(np.float64).ravel())
    assert abs(float(loss.item()) - l64) <= 1e-4 * abs(l64)
    for got, ref in ((G[0].cpu().numpy().ravel(), ga), (G[1].cpu().numpy().ravel(), gb)):
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 2e-3 * scale, (np.abs(got - ref).max(), scale)
        cos = float(got @ ref / (np.linalg.norm(got) * np.linalg.norm(ref)))
        assert cos > 0.9999


def test_training_forward_equals_inference_decoder(gpu, oracle):
    """The unrolled forward of the trainer and the NMS decoder (same weights,
    no early stop, T iterations) produce bit-identical soft outputs."""
    import ctypes

    import torch

    from gf2_b200 import _capi as C
    from gf2_b200.learned import NmsTrainer
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    T = 6
    tr = NmsTrainer(code, iterations=T, batch=8, device=gpu)
    rng = np.random.default_rng(4)
    a = (0.6 + 0.4 * rng.random((T, tr.L))).astype(np.float32)
    b = (0.4 * rng.random((T, tr.L))).astype(np.float32)
    tr.P[0].copy_(torch.from_numpy(a))
    tr.P[1].copy_(torch.from_numpy(b))
    _, _, llr, tl, tc = _batch(oracle, 6, 8, 1.5, 6, gpu)
    soft = torch.empty_like(tl)
    C.check(C.lib.gf2c_nms_loss_grad(tr._h, ctypes.c_void_p(tl.data_ptr()), ctypes.c_void_p(tc.data_ptr()), 8,
                                     ctypes.c_void_p(tr.P[0].data_ptr()), ctypes.c_void_p(tr.P[1].data_ptr()),
                                     ctypes.c_void_p(tr.G[0].data_ptr()), ctypes.c_void_p(tr.G[1].data_ptr()),
                                     ctypes.c_void_p(tr.loss_buf.data_ptr()), ctypes.c_void_p(soft.data_ptr()),
                                     None))
    torch.cuda.synchronize()
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, nms_alpha=a, nms_beta=b, early_stop=False)
    r = dec.decode_arrays(llr, T, beliefs=True)
    assert (r["beliefs"].view(np.uint32) == soft.cpu().numpy().view(np.uint32)).all()


def test_trained_weights_beat_plain_min_sum(gpu):
    """What the trained network gains over the same decoder without it: FER of
    the learned decoder vs plain min-sum (alpha = 1, beta = 0) with the same
    iteration budget on fresh frames."""
    from gf2_b200.learned import NmsTrainer
    from gf2_b200.montecarlo import simulate_point
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    T = 10
    tr = NmsTrainer(code, iterations=T, batch=256, ebn0_range=(2.0, 3.0), lr=1e-2, seed=11, device=gpu,
                    alpha0=1.0, beta0=0.0)
    first = tr.train_step()
    tr.train(200)
    last = tr.train_step()
    assert last < first, (first, last)
    learned = tr.decoder()
    plain = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, nms_alpha=np.ones((1, tr.L), np.float32),
                          nms_beta=np.zeros((1, tr.L), np.float32))
    kw = dict(batch=2048, max_frames=8192, min_frame_errors=10 ** 9, seed=999, device=gpu)
    p_l = simulate_point(learned, code, 2.4, T, **kw)
    p_p = simulate_point(plain, code, 2.4, T, **kw)
    # at 2.4 dB plain min-sum fails ~30% of frames in 10 iterations; the learned weights about half as many
    assert p_l["frame_errors"] < 0.75 * p_p["frame_errors"], (p_l["fer"], p_p["fer"])


def test_checkpoint_resume(gpu, tmp_path):
    from gf2_b200.learned import NmsTrainer
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate3_4)
    a = NmsTrainer(code, iterations=5, batch=32, device=gpu, seed=7)
    a.train(4)
    path = str(tmp_path / "ck.npz")
    a.save(path)
    a.train(4)
    b = NmsTrainer(code, iterations=5, batch=32, device=gpu, seed=0)
    b.load(path)
    assert b.step_no == 4 and b.frame_counter == 4 * 32
    b.train(4)
    wa, wb = a.weights(), b.weights()
    assert np.allclose(wa[0], wb[0], atol=1e-5) and np.allclose(wa[1], wb[1], atol=1e-5)


def _set_weights(tr, a, b):
    import torch
    tr.P[0].copy_(torch.from_numpy(a))
    tr.P[1].copy_(torch.from_numpy(b))


@pytest.mark.parametrize("idx,frames,ebn0", [(11, 4, 3.0), (6, 4, 1.6), (5, 2, 3.3)])
def test_layered_gradient_matches_fp64_oracle(gpu, oracle, idx, frames, ebn0):
    """Layered schedule (normal 5/6: up to 4 circulants of one block in a row
    group, so repeated variables inside a layer)."""
    import torch

    from gf2_b200.learned import NmsTrainer
    code = g.LdpcCode.dvb_t2_normal(idx) if idx < 6 else g.LdpcCode.dvb_t2_short(idx - 6)
    T = 3
    tr = NmsTrainer(code, iterations=T, batch=frames, device=gpu, schedule=g.SCHED_LAYERED)
    rng = np.random.default_rng(7)
    a = (0.7 + 0.3 * rng.random((T, tr.L))).astype(np.float32)
    b = (0.3 * rng.random((T, tr.L))).astype(np.float32)
    _set_weights(tr, a, b)
    oc, cw, llr, tl, tc = _batch(oracle, idx, frames, ebn0, 8, gpu)
    loss, G = tr.loss_grad(tl, tc)
    torch.cuda.synchronize()
    l64, ga, gb, _ = oc.nms_loss_grad(llr, cw, T, a.astype(np.float64).ravel(), b.astype(np.float64).ravel(),
                                      layered=True)
    assert abs(float(loss.item()) - l64) <= 1e-4 * abs(l64)
    for got, ref in ((G[0].cpu().numpy().ravel(), ga), (G[1].cpu().numpy().ravel(), gb)):
        scale = np.abs(ref).max()
        assert scale > 0
        assert np.abs(got - ref).max() <= 2e-3 * scale, (np.abs(got - ref).max(), scale)
        cos = float(got @ ref / (np.linalg.norm(got) * np.linalg.norm(ref)))
        assert cos > 0.9999


@pytest.mark.parametrize("idx", [6, 1])
def test_layered_training_forward_equals_inference_decoder(gpu, oracle, idx):
    """The layered training forward and the layered NMS decoder (same weights,
    FP32 messages, no early stop) give bit-identical posteriors; normal 3/5 has
    row groups with repeated variables."""
    import ctypes

    import torch

    from gf2_b200 import _capi as C
    from gf2_b200.learned import NmsTrainer
    code = g.LdpcCode.dvb_t2_normal(idx) if idx < 6 else g.LdpcCode.dvb_t2_short(idx - 6)
    T, F = 5, 3
    tr = NmsTrainer(code, iterations=T, batch=F, device=gpu, schedule=g.SCHED_LAYERED)
    rng = np.random.default_rng(9)
    a = (0.6 + 0.4 * rng.random((T, tr.L))).astype(np.float32)
    b = (0.4 * rng.random((T, tr.L))).astype(np.float32)
    _set_weights(tr, a, b)
    _, _, llr, tl, tc = _batch(oracle, idx, F, 1.4 if idx < 6 else 1.6, 10, gpu)
    soft = torch.empty_like(tl)
    C.check(C.lib.gf2c_nms_loss_grad(tr._h, ctypes.c_void_p(tl.data_ptr()), ctypes.c_void_p(tc.data_ptr()), F,
                                     ctypes.c_void_p(tr.P[0].data_ptr()), ctypes.c_void_p(tr.P[1].data_ptr()),
                                     ctypes.c_void_p(tr.G[0].data_ptr()), ctypes.c_void_p(tr.G[1].data_ptr()),
                                     ctypes.c_void_p(tr.loss_buf.data_ptr()), ctypes.c_void_p(soft.data_ptr()),
                                     None))
    torch.cuda.synchronize()
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, nms_alpha=a, nms_beta=b,
                        early_stop=False)
    r = dec.decode_arrays(llr, T, beliefs=True)
    assert (r["beliefs"].view(np.uint32) == soft.cpu().numpy().view(np.uint32)).all()


def test_layered_trained_weights_beat_plain_min_sum(gpu):
    """The gain of the trained layered network over layered plain min-sum
    (alpha = 1, beta = 0) at the same 10-iteration budget, on fresh frames."""
    from gf2_b200.learned import NmsTrainer
    from gf2_b200.montecarlo import simulate_point
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    T = 10
    tr = NmsTrainer(code, iterations=T, batch=256, ebn0_range=(1.4, 2.6), lr=1e-2, seed=12, device=gpu,
                    alpha0=1.0, beta0=0.0, schedule=g.SCHED_LAYERED)
    first = tr.train_step()
    tr.train(200)
    last = tr.train_step()
    assert last < first, (first, last)
    learned = tr.decoder()
    plain = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED,
                          nms_alpha=np.ones((1, tr.L), np.float32), nms_beta=np.zeros((1, tr.L), np.float32))
    kw = dict(batch=2048, max_frames=4096, min_frame_errors=10 ** 9, seed=998, device=gpu)
    fl = sum(simulate_point(learned, code, eb, T, **kw)["frame_errors"] for eb in (1.8, 2.0, 2.2))
    fp = sum(simulate_point(plain, code, eb, T, **kw)["frame_errors"] for eb in (1.8, 2.0, 2.2))
    assert fp > 50 and fl < 0.8 * fp, (fl, fp)
