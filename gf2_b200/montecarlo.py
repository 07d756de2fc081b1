"""Coded FER / BER Monte Carlo driver on the GPU.

The reference's coded error-rate loop is the example
crates/gf2-coding/examples/ldpc_awgn.rs:121-175 (a frame counts as an error
when the decoder does not converge or fails the syndrome, :157) and its
simulation module only runs uncoded BER (SimulationRunner,
crates/gf2-coding/src/simulation.rs:140-193).  Here one point runs batches of
seeded frames (channel kernel -> decoder -> error-count kernel) until a target
number of frame errors or a frame budget is reached.  Two frame-error counts
are kept:
  frame_errors          the decoded message differs from the transmitted one
                        (what a receiver sees: undetected errors included,
                        unconverged frames that happen to be right excluded)
  frame_errors_ref_rule the reference example's rule, a frame that did not
                        converge or failed the syndrome check
                        (!converged || !syndrome_check_passed,
                        examples/ldpc_awgn.rs:156-158)
plus undetected_errors (syndrome satisfied, message wrong).

Multi-GPU: frames are sharded by index (rank r of w decodes global frame
indices b*batch*w + r*batch + i of batch b), there is no exchange during
decoding, and the int64 counters are summed with one all-reduce at the end of
the point.
"""
import math

import numpy as np

from .ldpc import awgn_frames, sigma2_from_ebn0, words


def wilson(k, n, z=1.96):
    """Wilson score interval of a binomial proportion k/n."""
    if n == 0:
        return (0.0, 1.0)
    p = k / n
    den = 1.0 + z * z / n
    c = (p + z * z / (2 * n)) / den
    h = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / den
    return (max(0.0, c - h), min(1.0, c + h))


def shard_frame0(batch_index, batch, rank, world):
    """First global frame index of a rank's batch (disjoint across ranks)."""
    return (batch_index * world + rank) * batch


def reduce_counters(counters, group=None):
    """Sum int64 counters over the process group (no-op without one)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(counters, op=dist.ReduceOp.SUM, group=group)
    return counters


def simulate_point(decoder, code, ebn0_db, max_iter, batch=1024, max_frames=1 << 20, min_frame_errors=100,
                   seed=1, device=None, rank=0, world=1, ebn0_of_frame=None):
    import ctypes

    import torch

    from . import _capi as C
    device = device or torch.device("cuda", torch.cuda.current_device())
    k = code.k()
    totals = torch.zeros(2, dtype=torch.int64, device=device)  # frame errors, bit errors
    ref_rule = torch.zeros(2, dtype=torch.int64, device=device)  # !conv || !synd_ok, undetected
    hist = torch.zeros(max_iter + 1, dtype=torch.int64, device=device)
    frames = 0
    b = 0
    out = None
    st = torch.cuda.current_stream(device)
    while True:
        frame0 = shard_frame0(b, batch, rank, world)
        if ebn0_of_frame is None:
            s2 = sigma2_from_ebn0(ebn0_db, code.rate())
        else:
            s2 = np.array([sigma2_from_ebn0(ebn0_of_frame(frame0 + i), code.rate()) for i in range(batch)])
        info, _, llr = awgn_frames(code, seed, frame0, batch, s2, device=device, want_cw=False)
        out = decoder.decode_tensors(llr, max_iter, out=out)
        C.check(C.lib.gf2c_count_errors(ctypes.c_void_p(info.data_ptr()), ctypes.c_void_p(out["msg"].data_ptr()),
                                        batch, words(k), None, ctypes.c_void_p(totals.data_ptr()),
                                        ctypes.c_void_p(st.cuda_stream)))
        hist += torch.bincount(out["iters"].long().clamp(0, max_iter), minlength=max_iter + 1)
        failed = (out["conv"] == 0) | (out["synd_ok"] == 0)
        wrong = (out["msg"] != info).any(dim=1)
        ref_rule[0] += failed.sum()
        ref_rule[1] += (wrong & (out["synd_ok"] != 0)).sum()
        frames += batch
        b += 1
        fe = int(totals[0].item()) * world  # estimate across ranks without a collective
        if frames * world >= max_frames or fe >= min_frame_errors:
            break
    counters = torch.cat([totals, torch.tensor([frames], dtype=torch.int64, device=device), ref_rule, hist])
    reduce_counters(counters)
    fe, be, nf = int(counters[0]), int(counters[1]), int(counters[2])
    fr, ud = int(counters[3]), int(counters[4])
    h = counters[5:].cpu().numpy()
    lo, hi = wilson(fe, nf)
    return dict(ebn0_db=float(ebn0_db) if ebn0_of_frame is None else None, frames=nf, frame_errors=fe,
                bit_errors=be, fer=fe / nf if nf else 0.0, ber=be / (nf * k) if nf else 0.0, fer_ci=(lo, hi),
                frame_errors_ref_rule=fr, fer_ref_rule=fr / nf if nf else 0.0, fer_ref_rule_ci=wilson(fr, nf),
                undetected_errors=ud,
                mean_iters=float((h * np.arange(len(h))).sum() / max(1, h.sum())), iter_hist=h.tolist())
