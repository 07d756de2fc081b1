"""Precision report of the layered sum-product decoders against the FP64 judge.

For each Eb/N0 point of a sweep, one batch of seeded frames (channel kernel:
Philox info bits, encoder, BPSK, AWGN, LLR = 2y/sigma^2) is decoded by

  spa_fast_f16   layered sum-product on the SFU, messages stored in FP16
  spa_fast_f32   the same with FP32 message storage
  spa_exact_f16  layered sum-product with the exact (bit-reproducible) FP32
                 numerics, FP16 message storage
  spa_exact_f32  the same with FP32 message storage
  judge_fp64     layered sum-product in FP64 (gf2c_judge_spa64)

all with the same budget and syndrome early stop.  The reference's own
sum-product (crates/gf2-coding/src/ldpc/core.rs:762-787, llr.rs:210-215) is FP32
and unused there; the reference offers Llr::saturate(max) (llr.rs:117-119)
without a default saturation level, so the report defines one:

  non-saturated   |L_judge| < L_SAT = 16.6355, the largest message magnitude
                  of the FP32 decoders (2 atanh(1 - 2^-23)); beyond it the
                  FP32 decoders clamp where the judge does not.

Reported per point and decoder:
  dev_it1 / dev_it5  max |L - L_judge| over the non-saturated posteriors after
                     1 (and 5) iterations (frames whose iteration counts agree)
  rel_it1            max |L - L_judge| / max(|L_judge|, 1) after 1 iteration
  hd_frames          fraction of frames whose decoded message equals the judge's
  hd_decoded         the same over the frames the judge decodes (converges on);
                     frames no decoder decodes oscillate chaotically, so their
                     decisions are not a precision measure
  hd_bits            fraction of equal message bits
  fer, fer_ci        frames whose message differs from the transmitted bits,
                     with the Wilson 95 % interval
  fer_ref_rule       frames that did not converge (the reference's frame-error
                     rule, crates/gf2-coding/examples/ldpc_awgn.rs:156-158)
  mean_iters

Usage: python -m gf2_b200.precision [--frames 4096] [--json out.json]
"""
import argparse
import json
import sys

import numpy as np

from . import _capi as C
from .ldpc import LdpcCode, LdpcDecoder, awgn_frames, judge_spa64, sigma2_from_ebn0, unpack_bits
from .montecarlo import wilson

L_SAT = 16.635532
DECODERS = [
    ("spa_fast_f16", C.ALGO_SPA_FAST, C.MSG_F16),
    ("spa_fast_f32", C.ALGO_SPA_FAST, C.MSG_F32),
    ("spa_exact_f16", C.ALGO_SPA, C.MSG_F16),
    ("spa_exact_f32", C.ALGO_SPA, C.MSG_F32),
]


def _frame_errors(msg, info):
    """Frames whose packed message words differ (device tensors)."""
    return (msg != info).any(dim=1)


def _dev(bel, ref, mask):
    import torch
    d = (bel.double() - ref).abs()
    d = torch.where(mask, d, torch.zeros_like(d))
    return float(d.max().item()) if d.numel() else 0.0


def precision_point(code, ebn0, frames, seed, point, max_iter=50, decoders=None, device=None):
    import torch
    device = device or torch.device("cuda", torch.cuda.current_device())
    s2 = sigma2_from_ebn0(ebn0, code.rate())
    info, _, llr = awgn_frames(code, seed, point * frames, frames, s2, device=device, want_cw=False)
    k = code.k()
    jfull = judge_spa64(code, llr, max_iter, schedule=C.SCHED_LAYERED)
    j1 = judge_spa64(code, llr, 1, schedule=C.SCHED_LAYERED, beliefs=True)
    j5 = judge_spa64(code, llr, 5, schedule=C.SCHED_LAYERED, beliefs=True)
    out = {}
    jfe = _frame_errors(jfull["msg"], info)
    nj = int(jfe.sum().item())
    out["judge_fp64"] = dict(fer=nj / frames, fer_ci=wilson(nj, frames), frame_errors=nj,
                             fer_ref_rule=float((jfull["conv"] == 0).float().mean().item()),
                             mean_iters=float(jfull["iters"].float().mean().item()))
    mask1 = j1["beliefs"].abs() < L_SAT
    jbits = torch.from_numpy(unpack_bits(jfull["msg"].cpu().numpy().view(np.uint64), k))
    for name, algo, msg in (decoders or DECODERS):
        dec = LdpcDecoder(code, algorithm=algo, schedule=C.SCHED_LAYERED, msg_dtype=msg)
        full = dec.decode_tensors(llr, max_iter)
        one = dec.decode_tensors(llr, 1, beliefs=True)
        d1 = _dev(one["beliefs"], j1["beliefs"], mask1)
        rel1 = float(((one["beliefs"].double() - j1["beliefs"]).abs() /
                      j1["beliefs"].abs().clamp(min=1.0)).masked_fill(~mask1, 0).max().item())
        five = dec.decode_tensors(llr, 5, beliefs=True)
        same5 = (five["iters"] == j5["iters"])[:, None]
        mask5 = (j5["beliefs"].abs() < L_SAT) & same5
        d5 = _dev(five["beliefs"], j5["beliefs"], mask5)
        fe = _frame_errors(full["msg"], info)
        nfe = int(fe.sum().item())
        bits = torch.from_numpy(unpack_bits(full["msg"].cpu().numpy().view(np.uint64), k))
        same = (full["msg"] == jfull["msg"]).all(dim=1)
        jc = jfull["conv"] != 0
        out[name] = dict(dev_it1=d1, rel_it1=rel1, dev_it5=d5,
                         hd_frames=float(same.float().mean().item()),
                         hd_decoded=float(same[jc].float().mean().item()) if bool(jc.any()) else None,
                         judge_decoded=int(jc.sum().item()),
                         hd_bits=float((bits == jbits).float().mean().item()),
                         fer=nfe / frames, fer_ci=wilson(nfe, frames), frame_errors=nfe,
                         fer_ref_rule=float((full["conv"] == 0).float().mean().item()),
                         mean_iters=float(full["iters"].float().mean().item()))
        del dec, full, one, five
    torch.cuda.synchronize()
    return out


def sweep(code, points, frames, seed=11, max_iter=50, log=None):
    rows = []
    for p, eb in enumerate(points):
        r = precision_point(code, eb, frames, seed, p, max_iter)
        rows.append(dict(ebn0_db=eb, frames=frames, **{k: v for k, v in r.items()}))
        if log:
            log(format_row(eb, r))
    return rows


def format_row(eb, r):
    parts = [f"{eb:.1f} dB judge FER {r['judge_fp64']['fer']:.4f}"]
    for name, _, _ in DECODERS:
        x = r[name]
        hd = "-" if x["hd_decoded"] is None else f"{x['hd_decoded']:.4f}"
        parts.append(f"{name}: dev1 {x['dev_it1']:.2e} dev5 {x['dev_it5']:.2e} hd {x['hd_frames']:.4f} "
                     f"hd(decoded) {hd} FER {x['fer']:.4f}")
    return " | ".join(parts)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=4096)
    ap.add_argument("--max-iter", type=int, default=50)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--points", default="0.6,0.7,0.8,0.9,1.0,1.1,1.2,1.3,1.4")
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    code = LdpcCode.dvb_t2_normal(1)  # normal 3/5: n 64800, k 38880
    pts = [float(x) for x in a.points.split(",")]
    rows = sweep(code, pts, a.frames, a.seed, a.max_iter, log=lambda s: print(s, flush=True))
    res = dict(code="dvbt2-normal-3/5", schedule="layered", max_iter=a.max_iter, frames_per_point=a.frames,
               seed=a.seed, l_sat=L_SAT, rows=rows)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
