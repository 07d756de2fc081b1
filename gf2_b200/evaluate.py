"""Learned normalised / offset min-sum against plain sum-product: FER / BER
per Eb/N0 point and decoded throughput on one GPU.

    python -m gf2_b200.evaluate --frame normal --rate 1/2 --iters 10 --schedule layered \\
        --train-frames 1048576 --points 0.6:1.4:0.1 --max-frames 262144 --out result.json

Training: NmsTrainer (frames made by the channel kernel with Eb/N0 uniform in
the training range, Adam on the binary cross-entropy of the soft output), or
weights loaded with --weights (saved by --save-weights).
Evaluation: fresh seeded frames (a seed different from training) decoded by
  learned      the trained decoder, T iterations of its schedule, early stop;
  learned_fb   the same, then layered sum-product (FP16 messages, 50
               iterations) on the frames whose syndrome still fails, on the
               device (gf2c_decode_batch_fallback);
  minsum       plain min-sum with the same T and schedule (the method
               without the weights);
  spa50        50-iteration flooding sum-product in FP32 (the judge);
  spa50_layered  50-iteration layered sum-product (SFU, FP16 messages): the
               fastest plain BP decoder of the library.
--decoders selects a subset.  Each point stops after max_frames frames or
min_frame_errors frame errors.
The Eb/N0 at which a decoder reaches the target FER is interpolated (log FER
linear in Eb/N0 between the bracketing points), and the throughput (decoded
info Gbit/s, CUDA events, LLRs resident) of each decoder is measured on one
batch at the Eb/N0 where sum-product reaches the target.
"""
import argparse
import json
import math
import time

import numpy as np

from . import _capi as C
from .ldpc import CodeRate, LdpcCode, LdpcDecoder, awgn_frames, sigma2_from_ebn0
from .learned import NmsTrainer
from .montecarlo import simulate_point

RATES = {"1/2": CodeRate.Rate1_2, "3/5": CodeRate.Rate3_5, "2/3": CodeRate.Rate2_3, "3/4": CodeRate.Rate3_4,
         "4/5": CodeRate.Rate4_5, "5/6": CodeRate.Rate5_6}


def crossing(points, target):
    """Eb/N0 where FER falls to `target` (log-linear interpolation), or None."""
    pts = sorted((p["ebn0_db"], p["fer"]) for p in points)
    for (e0, f0), (e1, f1) in zip(pts, pts[1:]):
        if f0 >= target >= f1 and f0 > 0:
            if f1 <= 0:
                return e1
            return e0 + (math.log(f0) - math.log(target)) / (math.log(f0) - math.log(f1)) * (e1 - e0)
    return None


def throughput(decoder, code, ebn0, max_iter, frames, device, reps=3):
    import torch
    s2 = sigma2_from_ebn0(ebn0, code.rate())
    _, _, llr = awgn_frames(code, 99, 1 << 40, frames, s2, device=device, want_info=False, want_cw=False)
    out = decoder.decode_tensors(llr, max_iter)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = decoder.decode_tensors(llr, max_iter, out=out)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    t = float(np.median(ts))
    return dict(gbit_s=frames * code.k() / t / 1e9, ms=t * 1e3, frames=frames,
                mean_iters=float(out["iters"].float().mean().item()))


class FallbackDecoder:
    """decode_tensors() of a primary decoder with a device-side fallback
    decoder for the frames whose syndrome still fails (simulate_point's
    decoder interface)."""

    def __init__(self, primary, fallback, fallback_iters=50):
        self.primary, self.fallback, self.fallback_iters = primary, fallback, fallback_iters
        self.fallback_frames = 0

    def decode_tensors(self, llr, max_iter, out=None):
        out = self.primary.decode_with_fallback(self.fallback, llr, max_iter, self.fallback_iters, out=out)
        return out


def main(argv=None):
    import torch
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--frame", default="normal", choices=["normal", "short"])
    p.add_argument("--rate", default="1/2", choices=sorted(RATES))
    p.add_argument("--iters", type=int, default=10, help="unrolled / decoding iterations of the learned decoder")
    p.add_argument("--train-frames", type=int, default=1 << 20)
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--train-ebn0", default="0.5:1.5")
    p.add_argument("--lr", type=float, default=1e-2)
    p.add_argument("--points", default="0.6:1.4:0.1", help="start:stop:step Eb/N0 in dB (stop inclusive)")
    p.add_argument("--max-frames", type=int, default=1 << 18)
    p.add_argument("--min-frame-errors", type=int, default=200)
    p.add_argument("--eval-batch", type=int, default=2048)
    p.add_argument("--target-fer", type=float, default=1e-3)
    p.add_argument("--spa-iters", type=int, default=50)
    p.add_argument("--throughput-frames", type=int, default=4096)
    p.add_argument("--schedule", default="flooding", choices=["flooding", "layered"])
    p.add_argument("--msg16", action="store_true", help="FP16 message storage for the min-sum decoders")
    p.add_argument("--decoders", default="learned,minsum,spa50")
    p.add_argument("--weights", default=None, help="load trained weights (npz) instead of training")
    p.add_argument("--save-weights", default=None)
    p.add_argument("--throughput-ebn0", default=None, help="Eb/N0 (comma list) of the throughput measurements")
    p.add_argument("--out", default=None)
    a = p.parse_args(argv)
    dev = torch.device("cuda", 0)
    code = (LdpcCode.dvb_t2_normal if a.frame == "normal" else LdpcCode.dvb_t2_short)(RATES[a.rate])
    lo, hi = (float(x) for x in a.train_ebn0.split(":"))
    s0, s1, ds = (float(x) for x in a.points.split(":"))
    points = [round(s0 + i * ds, 6) for i in range(int(round((s1 - s0) / ds)) + 1)]

    sched = C.SCHED_LAYERED if a.schedule == "layered" else C.SCHED_FLOODING
    msg = C.MSG_F16 if a.msg16 else C.MSG_F32
    tr = NmsTrainer(code, iterations=a.iters, batch=a.batch, ebn0_range=(lo, hi), lr=a.lr, seed=1, device=dev,
                    schedule=sched)
    steps = max(1, a.train_frames // a.batch)
    train_s = 0.0
    if a.weights:
        tr.load(a.weights)
        steps = tr.step_no
        lo, hi = tr.ebn0_range  # the checkpoint's training range
    else:
        t0 = time.time()
        tr.train(steps, log_every=max(1, steps // 10), log=lambda s: print(s, flush=True))
        torch.cuda.synchronize()
        train_s = time.time() - t0
        if a.save_weights:
            tr.save(a.save_weights)
    alpha, beta = tr.weights()
    want = a.decoders.split(",")
    learned = tr.decoder(msg_dtype=msg)
    spa_lay = LdpcDecoder(code, algorithm=C.ALGO_SPA_FAST, schedule=C.SCHED_LAYERED, msg_dtype=C.MSG_F16)
    all_decs = {
        "learned": lambda: learned,
        "learned_fb": lambda: FallbackDecoder(learned, spa_lay, a.spa_iters),
        "minsum": lambda: LdpcDecoder(code, algorithm=C.ALGO_NMS, schedule=sched, msg_dtype=msg,
                                      nms_alpha=np.ones((1, tr.L), np.float32),
                                      nms_beta=np.zeros((1, tr.L), np.float32)),
        "spa50": lambda: LdpcDecoder(code, algorithm=C.ALGO_SPA),
        "spa50_layered": lambda: spa_lay,
    }
    decs = {k: all_decs[k]() for k in want}
    iters = {"learned": a.iters, "learned_fb": a.iters, "minsum": a.iters, "spa50": a.spa_iters,
             "spa50_layered": a.spa_iters}
    curves = {k: [] for k in decs}
    for eb in points:
        for name, dec in decs.items():
            if curves[name] and curves[name][-1]["fer"] < a.target_fer / 10:
                continue  # well below the target: higher Eb/N0 adds nothing to the crossing
            r = simulate_point(dec, code, eb, iters[name], batch=a.eval_batch, max_frames=a.max_frames,
                               min_frame_errors=a.min_frame_errors, seed=7, device=dev)
            r = {k: v for k, v in r.items() if k != "iter_hist"}
            r["decoder"] = name
            curves[name].append(r)
            print(json.dumps(r), flush=True)
    cross = {k: crossing(v, a.target_fer) for k, v in curves.items()}
    if a.throughput_ebn0 is None:
        tp_points = [cross.get("spa50") if cross.get("spa50") is not None else points[len(points) // 2]]
    else:
        tp_points = [float(x) for x in a.throughput_ebn0.split(",")]
    tp_all = {f"{e:.2f}": {k: throughput(d, code, e, iters[k], a.throughput_frames, dev) for k, d in decs.items()}
              for e in tp_points}
    eb_tp = tp_points[0]
    tp = tp_all[f"{eb_tp:.2f}"]

    def diff(x, y):
        return (cross[x] - cross[y]) if cross.get(x) is not None and cross.get(y) is not None else None
    summary = dict(
        code=f"dvbt2-{a.frame}-{a.rate}", n=code.n(), k=code.k(), learned_iters=a.iters, schedule=a.schedule,
        train=dict(frames=tr.frame_counter if a.weights else steps * a.batch, ebn0=[lo, hi], lr=a.lr,
                   seconds=round(train_s, 2),
                   final_loss=tr.history[-1] if tr.history else None, loaded=a.weights),
        target_fer=a.target_fer, ebn0_at_target=cross,
        gap_db_learned_vs_spa50=diff("learned", "spa50"),
        gap_db_learned_vs_spa50_layered=diff("learned", "spa50_layered"),
        gain_db_learned_vs_minsum=diff("minsum", "learned"),
        throughput_at_ebn0=eb_tp, throughput=tp, throughput_per_ebn0=tp_all,
        speedup_learned_vs_spa50=(tp["learned"]["gbit_s"] / tp["spa50"]["gbit_s"])
        if "learned" in tp and "spa50" in tp else None,
        alpha_mean_per_iter=[round(float(x), 4) for x in alpha.mean(axis=1)],
        beta_mean_per_iter=[round(float(x), 4) for x in beta.mean(axis=1)],
        curves=curves)
    print(json.dumps({k: v for k, v in summary.items() if k != "curves"}), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(summary, f, indent=1)
    return summary


if __name__ == "__main__":
    main()
