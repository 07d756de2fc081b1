#!/usr/bin/env python3
"""Decoded-throughput benchmark of the B200 LDPC decoder.

Metric: decoded information Gbit/s (sum of k over the frames of a step divided
by the step's device time).  Workloads (synthetic, seeded Philox frames made by
the library's channel kernel; they stand in for the reference's AWGN inputs):

  c2  (default) DVB-T2 normal-frame rate 3/5 (n=64800, k=38880), 4096 frames
      per launch, layered sum-product, messages stored FP16 / computed FP32,
      max 50 iterations with syndrome early stop; frame f at
      Eb/N0 = 0.6 + 0.1 (f mod 9) dB (the 0.6..1.4 dB sweep in one batch).
  c1  DVB-T2 short 1/2 (n=16200, k=7200), 256 frames, Eb/N0 1.0 dB,
      flooding sum-product FP32, max 50 iterations.
  c1ref  the c1 frames with the reference's own decoder (flooding min-sum FP32).

A step is one decode launch over the batch; its LLRs (frames x n x 4 bytes,
1 GB for c2) are larger than L2, so consecutive steps do not hit in L2.

`--impl reference` times the reference decoder's CPU restatement (flooding
min-sum, neighbour lists, one decoder per frame, all host threads) on a bounded
sample of the same frames.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decoded info Gbit/s on 1 B200 at matched FER: learned min-sum vs plain BP"
UNIT = "Gbit/s"

WORKLOADS = {
    "c2": dict(frame=0, rate=1, frames=4096, algo=3, sched=1, msg16=True, max_iter=50,
               ebn0=[0.6 + 0.1 * i for i in range(9)],
               desc="dvbt2-normal-3/5 layered sum-product (SFU), fp16 messages / fp32 math, 4096 frames, "
                    "Eb/N0 0.6..1.4 dB (frame f at 0.6+0.1*(f mod 9)), max 50 it, early stop"),
    "c2exact": dict(frame=0, rate=1, frames=4096, algo=1, sched=1, msg16=True, max_iter=50,
                    ebn0=[0.6 + 0.1 * i for i in range(9)],
                    desc="dvbt2-normal-3/5 layered sum-product (bit-exact numerics), fp16 messages, "
                         "4096 frames, Eb/N0 0.6..1.4 dB, max 50 it, early stop"),
    "c1": dict(frame=1, rate=0, frames=256, algo=1, sched=0, msg16=False, max_iter=50, ebn0=[1.0],
               desc="dvbt2-short-1/2 flooding sum-product fp32, 256 frames, Eb/N0 1.0 dB, max 50 it"),
    "c1ref": dict(frame=1, rate=0, frames=256, algo=0, sched=0, msg16=False, max_iter=50, ebn0=[1.0],
                  desc="dvbt2-short-1/2 flooding min-sum fp32 (reference decoder), 256 frames, "
                       "Eb/N0 1.0 dB, max 50 it"),
}
EDGES = {(0, 1): 285119, (1, 0): 48599, (0, 0): 226799, (0, 2): 215999}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    p.add_argument("--frames", type=int, default=0, help="override frames per rank (profiling)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    return p.parse_args()


def ebn0_of(w, frames):
    pts = w["ebn0"]
    return [pts[f % len(pts)] for f in range(frames)]


def alg_bytes(n, k, E, msg_bytes, iters):
    """Algorithmic bytes: per frame 4n + k/8 (LLR in, bits out) plus per executed
    iteration 2 E s_msg + 2 n 4 (read + write every c2v message and the FP32
    posterior once)."""
    b_iter = 2 * E * msg_bytes + 2 * n * 4
    b_fixed = 4 * n + k / 8
    return sum(b_fixed + it * b_iter for it in iters)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def read_traffic(workload):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"bp_decode_{workload}.md")
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_sample_frames(w, cores):
    per = len(w["ebn0"])
    return per * max(1, round(cores / per)) if per > 1 else max(1, cores)


def run_cpu_reference(w, seed, steps, warmup, cores=None):
    """The reference decoder's restatement on host threads: returns (Gbit/s, info)."""
    from oracle import pyoracle
    pyoracle.build()
    cores = cores or os.cpu_count() or 1
    code = pyoracle.Code.dvbt2(w["frame"], w["rate"])
    S = cpu_sample_frames(w, cores)
    eb = ebn0_of(w, S)
    _, _, llr = code.channel(seed, 0, S, eb)
    times = []
    iters = None
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        r = code.decode_faithful(llr, w["max_iter"], threads=cores)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
        iters = r["iters"]
    tot = sum(times)
    gbps = S * code.k * len(times) / tot / 1e9
    sample = (f"{S} frames of the workload (frames 0..{S - 1}, every Eb/N0 point), reference min-sum "
              f"flooding max {w['max_iter']} it, mean {float(iters.mean()):.1f} it/frame, "
              f"{len(times)} timed passes of {tot / len(times):.2f} s")
    return gbps, dict(cores=cores, sample=sample, frames=S)


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": w["desc"], "code": f"dvbt2 {'normal' if w['frame'] == 0 else 'short'} rate-idx {w['rate']}",
              "frames_per_gpu": args.frames or w["frames"], "l2": "inputs larger than L2 (no flush)",
              "parallelism": f"replicas x{world} (frames sharded by index, no data-path collective)"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        gbps, info = run_cpu_reference(w, 1, args.steps, args.warmup)
        line = {"metric": METRIC, "value": gbps, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox AWGN frames)",
                "config": config,
                "cpu_baseline": {"value": gbps, "unit": UNIT, "cores": info["cores"], "kind": "port",
                                 "sample": info["sample"]},
                "e2e": {"value": gbps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch

    import gf2_b200 as g

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_
        dist = dist_
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)

    frames = args.frames or w["frames"]
    code = g.LdpcCode.dvb_t2_normal(w["rate"]) if w["frame"] == 0 else g.LdpcCode.dvb_t2_short(w["rate"])
    n, k = code.n(), code.k()
    E = code.nnz()
    eb = ebn0_of(w, frames)
    s2 = np.array([g.sigma2_from_ebn0(e, code.rate()) for e in eb])
    seed = 1
    _, _, llr = g.awgn_frames(code, seed, rank * frames, frames, s2, device=dev, want_info=False, want_cw=False)
    dec = g.LdpcDecoder(code, algorithm=w["algo"], schedule=w["sched"], msg_dtype=g.MSG_F16 if w["msg16"] else g.MSG_F32)
    out = None
    for _ in range(max(args.warmup, 0)):
        out = dec.decode_tensors(llr, w["max_iter"], out=out)
    torch.cuda.synchronize()

    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for s in range(args.steps):
        out = dec.decode_tensors(llr, w["max_iter"], out=out)
        ev[s + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    launches = dec.last_launches() * args.steps
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    iters = out["iters"].cpu().numpy()
    conv = out["conv"].cpu().numpy()
    bits_per_step = frames * k * world
    value = bits_per_step * args.steps / (total_ms / 1e3) / 1e9

    msg_bytes = 2 if w["msg16"] else 4
    bytes_launch = alg_bytes(n, k, E, msg_bytes, iters.tolist())
    avg_launch_s = statistics.mean(step_ms) / 1e3
    achieved = bytes_launch / avg_launch_s / 1e9
    peak, peak_kind = measured_peak()
    traffic = read_traffic(args.workload)

    e2e = None
    if not args.no_e2e:
        # public C-ABI host path: pinned host LLRs -> H2D -> decode -> D2H results
        h_llr = torch.empty((frames, n), dtype=torch.float32, pin_memory=True)
        h_llr.copy_(llr.cpu())
        h_msg = torch.empty((frames, g.words(k)), dtype=torch.int64, pin_memory=True)
        h_it = torch.empty(frames, dtype=torch.int32, pin_memory=True)
        h_cv = torch.empty(frames, dtype=torch.uint8, pin_memory=True)
        h_so = torch.empty(frames, dtype=torch.uint8, pin_memory=True)
        import ctypes
        from gf2_b200 import _capi as C

        def host_step():
            C.check(C.lib.gf2c_decode_batch(dec._h, ctypes.c_void_p(h_llr.data_ptr()), frames, w["max_iter"],
                                            ctypes.c_void_p(h_msg.data_ptr()), ctypes.c_void_p(h_it.data_ptr()),
                                            ctypes.c_void_p(h_cv.data_ptr()), ctypes.c_void_p(h_so.data_ptr()),
                                            None, C.MEM_HOST, None))
        host_step()
        e2e_steps = max(1, min(args.steps, 5))
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            host_step()
        t1 = time.perf_counter()
        e2e_s = t1 - t0
        if dist:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": bits_per_step * e2e_steps / e2e_s / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": frames * n * 4,
               "d2h_bytes_per_step": frames * (g.words(k) * 8 + 4 + 1 + 1),
               "steps": e2e_steps, "timing": "host wall clock around synchronous C-ABI calls"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        gbps, info = run_cpu_reference(w, seed, 1, 0)
        cpu = {"value": gbps, "unit": UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f16-storage/f32-math" if w["msg16"] else "f32",
                "data": "synthetic (seeded Philox AWGN frames, BPSK, encoder output)", "config": config,
                "iterations": {"mean": float(iters.mean()), "max": int(iters.max()),
                               "converged_frac": float(conv.mean())},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_launch},
                "gpu_launches": launches, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
