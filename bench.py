#!/usr/bin/env python3
"""Decoded-throughput benchmark of the B200 LDPC decoder.

Metric: decoded information Gbit/s (sum of k over the frames of a step divided
by the step's device time).  Inputs are synthetic: seeded Philox frames made by
the library's channel kernel (info bits, encoder, BPSK, AWGN, LLR = 2y/sigma^2),
standing in for the reference's AWGN simulation inputs.

Workloads (one "step" = one decode of the whole batch):
  c2            DVB-T2 normal rate 3/5 (n=64800, k=38880), 4096 frames,
                layered sum-product (SFU), messages stored FP16 / computed FP32,
                max 50 iterations with syndrome early stop; frame f at
                Eb/N0 = 0.6 + 0.1 (f mod 9) dB (the 0.6..1.4 dB sweep in one batch).
  c2exact       c2 with the bit-exact FP32 sum-product numerics.
  c2ref         the c2 frames with the reference's decoder (flooding min-sum
                FP32, results bit-identical to the reference).
  c1            DVB-T2 short 1/2 (n=16200, k=7200), 256 frames, Eb/N0 1.0 dB,
                flooding sum-product FP32 (bit-exact numerics), max 50 it.
  c1ref         the c1 frames with the reference's decoder (flooding min-sum FP32).
  c3            mixed batch: 32768 frames drawn uniformly from the 12 DVB-T2
                codes, per-frame Eb/N0 ~ U[thr, thr + 1] dB (thr = the
                reference's AwgnChannel::shannon_limit(k/n)), per-frame budget
                ~ U{10..50}; one persistent launch replayed from a CUDA graph,
                launch shape from the autotuner; layered sum-product (SFU), FP16.
  c5 (default)  DVB-T2 normal 2/3 (n=64800, k=43200), 65536 frames, learned
                normalised/offset min-sum (per-iteration, per-row-group weights
                trained on the GPU by the library's layered forward / backward
                kernels, gf2_b200/weights), 10 layered iterations, FP16 messages,
                early stop; frames still failing the syndrome are re-decoded on
                the device by 50-iteration layered sum-product (one C-ABI call,
                gf2c_decode_batch_fallback); frame f at Eb/N0 = 2.2 + 0.1 (f mod 5)
                dB.  The line also carries plain layered sum-product (max 50 it)
                on the same frames: its Gbit/s and FER, for the comparison at
                matched FER the metric names.
  bch           DVB-T2 normal 3/5 outer BCH code (n=38880, k=38688, t=12),
                65536 packed words, frame f with f mod 13 random bit errors;
                syndromes, Berlekamp-Massey and Chien search on the device
                (metric: BCH decoded info Gbit/s).
  enc           DVB-T2 normal 3/5 LDPC encoder, 65536 packed random messages
                (metric: LDPC encoded info Gbit/s).

The LLR input of every workload is larger than L2 (no flush needed).
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
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decoded info Gbit/s on 1 B200 at matched FER: learned min-sum vs plain BP"
UNIT = "Gbit/s"

SINGLE = {
    "c2": dict(frame=0, rate=1, frames=4096, algo=3, sched=1, msg16=True, max_iter=50,
               ebn0=[0.6 + 0.1 * i for i in range(9)],
               desc="dvbt2-normal-3/5 layered sum-product (SFU), fp16 messages / fp32 math, 4096 frames, "
                    "Eb/N0 0.6..1.4 dB (frame f at 0.6+0.1*(f mod 9)), max 50 it, early stop"),
    "c2exact": dict(frame=0, rate=1, frames=4096, algo=1, sched=1, msg16=True, max_iter=50,
                    ebn0=[0.6 + 0.1 * i for i in range(9)],
                    desc="dvbt2-normal-3/5 layered sum-product (bit-exact numerics), fp16 messages, "
                         "4096 frames, Eb/N0 0.6..1.4 dB, max 50 it, early stop"),
    "c2ref": dict(frame=0, rate=1, frames=4096, algo=0, sched=0, msg16=False, max_iter=50,
                  ebn0=[0.6 + 0.1 * i for i in range(9)],
                  desc="dvbt2-normal-3/5 flooding min-sum fp32 (reference decoder), 4096 frames, "
                       "Eb/N0 0.6..1.4 dB (frame f at 0.6+0.1*(f mod 9)), max 50 it, early stop"),
    "c1": dict(frame=1, rate=0, frames=256, algo=1, sched=0, msg16=False, max_iter=50, ebn0=[1.0],
               desc="dvbt2-short-1/2 flooding sum-product fp32, 256 frames, Eb/N0 1.0 dB, max 50 it"),
    "c1ref": dict(frame=1, rate=0, frames=256, algo=0, sched=0, msg16=False, max_iter=50, ebn0=[1.0],
                  desc="dvbt2-short-1/2 flooding min-sum fp32 (reference decoder), 256 frames, "
                       "Eb/N0 1.0 dB, max 50 it"),
}
WORKLOADS = sorted(list(SINGLE) + ["c3", "c5", "bch", "enc"])
BCH_METRIC = "BCH decoded info Gbit/s on 1 B200 (DVB-T2 outer code, hard decision)"
BCH_DATA = "synthetic (seeded random messages, BCH-encoded, f mod 13 random bit errors per frame)"
BCH_DESC = ("dvbt2-normal-3/5 outer BCH (n=38880, k=38688, t=12) hard-decision decode, 65536 frames, "
            "frame f carries f mod 13 random bit errors (0..t, every frame corrected)")
ENC_METRIC = "LDPC encoded info Gbit/s on 1 B200 (DVB-T2 encoder)"
ENC_DATA = "synthetic (seeded random messages)"
ENC_DESC = "dvbt2-normal-3/5 LDPC encode (k=38880 -> n=64800), 65536 frames of random messages"


def metric_of(w):
    return {"bch": BCH_METRIC, "enc": ENC_METRIC}.get(w, METRIC)


def data_of(w, gpu_arm):
    if w in ("bch", "enc"):
        return BCH_DATA if w == "bch" else ENC_DATA
    return ("synthetic (seeded Philox AWGN frames, BPSK, encoder output)" if gpu_arm
            else "synthetic (seeded Philox AWGN frames)")


# (threads, CTAs per SM) of the workload's primary decoder from --shape, else None (autotuned)
FORCED_SHAPE = None


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c5", choices=WORKLOADS)
    p.add_argument("--frames", type=int, default=0, help="override frames per rank (profiling)")
    p.add_argument("--shape", default=None,
                   help="THREADS,CTAS_PER_SM: launch shape of the workload's (primary) decoder instead of the "
                        "autotuner's (profiling a small case at the full run's shape)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    return p.parse_args()


def alg_bytes(n, k, E, msg_bytes, iters):
    """Algorithmic bytes of one frame: 4n + k/8 (LLR in, bits out) plus per
    executed iteration 2 E s_msg + 2 n 4 (read + write every c2v message and the
    FP32 posterior once)."""
    return 4 * n + k / 8 + iters * (2 * E * msg_bytes + 2 * n * 4)


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


def source_hash(paths):
    """sha256 over the named source files (paths relative to the repository)."""
    import hashlib
    h = hashlib.sha256()
    for rel in paths:
        with open(os.path.join(ROOT, rel), "rb") as f:
            h.update(rel.encode() + b"\0" + f.read())
    return h.hexdigest()


def read_traffic(workload, frame_iters):
    """DRAM bytes of the launch: the per-frame-iteration DRAM traffic of the
    workload's dominant kernel from its ncu capture (profiles/traffic.json)
    times the frame-iterations the timed launch executed.  None when there is
    no capture or when the kernel's sources changed since it was taken (the
    entry records the sha256 of the sources it profiled)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            e = json.load(f).get(workload)
    except (OSError, ValueError):
        return None, "no ncu capture"
    if not e:
        return None, "no ncu capture of this workload"
    try:
        if source_hash(e["sources"]) != e["source_sha256"]:
            return None, "ncu capture predates the current kernel sources"
    except OSError:
        return None, "kernel sources missing"
    return e["dram_bytes_per_frame_iteration"] * frame_iters, e["capture"]


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU reference (the reference decoder's restatement)
# ---------------------------------------------------------------------------
def cpu_reference_frames(name):
    """(frame, rate, max_iter, ebn0 list) of the frames the CPU baseline decodes."""
    if name in SINGLE:
        w = SINGLE[name]
        return w["frame"], w["rate"], w["max_iter"], w["ebn0"]
    if name == "c5":
        return 0, 2, 50, C5_POINTS
    return 0, 1, 50, [1.0 + 0.1 * i for i in range(9)]  # c3: normal 3/5 sample


def run_cpu_reference(name, seed, steps, warmup, cores=None):
    from oracle import pyoracle
    pyoracle.build()
    cores = cores or os.cpu_count() or 1
    frame, rate, max_iter, pts = cpu_reference_frames(name)
    code = pyoracle.Code.dvbt2(frame, rate)
    per = len(pts)
    # A multiple of the thread count, at least two frames per thread, grown
    # until one pass takes about 10 s, so that no thread idles and the sample
    # is a stable measure (frame f at Eb/N0 point f mod per).
    S = cores * max(2, -(-per // cores))
    for _ in range(6):
        eb = [pts[f % per] for f in range(S)]
        _, _, llr = code.channel(seed, 0, S, eb)
        t0 = time.perf_counter()
        code.decode_faithful(llr, max_iter, threads=cores)
        dt = time.perf_counter() - t0
        if dt >= 5.0:
            break
        S = cores * max(2 * (S // cores), int(-(-S * 10.0 / max(dt, 1e-3) // cores)))
        S = min(S, cores * 256)
    times, iters = [], None
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        r = code.decode_faithful(llr, max_iter, threads=cores)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
        iters = r["iters"]
    tot = sum(times)
    gbps = S * code.k * len(times) / tot / 1e9
    sample = (f"{S} frames of the workload's code (dvbt2 {'normal' if frame == 0 else 'short'} rate-idx {rate}, "
              f"every Eb/N0 point), reference min-sum flooding max {max_iter} it, "
              f"mean {float(iters.mean()):.1f} it/frame, {len(times)} timed passes of {tot / len(times):.2f} s")
    return gbps, dict(cores=cores, sample=sample, frames=S)


# ---------------------------------------------------------------------------
# GPU workloads
# ---------------------------------------------------------------------------
class SingleCode:
    def __init__(self, name, dev, rank, frames):
        import numpy as np

        import gf2_b200 as g
        self.g = g
        w = SINGLE[name]
        self.w = w
        self.frames = frames or w["frames"]
        self.code = g.LdpcCode.dvb_t2_normal(w["rate"]) if w["frame"] == 0 else g.LdpcCode.dvb_t2_short(w["rate"])
        pts = w["ebn0"]
        s2 = np.array([g.sigma2_from_ebn0(pts[f % len(pts)], self.code.rate()) for f in range(self.frames)])
        _, _, self.llr = g.awgn_frames(self.code, 1, rank * self.frames, self.frames, s2, device=dev,
                                       want_info=False, want_cw=False)
        msg = g.MSG_F16 if w["msg16"] else g.MSG_F32
        from gf2_b200 import autotune
        sample = self.llr[:min(8192, self.frames)]  # the whole batch up to 8192 frames: its tail counts
        shape = FORCED_SHAPE or autotune.tune([self.code], w["algo"], w["sched"], msg,
                                              lambda d: d.decode_tensors(sample, w["max_iter"]),
                                              frames=sample.shape[0])[0]
        self.dec = g.LdpcDecoder(self.code, algorithm=w["algo"], schedule=w["sched"], msg_dtype=msg,
                                 threads_per_block=shape[0], blocks_per_sm=shape[1])
        self.out = None
        self.desc = w["desc"] + f", autotuned launch shape {tuple(shape)}"
        self.dtype = "f16 storage / f32 math" if w["msg16"] else "f32"
        self.msg_bytes = 2 if w["msg16"] else 4

    def step(self):
        self.out = self.dec.decode_tensors(self.llr, self.w["max_iter"], out=self.out)

    def launches(self):
        return self.dec.last_launches()

    def bits_per_step(self):
        return self.frames * self.code.k()

    def stats(self):
        it = self.out["iters"].cpu().numpy()
        conv = self.out["conv"].cpu().numpy()
        c = self.code
        b = sum(alg_bytes(c.n(), c.k(), c.nnz(), self.msg_bytes, int(i)) for i in it)
        return b, {"mean": float(it.mean()), "max": int(it.max()), "converged_frac": float(conv.mean()),
                   "frame_iterations": int(it.sum())}

    def host_step_factory(self):
        """The public C-ABI host path: pinned host LLRs in, results out."""
        import ctypes

        import torch

        from gf2_b200 import _capi as C
        n, k, F = self.code.n(), self.code.k(), self.frames
        h_llr = torch.empty((F, n), dtype=torch.float32, pin_memory=True)
        h_llr.copy_(self.llr.cpu())
        h_msg = torch.empty((F, self.g.words(k)), dtype=torch.int64, pin_memory=True)
        h_it = torch.empty(F, dtype=torch.int32, pin_memory=True)
        h_cv = torch.empty(F, dtype=torch.uint8, pin_memory=True)
        h_so = torch.empty(F, dtype=torch.uint8, pin_memory=True)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())

        def host_step():
            C.check(C.lib.gf2c_decode_batch(self.dec._h, vp(h_llr), F, self.w["max_iter"], vp(h_msg), vp(h_it),
                                            vp(h_cv), vp(h_so), None, C.MEM_HOST, None))
        return host_step, F * n * 4, F * (self.g.words(k) * 8 + 4 + 1 + 1)


class Mixed:
    """c3: 32768 frames over the 12 DVB-T2 codes in one persistent launch."""

    def __init__(self, dev, rank, frames):
        import numpy as np
        import torch

        import gf2_b200 as g
        from gf2_b200 import autotune
        self.g = g
        self.frames = frames or 32768
        self.codes = [g.LdpcCode.dvb_t2_normal(r) for r in range(6)] + [g.LdpcCode.dvb_t2_short(r) for r in range(6)]
        rng = np.random.default_rng(1000 + rank)
        cid = rng.integers(0, 12, self.frames)
        budget = rng.integers(10, 51, self.frames)
        thr = [shannon_limit(c.rate()) for c in self.codes]
        eb = np.array([thr[c] + rng.random() for c in cid])
        # generate per code, then lay frames out in the random order of cid
        llr_parts, offs = [], np.zeros(self.frames, np.int64)
        msg_off = np.zeros(self.frames, np.int64)
        base = 0
        mbase = 0
        for f in range(self.frames):
            msg_off[f] = mbase
            mbase += g.words(self.codes[cid[f]].k())
        for c in range(12):
            idx = np.nonzero(cid == c)[0]
            if len(idx) == 0:
                continue
            code = self.codes[c]
            s2 = np.array([g.sigma2_from_ebn0(eb[i], code.rate()) for i in idx])
            _, _, l = g.awgn_frames(code, 7, (rank * 12 + c) << 24, len(idx), s2, device=dev,
                                    want_info=False, want_cw=False)
            llr_parts.append(l.reshape(-1))
            offs[idx] = base + np.arange(len(idx)) * code.n()
            base += len(idx) * code.n()
        self.llr = torch.cat(llr_parts)
        self.llr_off = torch.from_numpy(offs).to(dev)
        self.cid = torch.from_numpy(cid.astype(np.int32)).to(dev)
        self.mit = torch.from_numpy(budget.astype(np.int32)).to(dev)
        self.msg_off = torch.from_numpy(msg_off).to(dev)
        self.msg = torch.zeros(int(mbase), dtype=torch.int64, device=dev)
        self.iters = torch.zeros(self.frames, dtype=torch.int32, device=dev)
        self.conv = torch.zeros(self.frames, dtype=torch.uint8, device=dev)
        self.so = torch.zeros(self.frames, dtype=torch.uint8, device=dev)
        self.cid_np = cid
        self.algo, self.sched, self.msg16 = g.ALGO_SPA_FAST, g.SCHED_LAYERED, g.MSG_F16

        def run(dec):
            dec.decode_mixed_tensors(self.llr, self.llr_off, self.cid, self.mit, self.msg, self.msg_off,
                                     self.iters, self.conv, self.so, use_graph=False)
        if FORCED_SHAPE:
            (threads, bps), self.tune_table = FORCED_SHAPE, []
        else:
            (threads, bps), self.tune_table = autotune.tune(self.codes, self.algo, self.sched, self.msg16, run,
                                                            frames=self.frames)
        self.shape = (threads, bps)
        self.dec = g.LdpcDecoder(self.codes[0], codes=self.codes, algorithm=self.algo, schedule=self.sched,
                                 msg_dtype=self.msg16, threads_per_block=threads, blocks_per_sm=bps)
        self.desc = (f"mixed batch: {self.frames} frames uniform over the 12 DVB-T2 codes, per-frame Eb/N0 "
                     f"U[thr, thr+1] (thr = shannon_limit(k/n)), per-frame budget U{{10..50}}, layered "
                     f"sum-product (SFU) fp16, an ordering kernel (frames grouped by code) and one persistent decode launch "
                     f"from a CUDA graph, autotuned shape "
                     f"threads={threads} blocks/SM={bps or 'max'}")
        self.dtype = "f16 storage / f32 math"

    def step(self):
        self.dec.decode_mixed_tensors(self.llr, self.llr_off, self.cid, self.mit, self.msg, self.msg_off, self.iters,
                                      self.conv, self.so, use_graph=True)

    def launches(self):
        return self.dec.last_launches()

    def bits_per_step(self):
        return int(sum(self.codes[c].k() for c in self.cid_np))

    def stats(self):
        it = self.iters.cpu().numpy()
        b = 0.0
        for c in range(12):
            sel = it[self.cid_np == c]
            code = self.codes[c]
            b += sum(alg_bytes(code.n(), code.k(), code.nnz(), 2, int(i)) for i in sel)
        return b, {"mean": float(it.mean()), "max": int(it.max()),
                   "converged_frac": float(self.conv.float().mean().item()), "frame_iterations": int(it.sum())}

    def host_step_factory(self):
        import ctypes

        import torch

        from gf2_b200 import _capi as C
        h = lambda t: t.cpu().pin_memory()
        h_llr, h_lo, h_cid, h_mit, h_mo = h(self.llr), h(self.llr_off), h(self.cid), h(self.mit), h(self.msg_off)
        h_msg = torch.empty_like(self.msg, device="cpu").pin_memory()
        h_it = torch.empty(self.frames, dtype=torch.int32).pin_memory()
        h_cv = torch.empty(self.frames, dtype=torch.uint8).pin_memory()
        h_so = torch.empty(self.frames, dtype=torch.uint8).pin_memory()
        vp = lambda t: ctypes.c_void_p(t.data_ptr())

        def host_step():
            C.check(C.lib.gf2c_decode_mixed(self.dec._h, vp(h_llr), vp(h_lo), vp(h_cid), vp(h_mit), self.frames,
                                            vp(h_msg), vp(h_mo), vp(h_it), vp(h_cv), vp(h_so), 0, C.MEM_HOST, None))
        h2d = h_llr.numel() * 4 + self.frames * (8 + 4 + 4 + 8)
        d2h = h_msg.numel() * 8 + self.frames * 6
        return host_step, h2d, d2h


C5_POINTS = [2.2 + 0.1 * i for i in range(5)]
C5_WEIGHTS = os.path.join(ROOT, "gf2_b200", "weights", "nms_layered_normal_2_3_T10.npz")


class LearnedScale:
    """c5: learned min-sum at scale with a sum-product fallback, against plain
    sum-product on the same frames (the metric's comparison at matched FER)."""

    def __init__(self, dev, rank, frames):
        import numpy as np
        import torch

        import gf2_b200 as g
        from gf2_b200.learned import NmsTrainer
        self.g = g
        self.torch = torch
        self.frames = frames or 65536
        self.code = g.LdpcCode.dvb_t2_normal(g.CodeRate.Rate2_3)
        self.T = 10
        tr = NmsTrainer(self.code, iterations=self.T, batch=256, ebn0_range=(2.0, 2.8), lr=1e-2, seed=1,
                        device=dev, alpha0=1.0, beta0=0.0, schedule=g.SCHED_LAYERED)
        if os.path.exists(C5_WEIGHTS):
            tr.load(C5_WEIGHTS)
            self.weights_desc = (f"trained on the GPU by the library's layered forward / backward kernels: "
                                 f"{tr.frame_counter} frames (Eb/N0 U[{tr.ebn0_range[0]}, {tr.ebn0_range[1]}] dB), "
                                 f"loaded from gf2_b200/weights")
        else:
            tr.train(400)
            self.weights_desc = "trained before timing: 400 Adam steps x 256 frames, Eb/N0 U[2.0, 2.8] dB"
        a, b = tr.weights()
        del tr
        pts = C5_POINTS
        s2 = np.array([g.sigma2_from_ebn0(pts[f % len(pts)], self.code.rate()) for f in range(self.frames)])
        self.info, _, self.llr = g.awgn_frames(self.code, 3, rank * self.frames, self.frames, s2, device=dev,
                                               want_cw=False)
        self.point_of = torch.tensor([f % len(pts) for f in range(self.frames)], device=dev)
        # launch shapes of both decoders from the autotuner (timed on the first 8192 frames)
        from gf2_b200 import autotune
        sample = self.llr[:min(8192, self.frames)]
        kw_nms = dict(algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, nms_alpha=a, nms_beta=b, msg_dtype=g.MSG_F16)
        kw_spa = dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
        sh_nms = FORCED_SHAPE or autotune.tune([self.code], g.ALGO_NMS, g.SCHED_LAYERED, g.MSG_F16,
                                               lambda d: d.decode_tensors(sample, self.T), nms_alpha=a, nms_beta=b,
                                               frames=sample.shape[0])[0]
        sh_spa, _ = autotune.tune([self.code], g.ALGO_SPA_FAST, g.SCHED_LAYERED, g.MSG_F16,
                                  lambda d: d.decode_tensors(sample, 50), frames=sample.shape[0])
        self.shapes = {"learned": sh_nms, "plain": sh_spa}
        self.nms = g.LdpcDecoder(self.code, threads_per_block=sh_nms[0], blocks_per_sm=sh_nms[1], **kw_nms)
        self.spa = g.LdpcDecoder(self.code, threads_per_block=sh_spa[0], blocks_per_sm=sh_spa[1], **kw_spa)
        self.out = None
        self.desc = (f"dvbt2-normal-2/3 learned normalised/offset min-sum ({self.T} layered iterations, per-iteration "
                     f"per-row-group weights {self.weights_desc}), fp16 messages, {self.frames} frames, "
                     f"frame f at Eb/N0 {pts[0]:.1f}+0.1*(f mod {len(pts)}) dB, early stop; frames still failing "
                     f"the syndrome re-decoded on the device by layered sum-product (SFU) max 50 it; compared with "
                     f"layered sum-product (SFU) max 50 it alone on the same frames; autotuned launch shapes "
                     f"(threads, CTAs/SM; 0 = default) learned {tuple(sh_nms)}, plain {tuple(sh_spa)}")
        self.dtype = "f16 storage / f32 math"

    def step(self):
        self.out = self.nms.decode_with_fallback(self.spa, self.llr, self.T, 50, out=self.out)

    def launches(self):
        return self.nms.last_launches()

    def bits_per_step(self):
        return self.frames * self.code.k()

    def _fer(self, out):
        torch = self.torch
        wrong = (out["msg"] != self.info).any(dim=1)
        per = torch.zeros(len(C5_POINTS), dtype=torch.int64, device=wrong.device)
        per.index_add_(0, self.point_of, wrong.long())
        n = self.frames // len(C5_POINTS)
        return int(wrong.sum()), {f"{p:.1f}": int(x) for p, x in zip(C5_POINTS, per.tolist())}, n

    def stats(self):
        import numpy as np

        from gf2_b200.montecarlo import wilson
        torch = self.torch
        it = self.out["iters"].cpu().numpy()
        fb = int(self.out["fallback_count"][0])
        c = self.code
        b = 0.0
        for i in it:
            i = int(i)
            b += alg_bytes(c.n(), c.k(), c.nnz(), 2, min(i, self.T))
            if i > self.T:
                b += alg_bytes(c.n(), c.k(), c.nnz(), 2, i - self.T)
        fe, per, n = self._fer(self.out)
        # plain sum-product on the same frames: throughput (CUDA events) and FER
        st = torch.cuda.current_stream()
        r = self.spa.decode_tensors(self.llr, 50)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record(st)
        for _ in range(reps):
            r = self.spa.decode_tensors(self.llr, 50, out=r)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        fe_p, per_p, _ = self._fer(r)
        plain = {"decoder": "layered sum-product (SFU), fp16 messages, max 50 it, early stop",
                 "value": self.frames * c.k() / ms / 1e6, "unit": UNIT, "ms_per_step": ms,
                 "mean_iters": float(r["iters"].float().mean().item()), "frame_errors": fe_p,
                 "fer": fe_p / self.frames, "fer_ci": wilson(fe_p, self.frames), "frame_errors_per_ebn0": per_p}
        return b, {"mean": float(it.mean()), "max": int(it.max()),
                   "converged_frac": float(self.out["conv"].float().mean().item()),
                   "fallback_frames": fb, "frame_iterations": int(np.minimum(it, self.T).sum()),
                   "frame_iterations_all_passes": int(it.sum()),
                   "fer": {"learned_with_fallback": fe / self.frames,
                           "learned_with_fallback_ci": wilson(fe, self.frames),
                           "frame_errors_per_ebn0": per, "frames_per_ebn0": n,
                           "plain": fe_p / self.frames},
                   "plain_bp": plain}

    def host_step_factory(self):
        """The fallback call on pinned host memory: the library copies the LLRs
        in, decodes (chunks whose copies overlap the decoding of the previous
        chunk) and copies the results out before it returns.  Under torchrun
        (several ranks on one host) each rank's end-to-end step covers its
        first 16384 frames, so that the pinned host buffers of all ranks stay
        a few GB each."""
        torch = self.torch
        world = int(os.environ.get("WORLD_SIZE", "1"))
        F = self.frames if world == 1 else min(self.frames, 16384)
        n, wk = self.code.n(), self.g.words(self.code.k())
        self.e2e_frames = F
        h_llr = torch.empty((F, n), dtype=torch.float32, pin_memory=True)
        h_llr.copy_(self.llr[:F])
        out = dict(msg=torch.empty((F, wk), dtype=torch.int64, pin_memory=True),
                   iters=torch.empty(F, dtype=torch.int32, pin_memory=True),
                   conv=torch.empty(F, dtype=torch.uint8, pin_memory=True),
                   synd_ok=torch.empty(F, dtype=torch.uint8, pin_memory=True))

        def host_step():
            self.nms.decode_with_fallback(self.spa, h_llr, self.T, 50, out=out)
        return host_step, F * n * 4, F * (wk * 8 + 4 + 1 + 1)


def shannon_limit(rate):
    """AwgnChannel::shannon_limit (crates/gf2-coding/src/channel.rs:271-295):
    bisection on the numerically integrated BPSK capacity."""
    import math

    import numpy as np

    def cap(snr):
        sq = math.sqrt(snr)
        npts, ymax = 1000, sq + 6.0
        dy = 2.0 * ymax / npts
        y = -ymax + np.arange(npts + 1) * dy
        fy = np.exp(-((y - sq) ** 2) / 2.0) / math.sqrt(2.0 * math.pi)
        arg = -2.0 * sq * y
        lt = np.where(arg > 20, arg / math.log(2.0),
                      np.where(arg < -20, 0.0, np.log2(1.0 + np.exp(np.minimum(arg, 20.0)))))
        wgt = np.ones(npts + 1)
        wgt[0] = wgt[-1] = 0.5
        return min(1.0, max(0.0, 1.0 - float((wgt * fy * lt).sum()) * dy))

    lo, hi = -10.0, 25.0
    for _ in range(60):
        mid = (lo + hi) / 2
        c = cap(10 ** (mid / 10))
        if abs(c - rate) < 1e-6:
            return mid
        if c > rate:
            hi = mid
        else:
            lo = mid
    return (lo + hi) / 2


def bch_frames(frames, seed):
    """Seeded BCH test words of the bch workload as one bit per byte (CPU):
    random messages, frame f with f mod 13 flipped bits at distinct positions."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n, k, t = 38880, 38688, 12
    msg = rng.integers(0, 2, (frames, k), dtype=np.uint8)
    errs = [(f, rng.choice(n, size=f % (t + 1), replace=False)) for f in range(frames)]
    return msg, errs


class BchBatch:
    """DVB-T2 normal 3/5 outer BCH decode of a device batch of packed words."""

    def __init__(self, dev, rank, frames):
        import numpy as np
        import torch

        import gf2_b200 as g
        self.g = g
        self.frames = frames or 65536
        self.code = g.BchCode.dvb_t2(0, 1)
        n, k, t = self.code.n(), self.code.k(), self.code.t()
        F, wk, wn = self.frames, g.words(k), g.words(n)
        gen = torch.Generator(device=dev)
        gen.manual_seed(1000 + rank)
        m = torch.randint(-2 ** 31, 2 ** 31, (F, 2 * wk), dtype=torch.int32, device=dev, generator=gen)
        self.msg_words = m.view(torch.int64)
        if k & 63:
            self.msg_words[:, -1] &= (1 << (k & 63)) - 1
        cw = g.BchEncoder(self.code).encode_words(self.msg_words)
        # f mod (t+1) errors per frame at distinct positions, XORed in on the host
        rng = np.random.default_rng(2000 + rank)
        h = cw.cpu().numpy().view(np.uint64)
        fi, wi, bi = [], [], []
        for f in range(F):
            pos = rng.choice(n, size=f % (t + 1), replace=False)
            fi.append(np.full(len(pos), f))
            wi.append(pos >> 6)
            bi.append(pos & 63)
        fi, wi, bi = np.concatenate(fi), np.concatenate(wi), np.concatenate(bi)
        np.bitwise_xor.at(h, (fi, wi), np.left_shift(np.uint64(1), bi.astype(np.uint64)))
        self.expect_flips = np.array([f % (t + 1) for f in range(F)], np.int32)
        self.cw = torch.from_numpy(h.view(np.int64)).to(dev)
        self.dec = g.BchDecoder(self.code)
        self.out = None
        self.desc = BCH_DESC
        self.dtype = "u16"
        self.stream = torch.cuda.current_stream(dev)

    def step(self):
        self.out = self.dec.decode_words(self.cw, stream=self.stream)

    def launches(self):
        return 2  # syndrome / Berlekamp-Massey kernel + Chien kernel

    def bits_per_step(self):
        return self.frames * self.code.k()

    def stats(self):
        fl = self.out["corrected"].cpu().numpy()
        ok = bool((fl == self.expect_flips).all()) and bool(torch_equal(self.out["msg"], self.msg_words))
        g, c = self.g, self.code
        per = 8 * g.words(c.n()) + 8 * g.words(c.k()) + 4
        return self.frames * per, {"corrected_mean": float(fl.mean()), "all_frames_recovered": ok,
                                   "errors_per_frame": "f mod 13"}

    def host_step_factory(self):
        """The public C-ABI host path: pinned packed words in, messages out."""
        import ctypes

        import torch

        from gf2_b200 import _capi as C
        g, c, F = self.g, self.code, self.frames
        h_cw = torch.empty_like(self.cw, device="cpu").pin_memory()
        h_cw.copy_(self.cw.cpu())
        h_msg = torch.empty((F, g.words(c.k())), dtype=torch.int64, pin_memory=True)
        h_fl = torch.empty(F, dtype=torch.int32, pin_memory=True)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())

        def host_step():
            C.check(C.lib.gf2c_bch_decode_batch(c.handle, vp(h_cw), F, vp(h_msg), vp(h_fl), None, C.MEM_HOST,
                                                None))
        return host_step, F * g.words(c.n()) * 8, F * (g.words(c.k()) * 8 + 4)


def torch_equal(a, b):
    import torch
    return torch.equal(a, b)


def run_cpu_bch(steps, warmup, cores=None, frames=None):
    """The BCH oracle (restatement of BchDecoder::decode) over a sample of the
    bch workload's words, chunks decoded concurrently on all host threads."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    from oracle import pyoracle
    pyoracle.build()
    cores = cores or os.cpu_count() or 1
    b = pyoracle.Bch(0, 1)
    S = frames or 13 * max(1, round(100 * cores / 13))
    msg, errs = bch_frames(S, 7)
    cw = b.encode(msg)
    for f, pos in errs:
        cw[f, pos] ^= 1
    chunks = np.array_split(np.arange(S), cores)
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        with ThreadPoolExecutor(cores) as ex:
            outs = list(ex.map(lambda ix: b.decode(cw[ix]), [c for c in chunks if len(c)]))
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    dm = np.concatenate([o[0] for o in outs])
    assert (dm == msg).all()
    tot = sum(times)
    gbps = S * b.k * len(times) / tot / 1e9
    sample = (f"{S} words of the bch workload's code (f mod 13 errors), BCH oracle decode on {cores} threads, "
              f"{len(times)} timed passes of {tot / len(times):.2f} s")
    return gbps, dict(cores=cores, sample=sample, frames=S)


class EncBatch:
    """DVB-T2 normal 3/5 LDPC encode of a device batch of packed messages."""

    def __init__(self, dev, rank, frames):
        import torch

        import gf2_b200 as g
        from gf2_b200 import _capi as C
        self.g, self.C, self.torch = g, C, torch
        self.frames = frames or 65536
        self.code = g.LdpcCode.dvb_t2_normal(1)
        k, n, F = self.code.k(), self.code.n(), self.frames
        gen = torch.Generator(device=dev)
        gen.manual_seed(3000 + rank)
        m = torch.randint(-2 ** 31, 2 ** 31, (F, 2 * g.words(k)), dtype=torch.int32, device=dev, generator=gen)
        self.msg = m.view(torch.int64)
        if k & 63:
            self.msg[:, -1] &= (1 << (k & 63)) - 1
        self.out = torch.zeros((F, g.words(n)), dtype=torch.int64, device=dev)
        self.stream = torch.cuda.current_stream(dev)
        self.desc = ENC_DESC
        self.dtype = "u32"

    def step(self):
        from gf2_b200.ldpc import _ptr, _stream_ptr
        self.C.check(self.C.lib.gf2c_encode_batch(self.code.handle, _ptr(self.msg), self.frames, _ptr(self.out),
                                                  self.C.MEM_DEVICE, _stream_ptr(self.stream)))

    def launches(self):
        return 1

    def bits_per_step(self):
        return self.frames * self.code.k()

    def stats(self):
        g, c = self.g, self.code
        s, w = c.syndrome_batch(self.out[:256].contiguous())
        self.torch.cuda.synchronize()
        per = 8 * g.words(c.k()) + 8 * g.words(c.n())
        return self.frames * per, {"codewords_checked": 256, "all_valid": bool((w.cpu() == 0).all())
                                   if hasattr(w, "cpu") else bool((w == 0).all())}

    def host_step_factory(self):
        """The public C-ABI host path: pinned packed messages in, codewords out."""
        import ctypes

        torch, g, C, c, F = self.torch, self.g, self.C, self.code, self.frames
        h_msg = torch.empty_like(self.msg, device="cpu").pin_memory()
        h_msg.copy_(self.msg.cpu())
        h_cw = torch.empty((F, g.words(c.n())), dtype=torch.int64, pin_memory=True)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())

        def host_step():
            C.check(C.lib.gf2c_encode_batch(c.handle, vp(h_msg), F, vp(h_cw), C.MEM_HOST, None))
        return host_step, F * g.words(c.k()) * 8, F * g.words(c.n()) * 8


def run_cpu_enc(steps, warmup, cores=None):
    """The oracle's systematic encoder (same unique codeword as the reference's
    RuEncodingMatrices::encode) on a sample of messages of the enc workload's
    code, chunks encoded concurrently on all host threads."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    from oracle import pyoracle
    pyoracle.build()
    cores = cores or os.cpu_count() or 1
    code = pyoracle.Code.dvbt2(0, 1)
    S = 512 * cores
    msg = np.random.default_rng(9).integers(0, 2, (S, code.k), dtype=np.uint8)
    chunks = [c for c in np.array_split(np.arange(S), cores) if len(c)]
    times = []
    with ThreadPoolExecutor(cores) as ex:
        for s in range(warmup + max(steps, 1)):
            t0 = time.perf_counter()
            list(ex.map(lambda ix: code.encode(msg[ix[0]:ix[-1] + 1]), chunks))
            dt = time.perf_counter() - t0
            if s >= warmup:
                times.append(dt)
    tot = sum(times)
    gbps = S * code.k * len(times) / tot / 1e9
    sample = (f"{S} messages of the enc workload's code, oracle encoder on {cores} threads, "
              f"{len(times)} timed passes of {tot / len(times):.2f} s")
    return gbps, dict(cores=cores, sample=sample, frames=S)


def make_workload(name, dev, rank, frames):
    if name in SINGLE:
        return SingleCode(name, dev, rank, frames)
    if name == "c3":
        return Mixed(dev, rank, frames)
    if name == "bch":
        return BchBatch(dev, rank, frames)
    if name == "enc":
        return EncBatch(dev, rank, frames)
    return LearnedScale(dev, rank, frames)


def main():
    args = parse()
    global FORCED_SHAPE
    if args.shape:
        FORCED_SHAPE = tuple(int(x) for x in args.shape.split(","))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        if args.workload == "bch":
            gbps, info = run_cpu_bch(args.steps, args.warmup)
            desc, decoder, metric = BCH_DESC, "reference BchDecoder::decode (CPU restatement)", BCH_METRIC
        elif args.workload == "enc":
            gbps, info = run_cpu_enc(args.steps, args.warmup)
            desc, decoder, metric = ENC_DESC, "reference systematic LDPC encoder (CPU restatement)", ENC_METRIC
        else:
            gbps, info = run_cpu_reference(args.workload, 1, args.steps, args.warmup)
            desc = SINGLE[args.workload]["desc"] if args.workload in SINGLE else args.workload
            decoder, metric = "reference flooding min-sum (CPU restatement)", METRIC
        line = {"metric": metric, "value": gbps, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": {"bch": "u16", "enc": "u32"}.get(args.workload, "f32"),
                "data": data_of(args.workload, False),
                "config": {"workload": desc, "decoder": decoder},
                "cpu_baseline": {"value": gbps, "unit": UNIT, "cores": info["cores"], "kind": "port",
                                 "sample": info["sample"]},
                "e2e": {"value": gbps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
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

    wl = make_workload(args.workload, dev, rank, args.frames)
    for _ in range(max(args.warmup, 0)):
        wl.step()
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
    launches = 0
    for s in range(args.steps):
        wl.step()
        launches += wl.launches()
        ev[s + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    bits = wl.bits_per_step() * world
    value = bits * args.steps / (total_ms / 1e3) / 1e9
    bytes_launch, iters = wl.stats()
    traffic, traffic_src = read_traffic(args.workload, iters.get("frame_iterations", 0))
    avg_launch_s = statistics.mean(step_ms) / 1e3
    achieved = bytes_launch / avg_launch_s / 1e9
    peak, peak_kind = measured_peak()

    e2e = None
    if not args.no_e2e:
        host_step, h2d, d2h = wl.host_step_factory()
        if host_step is not None:
            host_step()
            n_e2e = max(1, min(args.steps, 5))
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(n_e2e):
                host_step()
            e2e_s = time.perf_counter() - t0
            if dist:
                t = torch.tensor([e2e_s], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                e2e_s = float(t.item())
            e2e_bits = bits
            if getattr(wl, "e2e_frames", None) and wl.e2e_frames != getattr(wl, "frames", None):
                e2e_bits = bits * wl.e2e_frames // wl.frames
            e2e = {"value": e2e_bits * n_e2e / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "steps": n_e2e,
                   "timing": "host wall clock around synchronous C-ABI calls (pinned host buffers)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        if args.workload == "bch":
            gbps, info = run_cpu_bch(1, 0)
        elif args.workload == "enc":
            gbps, info = run_cpu_enc(1, 0)
        else:
            gbps, info = run_cpu_reference(args.workload, 1, 1, 0)
        cpu = {"value": gbps, "unit": UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"]}

    if rank == 0:
        config = {"workload": wl.desc, "frames_per_gpu": getattr(wl, "frames", None),
                  "l2": "inputs larger than L2 (no flush)",
                  "parallelism": f"replicas x{world} (frames sharded by index, no data-path collective)"}
        line = {"metric": metric_of(args.workload), "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype,
                "data": data_of(args.workload, True),
                "config": config,
                "iterations": iters,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                             "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_launch},
                "gpu_launches": launches, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
