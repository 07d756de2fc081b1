"""Launch-shape autotuner for the decoders.

A decoder runs a persistent kernel in which each CTA decodes one frame at a
time; its launch shape is (threads per block, CTAs per SM), i.e. the checks a
thread steps over in each row group (the tile) and the number of frames in
flight per SM.
The autotuner times every feasible shape on a sample batch with CUDA events
and keeps the fastest; results are cached in a JSON file keyed by device name,
the build of the library (a hash of libgf2cuda.so), codes, algorithm, schedule,
message type and the sample's frame count (GF2C_AUTOTUNE_CACHE overrides the
default ~/.cache/gf2_b200/autotune.json).
"""
import json
import math
import os

from .ldpc import LdpcDecoder


def cache_path():
    return os.environ.get("GF2C_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "gf2_b200", "autotune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d):
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


_LIB_HASH = None


def library_hash():
    """sha256 prefix of the loaded libgf2cuda.so: a shape timed on one build of
    the kernels is not reused by another."""
    global _LIB_HASH
    if _LIB_HASH is None:
        import hashlib
        from . import _capi
        with open(_capi.LIB_PATH, "rb") as f:
            _LIB_HASH = hashlib.sha256(f.read()).hexdigest()[:16]
    return _LIB_HASH


def _key(codes, algorithm, schedule, msg_dtype, device_name, frames=None):
    cs = ",".join(f"{c.n()}x{c.m()}x{c.nnz()}" for c in codes)
    fs = f"|f{frames}" if frames else ""  # a shape timed on a few frames is not reused for many
    return f"{device_name}|lib {library_hash()}|{cs}|a{algorithm}|s{schedule}|m{msg_dtype}{fs}"


def candidates(codes, schedule, msg_dtype=0, algorithm=3):
    """(threads per block, CTAs per SM) pairs; 0 = library choice.  Layered:
    one thread per check of a row group (threads 0 = the row group rounded up
    to 32), or for one code with FP16 messages and a fused-row algorithm 192 /
    128 threads (each thread two / three checks, so four / six frames in
    flight per SM at the same registers; 192 threads with 5 CTAs per SM is a
    64-register build), and for a mixed batch with the SFU sum-product 192
    threads (posteriors in the workspace); the CTAs per SM vary within what fits.  Flooding: the
    library's choice (512 threads, or the check-state kernel of the min-sum
    family) at any / 1 / 2 CTAs per SM, 256 and 384 threads, and 1024 threads
    (codes of check degree <= 8: more threads per frame for small batches).
    Shapes a decoder cannot have are skipped when it fails to build."""
    if schedule == 1:
        c = [(0, b) for b in (0, 1)]
        if len(codes) == 1 and msg_dtype == 1 and algorithm != 1:
            c += [(192, b) for b in (0, 3, 5)] + [(128, b) for b in (0, 4)]
        elif len(codes) > 1 and msg_dtype == 1 and algorithm == 3:  # mixed batch, SFU sum-product
            c += [(192, b) for b in (0, 3)]
        return c
    return [(0, 0), (0, 1), (0, 2), (256, 0), (384, 0), (1024, 0)]


def tune(codes, algorithm, schedule, msg_dtype, run, reps=3, nms_alpha=None, nms_beta=None, force=False,
         frames=None):
    """Return ((threads, blocks_per_sm), table).  `run(decoder)` decodes the
    sample batch once on the current stream; `frames` (its size) is part of the
    cache key, since the best shape depends on how many frames are in flight."""
    import torch
    dev_name = torch.cuda.get_device_name()
    key = _key(codes, algorithm, schedule, msg_dtype, dev_name, frames)
    cache = _load()
    if key in cache and not force:
        e = cache[key]
        return (e["threads"], e["blocks_per_sm"]), e.get("table", [])
    table = []
    best = None
    for threads, bps in candidates(codes, schedule, msg_dtype, algorithm):
        try:
            dec = LdpcDecoder(codes[0], codes=codes, algorithm=algorithm, schedule=schedule, msg_dtype=msg_dtype,
                              nms_alpha=nms_alpha, nms_beta=nms_beta, threads_per_block=threads,
                              blocks_per_sm=bps)
        except Exception:
            continue
        run(dec)
        torch.cuda.synchronize()
        # the median of at least `reps` timed runs and of about 100 ms of
        # decoding (a small batch takes a few milliseconds, too short for 3
        # runs to separate shapes that differ by a few percent)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        run(dec)
        ev1.record()
        torch.cuda.synchronize()
        n = max(reps, min(64, int(math.ceil(100.0 / max(ev0.elapsed_time(ev1), 1e-3)))))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
        ev[0].record()
        for i in range(n):
            run(dec)
            ev[i + 1].record()
        torch.cuda.synchronize()
        ms = sorted(ev[i].elapsed_time(ev[i + 1]) for i in range(n))[n // 2]
        table.append([threads, bps, ms])
        if best is None or ms < best[2]:
            best = (threads, bps, ms)
        del dec
    if best is None:
        raise RuntimeError("no feasible launch shape")
    cache[key] = {"threads": best[0], "blocks_per_sm": best[1], "ms": best[2], "table": table}
    _store(cache)
    return (best[0], best[1]), table
