"""Build libgf2cuda.so (sm_100a) in-tree with nvcc.

Every translation unit is compiled with -fmad=false so that no floating-point
multiply-add is contracted: the decoders' arithmetic is a fixed sequence of
separately rounded IEEE operations (the property the bit-exact parity tests
rely on).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgf2cuda.so")
SOURCES = ["capi.cu", "code_host.cpp", "decode.cu", "layered.cu", "layered_sfu16.cu", "layered_sfu32.cu", "layered_nms16.cu", "layered_nms32.cu", "layered_spa16.cu", "layered_spa32.cu", "encode_channel.cu", "learned.cu", "noalloc.cu", "spa64.cu", "state_flood.cu", "bch.cu", "gf2io.cpp", "dense_encode.cu"]
HEADERS = ["internal.h", "numeric.cuh", "layered_impl.cuh", "dvbt2_tables.h", "../../include/gf2cuda.h"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags():
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
            "-fmad=false", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-v" if os.environ.get("GF2C_PTXAS_V") else "-O3"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    objs = []
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    procs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(HERE, "_build", src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc()] + flags() + ["-c", s, "-o", o]
            if src.endswith(".cpp"):
                cmd = [nvcc(), "-x", "cu"] + flags() + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode()}")
        if verbose and out:
            print(out.decode(), file=sys.stderr)
    if force or _stale(OUT, objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + \
              ["-lcudart"]
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
