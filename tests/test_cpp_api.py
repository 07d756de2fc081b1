"""The C++ host API (gf2_b200/cpp/gf2cuda.hpp) compiles against the C ABI and
runs: code construction on the CPU, decoding on the GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "example")
    lib = os.path.join(ROOT, "gf2_b200")
    subprocess.check_call([gxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           "-I" + os.path.join(ROOT, "gf2_b200", "cpp"),
                           os.path.join(ROOT, "gf2_b200", "cpp", "example.cpp"), "-L" + lib, "-lgf2cuda",
                           "-Wl,-rpath," + lib, "-o", exe])
    return exe


def test_cpp_api_codes(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe, "codes"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "codes ok" in out.stdout


@pytest.mark.gpu
def test_cpp_api_decode(gpu, tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe, "decode"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "decode ok" in out.stdout
