"""GPU test of gf2c_decode_batch_noalloc, the allocation-free decode entry point
for callers that cannot call cudaMalloc (stream capture into a CUDA graph,
externally owned device-memory pools, real-time paths).

It is called through the C ABI twice in a row -- two different codes, so the
second call replaces the code tables held in the shared static scratch -- and
each result must equal, bit for bit (the tolerance of the min-sum parity tests),
the result of the allocating entry point gf2c_decode_batch on the same device
inputs.  The file is named to be collected last, so a failure here stops a
`pytest -x` run only after every other test has run.
"""
import ctypes

import numpy as np
import pytest

import gf2_b200 as g
from gf2_b200 import _capi as C

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _outputs(torch, frames, k, dev):
    return (torch.zeros((frames, g.words(k)), dtype=torch.int64, device=dev),
            torch.zeros(frames, dtype=torch.int32, device=dev),
            torch.zeros(frames, dtype=torch.uint8, device=dev),
            torch.zeros(frames, dtype=torch.uint8, device=dev))


@pytest.mark.parametrize("first,second", [((1, 0), (0, 1))])
def test_noalloc_matches_decode_batch_twice(gpu, first, second):
    import torch
    stream = torch.cuda.current_stream(gpu)
    for frame_size, rate in (first, second):
        code = g.LdpcCode.dvb_t2_short(rate) if frame_size == 1 else g.LdpcCode.dvb_t2_normal(rate)
        frames, max_iter = 48, 30
        eb = np.array([0.8 + 0.05 * (f % 16) for f in range(frames)]) + (0.7 if frame_size == 0 else 0.0)
        s2 = np.array([g.sigma2_from_ebn0(e, code.rate()) for e in eb])
        _, _, llr = g.awgn_frames(code, 77, 1000 * rate, frames, s2, device=gpu, want_info=False, want_cw=False)
        ref = g.LdpcDecoder(code).decode_tensors(llr, max_iter)
        msg, it, cv, so = _outputs(torch, frames, code.k(), gpu)
        C.check(C.lib.gf2c_decode_batch_noalloc(code.handle, _vp(llr), frames, max_iter, _vp(msg), _vp(it),
                                                _vp(cv), _vp(so), ctypes.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        assert torch.equal(msg, ref["msg"])
        assert torch.equal(it, ref["iters"])
        assert torch.equal(cv, ref["conv"])
        assert torch.equal(so, ref["synd_ok"])
        assert int(it.max()) > 1  # the frames exercised real iterations


def test_noalloc_rejects_codes_beyond_the_static_scratch(gpu):
    import torch
    # 4M checks x 2 edges: the code tables alone exceed the 64 MiB scratch
    m, n = 4_000_000, 8_000_000
    rows = np.repeat(np.arange(m, dtype=np.int64), 2)
    cols = np.arange(n, dtype=np.int64)
    code = g.LdpcCode.from_edges(m, n, np.stack([rows, cols], 1))
    llr = torch.zeros((1, n), dtype=torch.float32, device=gpu)
    msg, it, cv, so = _outputs(torch, 1, code.k(), gpu)
    rc = C.lib.gf2c_decode_batch_noalloc(code.handle, _vp(llr), 1, 5, _vp(msg), _vp(it), _vp(cv), _vp(so), None)
    assert rc == C.ERR_UNSUPPORTED
    assert b"64 MiB" in C.lib.gf2c_last_error()
