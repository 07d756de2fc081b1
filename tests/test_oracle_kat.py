"""CPU tests of the oracle against the reference's own known-answer tests.

The reference (Rust) cannot be built in this image; its unit and integration
tests are restated here against the C++ oracle, which pins the restatement.
Each test names the reference test it restates (paths relative to
crates/gf2-coding/ unless noted).
"""
import numpy as np
import pytest

NAMES = ["normal 1/2", "normal 3/5", "normal 2/3", "normal 3/4", "normal 4/5", "normal 5/6",
         "short 1/2", "short 3/5", "short 2/3", "short 3/4", "short 4/5", "short 5/6"]

# (n, k, q) from DvbParams::for_code tests (src/ldpc/dvb_t2/params.rs:88-259) and the
# Tanner-graph edge counts of the 12 codes (no duplicate table entries cancel).
DVB = [(64800, 32400, 90, 226799), (64800, 38880, 72, 285119), (64800, 43200, 60, 215999),
       (64800, 48600, 45, 226799), (64800, 51840, 36, 233279), (64800, 54000, 30, 237599),
       (16200, 7200, 25, 48599), (16200, 9720, 18, 58319), (16200, 10800, 15, 53999),
       (16200, 11880, 12, 47519), (16200, 12600, 10, 44999), (16200, 13320, 8, 49319)]


@pytest.mark.parametrize("idx", range(12))
def test_dvbt2_params_and_structure(oracle, idx):
    n, k, q, E = DVB[idx]
    c = oracle.Code.dvbt2(idx // 6, idx % 6)
    assert (c.n, c.k, c.m, c.layers, c.nnz) == (n, k, n - k, q, E)
    ip, ix = c.csr()
    dc = np.diff(ip)
    cp, cx = c.csc()
    dv = np.diff(cp)
    # staircase: parity columns have degree 2 except the last (builder.rs:106-115)
    assert (dv[k:-1] == 2).all() and dv[-1] == 1
    # check 0 misses the sub-diagonal: exactly one check one below its row group's degree
    assert dc[0] == dc[q] - 1
    # zero codeword is valid (tests/dvb_t2_ldpc_tests.rs)
    assert c.syndrome(np.zeros(n, np.uint8)).sum() == 0
    # CSR rows ascending, CSC rows ascending (sparse.rs:166-203, 297-328)
    for r in range(0, c.m, max(1, c.m // 50)):
        row = ix[ip[r]:ip[r + 1]]
        assert (np.diff(row) > 0).all()
    for v in range(0, n, max(1, n // 50)):
        col = cx[cp[v]:cp[v + 1]]
        assert (np.diff(col) > 0).all()


def test_dvbt2_edge_formula(oracle):
    # builder.rs:84-92: info bit b*360+j connects to (x + j q) mod m
    c = oracle.Code.dvbt2(1, 0)  # short 1/2, first table row starts with x = 20
    ip, ix = c.csr()
    m, q = c.m, 25
    for j in (0, 1, 359):
        p = (20 + j * q) % m
        assert j in set(ix[ip[p]:ip[p + 1]].tolist())


def test_from_coo_xor_cancellation(oracle):
    # gf2-core sparse.rs:155-163 doc test: duplicates cancel
    c = oracle.Code.edges(2, 3, [(0, 1), (0, 1), (1, 2)])
    assert c.nnz == 1
    ip, ix = c.csr()
    assert ix.tolist() == [2]


def test_qc_circulant_convention(oracle):
    # tests/qc_ldpc_tests.rs:61-119: row i of a shift-s circulant has column (i+s) mod Z
    c = oracle.Code.qc([[1]], 4)
    ip, ix = c.csr()
    assert ix.tolist() == [1, 2, 3, 0]
    c = oracle.Code.qc([[-1, -1, 1]], 3)
    ip, ix = c.csr()
    assert ix.tolist() == [7, 8, 6]
    c = oracle.Code.qc([[0, 1], [1, 0]], 3)
    assert (c.m, c.n) == (6, 6)


def test_qc_invalid_shift(oracle):
    # tests/qc_ldpc_tests.rs:179-213: invalid shifts panic
    with pytest.raises(oracle.OracleError):
        oracle.Code.qc([[5]], 3)


SPC = [(0, 0), (0, 1), (0, 2)]


def test_decoder_kat_spc(oracle):
    # src/ldpc/core.rs:1149-1186 (trivial decode, single error) and 1244-1266 (batch)
    c = oracle.Code.edges(1, 3, SPC)
    llr = np.array([[10, 10, 10], [-5, -5, 2], [-10, -10, 10], [10, 10, 10]], np.float32)
    r = c.decode_faithful(llr, 20)
    assert r["conv"].all() and r["synd_ok"].all()
    assert r["iters"].max() <= 2
    assert r["msg"].sum(axis=1).tolist() == [0, 2, 2, 0]
    # [-5,-5,2]: c2v = (-2,-2,+5) -> beliefs (-7,-7,7)
    assert r["beliefs"][1].tolist() == [-7.0, -7.0, 7.0]


def test_decoder_zero_iterations(oracle):
    # decode_iterative with max_iterations = 0 on a fresh decoder (core.rs:889-938):
    # beliefs stay zero, the all-zero word passes the syndrome, converged = false
    c = oracle.Code.edges(1, 3, SPC)
    r = c.decode_faithful(np.array([[-10, -10, 10]], np.float32), 0)
    assert r["iters"][0] == 0 and not r["conv"][0] and r["synd_ok"][0]
    assert r["msg"].sum() == 0


def test_decoder_simd_validation_short(oracle):
    # tests/ldpc_simd_validation.rs:27-43: short 1/2, all +5 converges within 10 iterations
    c = oracle.Code.dvbt2(1, 0)
    r = c.decode_faithful(np.full((1, c.n), 5.0, np.float32), 10)
    assert r["conv"][0] and r["msg"].sum() == 0


def test_decoder_infinite_llr(oracle):
    # tests/ldpc_validation.rs:349-422: +inf LLRs decode to the zero word
    c = oracle.Code.dvbt2(1, 0)
    r = c.decode_faithful(np.full((1, c.n), np.inf, np.float32), 5)
    assert r["conv"][0] and r["iters"][0] == 1 and r["msg"].sum() == 0


def test_minsum_scalar_kat(oracle):
    # llr.rs doc/unit tests: min-sum [3,-2,4] -> -2; [3,2,4] -> 2 (via a 4-edge check)
    c = oracle.Code.edges(1, 4, [(0, 0), (0, 1), (0, 2), (0, 3)])
    # c2v of edge 3 = minsum(x0, x1, x2); belief3 = llr3 + c2v3
    r = c.decode_faithful(np.array([[3, -2, 4, 0.0]], np.float32), 1)
    assert r["beliefs"][0][3] == -2.0
    r = c.decode_faithful(np.array([[3, 2, 4, 0.0]], np.float32), 1)
    assert r["beliefs"][0][3] == 2.0


def test_nms_oms_kat(oracle):
    # llr.rs:551-719: normalized 0.875*4 = 3.5; offset (4,6), beta 0.5 -> 3.5; clamp (0.3, 6) -> 0
    c = oracle.Code.edges(1, 3, [(0, 0), (0, 1), (0, 2)])
    llr = np.array([[4, 6, 0.0]], np.float32)
    r = c.decode(llr, 1, algo=3, alpha=np.array([0.875], np.float32), beta=np.array([0.0], np.float32))
    assert r["beliefs"][0][2] == np.float32(0.875) * np.float32(4.0)
    r = c.decode(llr, 1, algo=3, alpha=np.array([1.0], np.float32), beta=np.array([0.5], np.float32))
    assert r["beliefs"][0][2] == 3.5
    r = c.decode(np.array([[0.3, 6, 0.0]], np.float32), 1, algo=3, alpha=np.array([1.0], np.float32),
                 beta=np.array([0.5], np.float32))
    assert r["beliefs"][0][2] == 0.0


def test_faithful_equals_fast_awgn(oracle):
    # the reference-faithful decoder (neighbour lists, linear searches, AVX2
    # min-sum emulation) and the edge-indexed oracle agree bit for bit
    c = oracle.Code.dvbt2(1, 0)
    _, _, llr = c.channel(7, 0, 4, 1.2)
    a = c.decode_faithful(llr, 30)
    b = c.decode(llr, 30)
    for key in ("msg", "iters", "conv", "synd_ok"):
        assert (a[key] == b[key]).all()
    assert (a["beliefs"] == b["beliefs"]).all()


def test_faithful_equals_fast_dc_above_8(oracle):
    # normal 3/5 has dc = 11: the AVX2 8-lane chunk path is exercised
    c = oracle.Code.dvbt2(1, 1)  # short 3/5, dc = 9
    _, _, llr = c.channel(11, 0, 2, 1.5)
    a = c.decode_faithful(llr, 20)
    b = c.decode(llr, 20)
    assert (a["iters"] == b["iters"]).all() and (a["msg"] == b["msg"]).all()
    assert (a["beliefs"] == b["beliefs"]).all()


def test_philox_kat(oracle):
    # Random123 known-answer vectors for philox4x32_10
    assert oracle.philox4x32([0, 0, 0, 0], [0, 0]).tolist() == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox4x32([0xffffffff] * 4, [0xffffffff] * 2).tolist() == [
        0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox4x32([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]).tolist() == [
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_own_math_accuracy(oracle):
    L = oracle.lib()
    import ctypes
    xs = np.concatenate([np.linspace(1e-300, 1, 2000), [2.0 ** -53, 0.5, 0.999999999]])
    for x in xs:
        assert abs(L.or_own_log(float(x)) - np.log(x)) <= 4e-16 * max(1.0, abs(np.log(x)))
    s, c = ctypes.c_double(), ctypes.c_double()
    for u in np.linspace(0, 1, 1001, endpoint=False):
        L.or_own_sincos2pi(float(u), ctypes.byref(s), ctypes.byref(c))
        assert abs(s.value - np.sin(2 * np.pi * u)) < 1e-15 and abs(c.value - np.cos(2 * np.pi * u)) < 1e-15


def test_channel_statistics(oracle):
    # channel.rs:153-158 sigma^2 and the LLR mean/variance of BPSK over AWGN
    c = oracle.Code.dvbt2(1, 0)
    info, cw, llr = c.channel(1, 0, 16, 1.0)
    s2 = oracle.sigma2(1.0, c.rate)
    assert abs(s2 - 1.0 / (2 * (7200 / 16200) * 10 ** 0.1)) < 1e-15
    assert abs(info.mean() - 0.5) < 0.01
    assert all(c.syndrome(x).sum() == 0 for x in cw)
    sym = 1.0 - 2.0 * cw
    z = (llr * s2 / 2.0 - sym) / np.sqrt(s2)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    assert (info == cw[:, :c.k]).all()


def test_encoder_unique_codeword_short(oracle):
    # richardson_urbanke.rs:158-289: pivots from the right are exactly k..n-1 for
    # DVB-T2, so the accumulator equals the reference's RREF encoder
    c = oracle.Code.dvbt2(1, 5)  # short 5/6: m = 2880
    ip, ix = c.csr()
    g = oracle.Code.edges(c.m, c.n, np.stack([np.repeat(np.arange(c.m), np.diff(ip)), ix], 1))
    mc, pc = g.encoder_columns()
    assert (np.sort(pc) == np.arange(c.k, c.n)).all() and (mc == np.arange(c.k)).all()
    rng = np.random.default_rng(3)
    msg = rng.integers(0, 2, (4, c.k), dtype=np.uint8)
    a = c.encode(msg)
    b = g.encode(msg)
    assert (a == b).all()
    assert all(c.syndrome(x).sum() == 0 for x in a)


def test_encoder_generic_spc(oracle):
    # core.rs:1214-1241 (encoder batch on the [3,2] SPC code): message bits in the
    # non-pivot columns, even parity
    c = oracle.Code.edges(1, 3, SPC)
    msg = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], np.uint8)
    cw = c.encode(msg)
    assert cw.tolist() == [[0, 0, 0], [1, 0, 1], [0, 1, 1], [1, 1, 0]]


def test_f16_rounding(oracle):
    f = oracle.f32_to_f16_bits
    assert f(1.0) == 0x3C00 and f(-2.0) == 0xC000 and f(65504.0) == 0x7BFF and f(65520.0) == 0x7C00
    assert f(5.960464477539063e-08) == 0x0001  # smallest subnormal
    for x in np.random.default_rng(0).normal(0, 100, 2000).astype(np.float32):
        assert f(float(x)) == int(np.float16(x).view(np.uint16))


def test_spa_layered_fp16_oracles_consistent(oracle):
    c = oracle.Code.dvbt2(1, 0)
    info, cw, llr = c.channel(5, 0, 6, 1.3)
    r32 = c.decode(llr, 50, algo=1)
    r64 = c.decode_spa64(llr, 50)
    lay = c.decode(llr, 50, algo=1, sched=1, msg16=True)
    # all three decode these frames; layered needs fewer iterations
    assert (r64["conv"]).all() and r32["conv"].all() and lay["conv"].all()
    assert (r32["msg"] == info).all() and (lay["msg"] == info).all()
    assert lay["iters"].mean() < r32["iters"].mean()


def test_nms_gradient_fd(oracle):
    # FP64 learned-min-sum gradient against central finite differences
    c = oracle.Code.dvbt2(1, 5)
    info, cw, llr = c.channel(9, 0, 2, 3.0)
    T, L = 3, c.layers
    rng = np.random.default_rng(1)
    a = 0.8 + 0.1 * rng.random(T * L)
    b = 0.1 + 0.1 * rng.random(T * L)
    loss, ga, gb, _ = c.nms_loss_grad(llr, cw, T, a, b)
    for idx in (0, L + 3, 2 * L + 5):
        for arr, g in ((a, ga), (b, gb)):
            h = 1e-6
            p = arr.copy(); p[idx] += h
            m = arr.copy(); m[idx] -= h
            lp = c.nms_loss_grad(llr, cw, T, p if arr is a else a, p if arr is b else b)[0]
            lm = c.nms_loss_grad(llr, cw, T, m if arr is a else a, m if arr is b else b)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd)


@pytest.mark.parametrize("frame,rate", [(1, 5), (1, 0), (0, 5)])
def test_nms_layered_gradient_fd(oracle, frame, rate):
    """FP64 layered learned-min-sum gradient against central finite differences;
    normal 5/6 has row groups with up to 4 circulants in one block (repeated
    variables inside a layer)."""
    c = oracle.Code.dvbt2(frame, rate)
    info, cw, llr = c.channel(9, 0, 1 if frame == 0 else 2, 3.0 if rate == 5 else 1.4)
    T, L = 3, c.layers
    rng = np.random.default_rng(2)
    a = 0.8 + 0.1 * rng.random(T * L)
    b = 0.1 + 0.1 * rng.random(T * L)
    loss, ga, gb, out = c.nms_loss_grad(llr, cw, T, a, b, layered=True)
    assert np.isfinite(loss) and np.abs(ga).max() > 0
    for idx in (0, L + 3, 2 * L + 5, T * L - 1):
        for arr, g in ((a, ga), (b, gb)):
            h = 1e-6
            p = arr.copy(); p[idx] += h
            m = arr.copy(); m[idx] -= h
            lp = c.nms_loss_grad(llr, cw, T, p if arr is a else a, p if arr is b else b, layered=True)[0]
            lm = c.nms_loss_grad(llr, cw, T, m if arr is a else a, m if arr is b else b, layered=True)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


def test_nms_layered_forward_equals_layered_decoder(oracle):
    """With alpha = 1, beta = 0 the layered training forward is plain layered
    min-sum: its final posterior equals the layered min-sum oracle decoder's
    (FP64 vs FP32 values, same decisions)."""
    c = oracle.Code.dvbt2(1, 0)
    info, cw, llr = c.channel(3, 0, 3, 1.6)
    T, L = 4, c.layers
    _, _, _, out = c.nms_loss_grad(llr, cw, T, np.ones(T * L), np.zeros(T * L), layered=True)
    r = c.decode(llr, T, algo=3, sched=1, alpha=np.ones((T, L), np.float32), beta=np.zeros((T, L), np.float32))
    ran = r["iters"] == T
    assert ran.any()
    assert np.allclose(out[ran], r["beliefs"][ran], rtol=1e-4, atol=1e-4)
