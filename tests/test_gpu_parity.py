"""GPU parity tests: the sm_100a library against the CPU oracle on the same
seeded inputs, through the C ABI.

Bars: reference min-sum decoding is bit-exact (hard decisions, iteration
counts, flags, and posteriors, whose bits match the edge-indexed oracle and
whose values equal the reference-faithful oracle's); encoder, syndrome and
channel are bit-exact; the library's other decoders (sum-product FP32, layered,
FP16 message storage, normalised/offset min-sum) are bit-exact against their
oracle restatement.
"""
import numpy as np
import pytest

import gf2_b200 as g

pytestmark = pytest.mark.gpu


def dvb(idx):
    return g.LdpcCode.dvb_t2_normal(idx) if idx < 6 else g.LdpcCode.dvb_t2_short(idx - 6)


def unpack_msg(r, k):
    return g.unpack_bits(r["msg"], k)


def assert_same_decode(gpu, ora, k, bitwise=True):
    assert (gpu["iters"] == ora["iters"]).all(), (gpu["iters"], ora["iters"])
    assert (gpu["conv"] == ora["conv"]).all()
    assert (gpu["synd_ok"] == ora["synd_ok"]).all()
    assert (unpack_msg(gpu, k) == ora["msg"]).all()
    if "beliefs" in gpu:
        if bitwise:
            assert (gpu["beliefs"].view(np.uint32) == ora["beliefs"].view(np.uint32)).all()
        else:
            assert (gpu["beliefs"] == ora["beliefs"]).all()


def test_minsum_reference_parity_short_1_2(gpu, oracle):
    """The full config-1 batch: short 1/2, 256 frames, Eb/N0 1.0 dB, 50 iterations."""
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    ocode = oracle.Code.dvbt2(1, 0)
    _, _, llr = ocode.channel(1, 0, 256, 1.0)
    dec = g.LdpcDecoder(code)
    r = dec.decode_arrays(llr, 50, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 50), code.k(), bitwise=True)
    assert_same_decode(r, ocode.decode_faithful(llr, 50), code.k(), bitwise=False)


@pytest.mark.parametrize("idx,ebn0", [(1, 1.2), (5, 3.0), (9, 2.5)])
def test_minsum_reference_parity_codes(gpu, oracle, idx, ebn0):
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    _, _, llr = ocode.channel(2, 0, 12, ebn0)
    r = g.LdpcDecoder(code).decode_arrays(llr, 30, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 30), code.k(), bitwise=True)
    f = ocode.decode_faithful(llr[:4], 30)
    assert (r["iters"][:4] == f["iters"]).all() and (r["beliefs"][:4] == f["beliefs"]).all()


def test_decoder_kats(gpu):
    # ldpc/core.rs:1149-1294 decoder tests, through the library
    spc = g.LdpcCode.from_edges(1, 3, [(0, 0), (0, 1), (0, 2)])
    dec = g.LdpcDecoder(spc)
    r = dec.decode_iterative([g.Llr(10.0)] * 3, 10)
    assert r.converged and r.syndrome_check_passed and r.decoded_bits.sum() == 0 and r.iterations <= 2
    r = dec.decode_iterative([g.Llr(-5.0), g.Llr(-5.0), g.Llr(2.0)], 20)
    assert r.converged and r.decoded_bits.sum() == 2
    # no state leakage between decodes (core.rs:1188-1212)
    for llr, ones in (([10, 10, 10], 0), ([-10, -10, 10], 2), ([10, 10, 10], 0)):
        r = dec.decode_iterative(np.array(llr, np.float32), 10)
        assert r.converged and r.decoded_bits.sum() == ones
    res = g.LdpcDecoder.decode_batch(spc, [[10, 10, 10], [-10, -10, 10], [10, 10, 10]], 10)
    assert [x.decoded_bits.sum() for x in res] == [0, 2, 0] and all(x.converged for x in res)
    assert g.LdpcDecoder.decode_batch(spc, [], 10) == []
    r = dec.decode_iterative(np.array([-10, -10, 10], np.float32), 0)
    assert r.iterations == 0 and not r.converged and r.syndrome_check_passed and r.decoded_bits.sum() == 0
    with pytest.raises(ValueError):
        dec.decode_iterative([1.0, 2.0], 5)
    short = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    d2 = g.LdpcDecoder(short)
    r = d2.decode_iterative(np.full(short.n(), 5.0, np.float32), 10)   # ldpc_simd_validation.rs:27-43
    assert r.converged
    r = d2.decode_iterative(np.full(short.n(), np.inf, np.float32), 5)  # ldpc_validation.rs:349-422
    assert r.converged and r.iterations == 1 and r.decoded_bits.sum() == 0


@pytest.mark.parametrize("sched,msg16", [(0, False), (1, False), (1, True), (0, True)])
def test_spa_parity(gpu, oracle, sched, msg16):
    """Exact FP32 sum-product (flooding: the config-1 decoder) bit-exact against
    its CPU restatement; the flooding FP32 case on the full 256-frame batch."""
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    ocode = oracle.Code.dvbt2(1, 0)
    _, _, llr = ocode.channel(3, 0, 256 if (sched, msg16) == (0, False) else 24, 1.0)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_SPA, schedule=sched, msg_dtype=g.MSG_F16 if msg16 else g.MSG_F32)
    r = dec.decode_arrays(llr, 50, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 50, algo=1, sched=sched, msg16=msg16), code.k())


@pytest.mark.parametrize("idx", [1, 5, 0])
def test_layered_dup_blocks_parity(gpu, oracle, idx):
    """Normal 3/5 and 5/6 have up to 3 and 4 circulants in one (row group, block)."""
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    _, _, llr = ocode.channel(4, 0, 6, 1.6 if idx != 5 else 3.3)
    for algo, oalgo in ((g.ALGO_MINSUM, 0), (g.ALGO_SPA, 1)):
        dec = g.LdpcDecoder(code, algorithm=algo, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
        r = dec.decode_arrays(llr, 20, beliefs=True)
        assert_same_decode(r, ocode.decode(llr, 20, algo=oalgo, sched=1, msg16=True), code.k())


@pytest.mark.parametrize("idx,sched,msg16,ebn0", [(6, 1, True, 1.1), (1, 1, True, 1.2), (5, 1, False, 3.3),
                                                  (6, 0, False, 1.1)])
def test_spa_fast_against_fp64(gpu, oracle, idx, sched, msg16, ebn0):
    """SFU sum-product: not bit-exact; judged against the FP64 sum-product oracle
    (same schedule) by frame errors and by the deviation of the posteriors.
    Normal 3/5 and 5/6 (layered) hold row groups with up to 3 and 4 circulants
    in one block: the one-barrier path for repeated variables."""
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    info, _, llr = ocode.channel(21, 0, 48, ebn0)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_SPA_FAST, schedule=sched,
                        msg_dtype=g.MSG_F16 if msg16 else g.MSG_F32)
    r = dec.decode_arrays(llr, 50, beliefs=True)
    ref = ocode.decode_spa64(llr, 50, sched=sched)
    bits = unpack_msg(r, code.k())
    fe_gpu = int((bits != info).any(axis=1).sum())
    fe_ref = int((ref["msg"] != info).any(axis=1).sum())
    assert abs(fe_gpu - fe_ref) <= 2, (fe_gpu, fe_ref)
    both = r["conv"] & ref["conv"]
    assert both.sum() >= 0.8 * ref["conv"].sum()
    assert (bits[both] == ref["msg"][both]).all()
    # same decisions after one iteration, posteriors within 1e-2 relative + FP16 step
    r1 = dec.decode_arrays(llr[:8], 1, beliefs=True)
    ref1 = ocode.decode_spa64(llr[:8], 1, sched=sched)
    dev = np.abs(r1["beliefs"] - ref1["beliefs"])
    assert (dev <= 2e-2 * np.abs(ref1["beliefs"]) + 2e-2).mean() > 0.999


@pytest.mark.parametrize("sched", [0, 1])
def test_nms_parity(gpu, oracle, sched):
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate3_5)
    ocode = oracle.Code.dvbt2(1, 1)
    _, _, llr = ocode.channel(6, 0, 16, 1.6)
    rng = np.random.default_rng(0)
    T, L = 6, code.layers()
    a = (0.6 + 0.4 * rng.random((T, L))).astype(np.float32)
    b = (0.3 * rng.random((T, L))).astype(np.float32)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, schedule=sched, nms_alpha=a, nms_beta=b)
    r = dec.decode_arrays(llr, 20, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 20, algo=3, sched=sched, alpha=a, beta=b), code.k())


@pytest.mark.parametrize("idx,msg16", [(6, True), (1, True), (3, False)])
def test_minsum_flooding_fp16_and_placements(gpu, oracle, idx, msg16):
    """Check-state kernel: FP16 magnitudes (short 1/2: states and posteriors in
    shared memory; normal 3/5: both in the workspace) and normal 3/4 (states in
    the workspace, 16200 checks)."""
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    _, _, llr = ocode.channel(12, 3, 10, 1.0 if idx != 3 else 2.6)
    dec = g.LdpcDecoder(code, msg_dtype=g.MSG_F16 if msg16 else g.MSG_F32)
    r = dec.decode_arrays(llr, 25, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 25, msg16=msg16), code.k())


def test_minsum_flooding_qc_and_normal_nms(gpu, oracle):
    # a QC code (identity variable order, circulant descriptors)
    rng = np.random.default_rng(5)
    base = [[int(s) if rng.random() < 0.7 else -1 for s in rng.integers(0, 96, 24)] for _ in range(8)]
    q = g.LdpcCode.from_quasi_cyclic(g.QuasiCyclicLdpc(base, 96))
    oq = oracle.Code.qc(base, 96)
    llr = rng.normal(1.2, 1.5, (12, q.n())).astype(np.float32)
    r = g.LdpcDecoder(q).decode_arrays(llr, 15, beliefs=True)
    assert_same_decode(r, oq.decode(llr, 15), q.k())
    # normalised / offset min-sum on a normal frame (per-row-group weights)
    code = dvb(2)
    ocode = oracle.Code.dvbt2(0, 2)
    _, _, llr = ocode.channel(13, 0, 6, 2.0)
    T, L = 5, code.layers()
    a = (0.6 + 0.4 * rng.random((T, L))).astype(np.float32)
    b = (0.3 * rng.random((T, L))).astype(np.float32)
    dec = g.LdpcDecoder(code, algorithm=g.ALGO_NMS, nms_alpha=a, nms_beta=b)
    r = dec.decode_arrays(llr, 12, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 12, algo=3, alpha=a, beta=b), code.k())


def test_device_tensor_path_matches_host(gpu, oracle):
    import torch
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate2_3)
    ocode = oracle.Code.dvbt2(1, 2)
    _, _, llr = ocode.channel(8, 0, 40, 2.0)
    dec = g.LdpcDecoder(code)
    h = dec.decode_arrays(llr, 40)
    d = dec.decode_tensors(torch.from_numpy(llr).to(gpu), 40)
    torch.cuda.synchronize()
    assert (d["msg"].cpu().numpy().view(np.uint64) == h["msg"]).all()
    assert (d["iters"].cpu().numpy() == h["iters"]).all()
    assert dec.last_launches() == 1


@pytest.mark.parametrize("kw", [dict(), dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)])
def test_pipelined_host_path_matches_device(gpu, kw):
    """Host-memory batches of 64 MB and more run in equal chunks on two streams
    (copies overlapping the decode, the last chunk hardest frames first);
    device batches of more frames than CTAs run hardest frames first: every
    output equals the one-launch device path and small batches."""
    import torch
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate3_5)
    F = 2048  # 133 MB of LLRs
    pts = [0.8 + 0.1 * i for i in range(9)]
    s2 = np.array([g.sigma2_from_ebn0(pts[f % 9], code.rate()) for f in range(F)])
    _, _, llr = g.awgn_frames(code, 5, 0, F, s2, device=gpu, want_info=False, want_cw=False)
    dec = g.LdpcDecoder(code, **kw)
    d = dec.decode_tensors(llr, 30, beliefs=True)
    torch.cuda.synchronize()
    assert dec.last_launches() == 3  # frame keys, hardest-first order, decode
    h = dec.decode_arrays(llr.cpu().numpy(), 30, beliefs=True)
    assert dec.last_launches() > 3
    # the order does not change a frame's results: batches too small to be reordered
    parts = [dec.decode_tensors(llr[i:i + 128], 30, beliefs=True) for i in range(0, F, 128)]
    torch.cuda.synchronize()
    assert dec.last_launches() == 1
    for key in ("msg", "iters", "conv", "beliefs"):
        assert (torch.cat([p[key] for p in parts]) == d[key]).all(), key
    assert (d["msg"].cpu().numpy().view(np.uint64) == h["msg"]).all()
    assert (d["iters"].cpu().numpy() == h["iters"]).all()
    assert (d["conv"].cpu().numpy() == h["conv"]).all()
    assert (d["beliefs"].cpu().numpy().view(np.uint32) == h["beliefs"].view(np.uint32)).all()
    assert 0 < int(h["conv"].sum()) < F


@pytest.mark.parametrize("idx", range(12))
def test_encoder_syndrome_parity(gpu, oracle, idx):
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    rng = np.random.default_rng(idx)
    msg = rng.integers(0, 2, (5, code.k()), dtype=np.uint8)
    msg[0] = 0
    cw = g.LdpcEncoder(code).encode_packed(g.pack_bits(msg, code.k()))
    assert (g.unpack_bits(cw, code.n()) == ocode.encode(msg)).all()
    s, w = code.syndrome_batch(cw)
    assert (w == 0).all() and (s == 0).all()
    bad = g.unpack_bits(cw, code.n()).copy()
    bad[1, 7] ^= 1
    bad[2, code.n() - 1] ^= 1
    s, w = code.syndrome_batch(g.pack_bits(bad, code.n()))
    for f in range(5):
        os_ = ocode.syndrome(bad[f])
        assert w[f] == os_.sum()
        assert (g.unpack_bits(s[f:f + 1], code.m())[0] == os_).all()


def test_encoder_generic_codes(gpu, oracle):
    spc = g.LdpcCode.from_edges(1, 3, [(0, 0), (0, 1), (0, 2)])
    enc = g.LdpcEncoder(spc)
    cws = enc.encode_batch([np.array(m, np.uint8) for m in ([0, 0], [1, 0], [0, 1], [1, 1])])
    assert [c.tolist() for c in cws] == [[0, 0, 0], [1, 0, 1], [0, 1, 1], [1, 1, 0]]
    assert enc.encode_batch([]) == []
    base = [[0, 3, 1, -1, 2, 0], [2, -1, 4, 1, 0, 3], [-1, 1, 0, 3, 4, 1]]
    q = g.LdpcCode.from_quasi_cyclic(g.QuasiCyclicLdpc(base, 7))
    oq = oracle.Code.qc(base, 7)
    msg = np.random.default_rng(5).integers(0, 2, (6, q.k()), dtype=np.uint8)
    try:
        ref = oq.encode(msg)
    except oracle.OracleError:
        pytest.skip("random QC base is rank deficient")
    cw = g.LdpcEncoder(q).encode_packed(g.pack_bits(msg, q.k()))
    assert (g.unpack_bits(cw, q.n()) == ref).all()


@pytest.mark.parametrize("idx", [6, 1])
def test_channel_parity(gpu, oracle, idx):
    code = dvb(idx)
    ocode = oracle.Code.dvbt2(idx // 6, idx % 6)
    frames = 6
    eb = np.array([0.5, 1.0, 1.5, 2.0, 2.5, 3.0])
    s2 = np.array([oracle.sigma2(e, ocode.rate) for e in eb])
    info, cw, llr = g.awgn_frames(code, 1234, 77, frames, s2)
    oi, oc, ol = ocode.channel(1234, 77, frames, eb)
    assert (g.unpack_bits(info, code.k()) == oi).all()
    assert (g.unpack_bits(cw, code.n()) == oc).all()
    assert (llr.view(np.uint32) == ol.view(np.uint32)).all()


def test_mixed_batch_matches_single(gpu, oracle):
    idxs = [6, 7, 11, 1]
    codes = [dvb(i) for i in idxs]
    dec = g.LdpcDecoder(codes[0], codes=codes)
    rng = np.random.default_rng(2)
    F = 20
    cid = rng.integers(0, len(codes), F).astype(np.int32)
    mit = rng.integers(0, 30, F).astype(np.int32)
    llrs, lo, mo = [], [], []
    off = moff = 0
    for f in range(F):
        oc = oracle.Code.dvbt2(idxs[cid[f]] // 6, idxs[cid[f]] % 6)
        _, _, l = oc.channel(10, f, 1, 1.0 + 0.5 * rng.random() + (2.0 if idxs[cid[f]] == 11 else 0.0))
        llrs.append(l[0])
        lo.append(off)
        mo.append(moff)
        off += oc.n
        moff += g.words(oc.k)
    r = dec.decode_mixed_arrays(np.concatenate(llrs), lo, cid, mit, mo)
    for f in range(F):
        c = codes[cid[f]]
        single = g.LdpcDecoder(c).decode_arrays(llrs[f][None, :], int(mit[f]))
        assert r["iters"][f] == single["iters"][0]
        assert r["conv"][f] == single["conv"][0]
        w = g.words(c.k())
        assert (r["msg"][mo[f]:mo[f] + w] == single["msg"][0]).all()


def test_mixed_layered_batch_matches_single(gpu, oracle):
    """A mixed layered batch runs every frame with its own code's slot count:
    the results equal per-code decoders with the same options."""
    idxs = [6, 1, 11, 9]  # short 1/2 (7 slots), normal 3/5 (11), short 5/6 (19), short 3/4 (13)
    codes = [dvb(i) for i in idxs]
    kw = dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    dec = g.LdpcDecoder(codes[0], codes=codes, **kw)
    F = 16
    cid = np.array([f % len(codes) for f in range(F)], np.int32)
    mit = np.array([5 + 3 * (f % 7) for f in range(F)], np.int32)
    llrs, lo, mo = [], [], []
    off = moff = 0
    for f in range(F):
        i = idxs[cid[f]]
        oc = oracle.Code.dvbt2(i // 6, i % 6)
        _, _, l = oc.channel(21, f, 1, {6: 1.2, 1: 1.1, 11: 3.2, 9: 2.4}[i])
        llrs.append(l[0])
        lo.append(off)
        mo.append(moff)
        off += oc.n
        moff += g.words(oc.k)
    r = dec.decode_mixed_arrays(np.concatenate(llrs), lo, cid, mit, mo)
    for f in range(F):
        c = codes[cid[f]]
        single = g.LdpcDecoder(c, **kw).decode_arrays(llrs[f][None, :], int(mit[f]))
        assert r["iters"][f] == single["iters"][0]
        assert r["conv"][f] == single["conv"][0]
        w = g.words(c.k())
        assert (r["msg"][mo[f]:mo[f] + w] == single["msg"][0]).all()


def test_mixed_batch_graph_replay(gpu):
    import torch
    codes = [g.LdpcCode.dvb_t2_short(0), g.LdpcCode.dvb_t2_short(4)]
    dec = g.LdpcDecoder(codes[0], codes=codes)
    F = 16
    cid = torch.tensor([f % 2 for f in range(F)], dtype=torch.int32, device=gpu)
    n = [c.n() for c in codes]
    lo = torch.tensor([sum(n[f % 2] for f in range(i)) for i in range(F)], dtype=torch.int64, device=gpu)
    total = sum(n[f % 2] for f in range(F))
    outs = []
    for rep in range(3):
        llr = torch.full((total,), 4.0, device=gpu)
        mit = torch.full((F,), 10, dtype=torch.int32, device=gpu)
        msg = torch.zeros(F * 256, dtype=torch.int64, device=gpu)
        mo = torch.arange(F, dtype=torch.int64, device=gpu) * 256
        it = torch.zeros(F, dtype=torch.int32, device=gpu)
        cv = torch.zeros(F, dtype=torch.uint8, device=gpu)
        so = torch.zeros(F, dtype=torch.uint8, device=gpu)
        dec.decode_mixed_tensors(llr, lo, cid, mit, msg, mo, it, cv, so, use_graph=True)
        torch.cuda.synchronize()
        outs.append((it.cpu().numpy(), cv.cpu().numpy()))
    for it, cv in outs:
        assert (it == 1).all() and cv.all()


@pytest.mark.parametrize("use_graph", [False, True])
def test_mixed_batch_code_order(gpu, use_graph):
    """Mixed batches are decoded code by code (an ordering kernel before the
    persistent decode): 2500 frames in random code order and one invalid code
    id; every frame's results equal a single-code decode of it, the invalid
    frame reports -1 iterations."""
    import torch
    codes = [g.LdpcCode.dvb_t2_short(0), g.LdpcCode.dvb_t2_normal(1), g.LdpcCode.dvb_t2_short(2)]
    kw = dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    dec = g.LdpcDecoder(codes[0], codes=codes, **kw)
    rng = np.random.default_rng(11)
    F = 2500
    cid = rng.choice(3, F, p=[0.45, 0.1, 0.45]).astype(np.int32)
    budget = [12, 20, 9]
    mit = np.array([budget[c] for c in cid], np.int32)
    ebn0 = [1.2, 1.1, 2.2]
    singles, llr_parts, lo = {}, [], np.zeros(F, np.int64)
    base = 0
    for c in range(3):
        idx = np.nonzero(cid == c)[0]
        s2 = np.array([g.sigma2_from_ebn0(ebn0[c] + 0.1 * (i % 5), codes[c].rate()) for i in idx])
        _, _, l = g.awgn_frames(codes[c], 9, c << 20, len(idx), s2, device=gpu, want_info=False, want_cw=False)
        singles[c] = (idx, g.LdpcDecoder(codes[c], **kw).decode_tensors(l, budget[c]))
        llr_parts.append(l.reshape(-1))
        lo[idx] = base + np.arange(len(idx)) * codes[c].n()
        base += len(idx) * codes[c].n()
    bad = 7
    cid_run = cid.copy()
    cid_run[bad] = 5  # outside the decoder's codes
    W = max(g.words(c.k()) for c in codes)
    msg = torch.zeros(F * W, dtype=torch.int64, device=gpu)
    mo = torch.arange(F, dtype=torch.int64, device=gpu) * W
    it = torch.zeros(F, dtype=torch.int32, device=gpu)
    cv = torch.zeros(F, dtype=torch.uint8, device=gpu)
    so = torch.zeros(F, dtype=torch.uint8, device=gpu)
    dec.decode_mixed_tensors(torch.cat(llr_parts), torch.from_numpy(lo).to(gpu), torch.from_numpy(cid_run).to(gpu),
                             torch.from_numpy(mit).to(gpu), msg, mo, it, cv, so, use_graph=use_graph)
    torch.cuda.synchronize()
    assert dec.last_launches() == 2
    itn, cvn, msgn = it.cpu().numpy(), cv.cpu().numpy(), msg.cpu().numpy().view(np.uint64).reshape(F, W)
    assert itn[bad] == -1
    for c in range(3):
        idx, r = singles[c]
        keep = idx != bad
        w = g.words(codes[c].k())
        assert (itn[idx[keep]] == r["iters"].cpu().numpy()[keep]).all()
        assert (cvn[idx[keep]] == r["conv"].cpu().numpy()[keep]).all()
        assert (msgn[idx[keep], :w] == r["msg"].cpu().numpy().view(np.uint64)[keep]).all()


def test_edge_cases(gpu, oracle):
    # frames == 0 is a no-op; degree-1 check gives a zero message (core.rs:807-811)
    code = g.LdpcCode.from_edges(3, 5, [(0, 0), (1, 1), (1, 2), (2, 2), (2, 3), (2, 4), (1, 4)])
    ocode = oracle.Code.edges(3, 5, [(0, 0), (1, 1), (1, 2), (2, 2), (2, 3), (2, 4), (1, 4)])
    dec = g.LdpcDecoder(code)
    r = dec.decode_arrays(np.zeros((0, 5), np.float32), 5)
    assert r["iters"].shape == (0,)
    llr = np.random.default_rng(0).normal(1.0, 2.0, (50, 5)).astype(np.float32)
    r = dec.decode_arrays(llr, 7, beliefs=True)
    assert_same_decode(r, ocode.decode(llr, 7), code.k())
    # high-degree generic code (dc up to 40 -> the 64-slot kernel)
    rng = np.random.default_rng(1)
    edges = [(r_, int(v)) for r_ in range(20) for v in rng.choice(200, size=int(rng.integers(2, 41)), replace=False)]
    code = g.LdpcCode.from_edges(20, 200, edges)
    ocode = oracle.Code.edges(20, 200, edges)
    llr = rng.normal(2.0, 2.0, (30, 200)).astype(np.float32)
    for algo, oalgo in ((g.ALGO_MINSUM, 0), (g.ALGO_SPA, 1)):
        r = g.LdpcDecoder(code, algorithm=algo).decode_arrays(llr, 9, beliefs=True)
        assert_same_decode(r, ocode.decode(llr, 9, algo=oalgo), code.k())
    # early_stop = 0 runs every frame to max_iter
    short = g.LdpcCode.dvb_t2_short(0)
    r = g.LdpcDecoder(short, early_stop=False).decode_arrays(np.full((2, short.n()), 5.0, np.float32), 7)
    assert (r["iters"] == 7).all() and r["conv"].all()


@pytest.mark.parametrize("idx,algo", [(1, g.ALGO_SPA_FAST), (1, g.ALGO_NMS), (2, g.ALGO_MINSUM), (6, g.ALGO_SPA_FAST),
                                      (5, g.ALGO_NMS), (9, g.ALGO_SPA_FAST)])
@pytest.mark.parametrize("threads,bps", [(192, 0), (192, 5), (128, 0)])
def test_layered_shapes_bit_identical(gpu, oracle, idx, algo, threads, bps):
    """Several checks per thread (192 / 128 threads, more frames in flight per
    SM; 192 threads at 5 CTAs per SM is a separate 64-register build) give
    results bit-identical to one thread per check, for codes with
    repeated-variable row groups (normal 3/5, 5/6), the missing staircase
    corner, and short frames (posteriors in shared memory)."""
    import torch
    code = dvb(idx)
    L = code.layers()
    kw = dict(algorithm=algo, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    if algo == g.ALGO_NMS:
        rng = np.random.default_rng(idx)
        kw.update(nms_alpha=(0.7 + 0.3 * rng.random((4, L))).astype(np.float32),
                  nms_beta=(0.3 * rng.random((4, L))).astype(np.float32))
    ebn0 = {1: 1.2, 2: 2.2, 6: 1.1, 5: 3.3, 9: 2.4}[idx]
    _, _, llr = g.awgn_frames(code, 17, 0, 400, g.sigma2_from_ebn0(ebn0, code.rate()), device=gpu,
                              want_info=False, want_cw=False)
    ref = g.LdpcDecoder(code, **kw).decode_tensors(llr, 30, beliefs=True)
    r = g.LdpcDecoder(code, threads_per_block=threads, blocks_per_sm=bps, **kw).decode_tensors(llr, 30, beliefs=True)
    torch.cuda.synchronize()
    for key in ("msg", "iters", "conv", "synd_ok"):
        assert torch.equal(r[key], ref[key]), key
    assert torch.equal(r["beliefs"].view(torch.int32), ref["beliefs"].view(torch.int32))


def test_layered_minsum_equals_oracle_after_unit_weight_routing(gpu, oracle):
    """Layered min-sum runs on the normalised / offset min-sum kernels with
    alpha = 1, beta = 0: still bit-identical to the layered min-sum oracle."""
    code = dvb(1)
    ocode = oracle.Code.dvbt2(0, 1)
    _, _, llr = ocode.channel(12, 0, 6, 1.3)
    for msg16 in (False, True):
        dec = g.LdpcDecoder(code, algorithm=g.ALGO_MINSUM, schedule=g.SCHED_LAYERED,
                            msg_dtype=g.MSG_F16 if msg16 else g.MSG_F32)
        r = dec.decode_arrays(llr, 15, beliefs=True)
        assert_same_decode(r, ocode.decode(llr, 15, algo=0, sched=1, msg16=msg16), code.k())


@pytest.mark.parametrize("kind", ["layered_sfu16", "flooding_minsum"])
def test_mixed_host_pipeline_equals_device(gpu, kind):
    """A mixed batch from host memory large enough for the pipelined path
    (chunks of frames in memory order, copies on their own stream, each
    chunk's frame order made on the host) gives the device call's results;
    frames are laid out code by code, not in frame order."""
    import torch
    codes = [g.LdpcCode.dvb_t2_short(0), g.LdpcCode.dvb_t2_normal(1), g.LdpcCode.dvb_t2_short(2)]
    kw = (dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
          if kind == "layered_sfu16" else {})
    dec = g.LdpcDecoder(codes[0], codes=codes, **kw)
    rng = np.random.default_rng(12)
    F = 2500
    cid = rng.choice(3, F, p=[0.45, 0.1, 0.45]).astype(np.int32)
    mit = rng.integers(5, 30, F).astype(np.int32)
    ebn0 = [1.2, 1.1, 2.2]
    parts, lo, base = [], np.zeros(F, np.int64), 0
    for c in range(3):
        idx = np.nonzero(cid == c)[0]
        s2 = np.array([g.sigma2_from_ebn0(ebn0[c] + 0.1 * (i % 5), codes[c].rate()) for i in idx])
        _, _, l = g.awgn_frames(codes[c], 10, c << 20, len(idx), s2, device=gpu, want_info=False, want_cw=False)
        parts.append(l.reshape(-1))
        lo[idx] = base + np.arange(len(idx)) * codes[c].n()
        base += len(idx) * codes[c].n()
    llr = torch.cat(parts)
    assert llr.numel() * 4 >= 64 << 20
    W = max(g.words(c.k()) for c in codes)
    mo = np.arange(F, dtype=np.int64) * W
    d = dict(msg=torch.zeros(F * W, dtype=torch.int64, device=gpu), iters=torch.zeros(F, dtype=torch.int32, device=gpu),
             conv=torch.zeros(F, dtype=torch.uint8, device=gpu), so=torch.zeros(F, dtype=torch.uint8, device=gpu))
    dt = lambda x: torch.from_numpy(x).to(gpu)
    dec.decode_mixed_tensors(llr, dt(lo), dt(cid), dt(mit), d["msg"], dt(mo), d["iters"], d["conv"], d["so"],
                             use_graph=False)
    torch.cuda.synchronize()
    h = dec.decode_mixed_arrays(llr.cpu().numpy(), lo, cid, mit, mo)
    assert dec.last_launches() > 2  # several chunks
    assert (h["iters"] == d["iters"].cpu().numpy()).all()
    assert (h["conv"] == d["conv"].cpu().numpy().astype(bool)).all()
    assert (h["synd_ok"] == d["so"].cpu().numpy().astype(bool)).all()
    hm = h["msg"].view(np.int64)
    assert (hm == d["msg"].cpu().numpy()[:hm.size]).all()


@pytest.mark.parametrize("idx,msg", [(1, g.MSG_F16), (1, g.MSG_F32), (6, g.MSG_F16), (5, g.MSG_F16), (5, g.MSG_F32)])
def test_layered_compressed_states_equal_per_edge_messages(gpu, monkeypatch, idx, msg):
    """The single-code min-sum family kernels keep one compressed state per
    check; with staging disabled the decoder runs the per-edge-message kernel.
    Both give bit-identical results (normal 3/5 and 5/6: repeated-variable row
    groups; short 1/2: posteriors in shared memory; FP16 and FP32 messages)."""
    import torch
    code = dvb(idx)
    L = code.layers()
    rng = np.random.default_rng(30 + idx)
    kw = dict(algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, msg_dtype=msg,
              nms_alpha=(0.7 + 0.3 * rng.random((6, L))).astype(np.float32),
              nms_beta=(0.3 * rng.random((6, L))).astype(np.float32))
    ebn0 = {1: 1.3, 6: 1.4, 5: 3.3}[idx]
    _, _, llr = g.awgn_frames(code, 19, 0, 300, g.sigma2_from_ebn0(ebn0, code.rate()), device=gpu,
                              want_info=False, want_cw=False)
    states = g.LdpcDecoder(code, **kw).decode_tensors(llr, 25, beliefs=True)
    monkeypatch.setenv("GF2C_NO_STAGE", "1")
    per_edge = g.LdpcDecoder(code, **kw).decode_tensors(llr, 25, beliefs=True)
    torch.cuda.synchronize()
    for key in ("msg", "iters", "conv", "synd_ok"):
        assert torch.equal(states[key], per_edge[key]), key
    assert torch.equal(states["beliefs"].view(torch.int32), per_edge["beliefs"].view(torch.int32))


def test_mixed_batch_two_checks_per_thread(gpu):
    """A mixed batch at 192 threads (two checks per thread, posteriors in the
    workspace) gives the one-check-per-thread mixed decoder's results on every
    frame, short and normal codes, with repeated-variable row groups."""
    import torch
    codes = [g.LdpcCode.dvb_t2_short(0), g.LdpcCode.dvb_t2_normal(1), g.LdpcCode.dvb_t2_short(4),
             g.LdpcCode.dvb_t2_normal(5)]
    kw = dict(algorithm=g.ALGO_SPA_FAST, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16)
    rng = np.random.default_rng(21)
    F = 1200
    cid = rng.integers(0, 4, F).astype(np.int32)
    mit = rng.integers(5, 40, F).astype(np.int32)
    ebn0 = [1.2, 1.1, 2.6, 3.3]
    parts, lo, base = [], np.zeros(F, np.int64), 0
    for c in range(4):
        idx = np.nonzero(cid == c)[0]
        s2 = np.array([g.sigma2_from_ebn0(ebn0[c] + 0.1 * (i % 5), codes[c].rate()) for i in idx])
        _, _, l = g.awgn_frames(codes[c], 23, c << 20, len(idx), s2, device=gpu, want_info=False, want_cw=False)
        parts.append(l.reshape(-1))
        lo[idx] = base + np.arange(len(idx)) * codes[c].n()
        base += len(idx) * codes[c].n()
    llr = torch.cat(parts)
    W = max(g.words(c.k()) for c in codes)
    dt = lambda x: torch.from_numpy(x).to(gpu)
    res = []
    for threads in (0, 192):
        dec = g.LdpcDecoder(codes[0], codes=codes, threads_per_block=threads, **kw)
        o = dict(msg=torch.zeros(F * W, dtype=torch.int64, device=gpu), it=torch.zeros(F, dtype=torch.int32, device=gpu),
                 cv=torch.zeros(F, dtype=torch.uint8, device=gpu), so=torch.zeros(F, dtype=torch.uint8, device=gpu))
        dec.decode_mixed_tensors(llr, dt(lo), dt(cid), dt(mit), o["msg"], dt(np.arange(F, dtype=np.int64) * W), o["it"],
                                 o["cv"], o["so"], use_graph=False)
        torch.cuda.synchronize()
        res.append(o)
    for k in ("msg", "it", "cv", "so"):
        assert torch.equal(res[0][k], res[1][k]), k


@pytest.mark.parametrize("msg16", [True, False])
def test_layered_nms_special_llrs_equal_oracle(gpu, oracle, msg16):
    """Layered normalised / offset min-sum with +-inf, NaN and +-0 channel
    values among ordinary ones: iterations, flags and decisions equal the
    oracle's, posteriors bitwise equal where the oracle's is a number and NaN
    where it is NaN (a NaN magnitude is never a check's minimum on either
    side)."""
    code = g.LdpcCode.dvb_t2_short(g.CodeRate.Rate1_2)
    ocode = oracle.Code.dvbt2(1, 0)
    _, _, llr = ocode.channel(31, 0, 12, 2.0)
    llr = llr.copy()
    rng = np.random.default_rng(8)
    for f in range(12):
        idx = rng.choice(code.n(), 40, replace=False)
        llr[f, idx[:10]] = np.inf
        llr[f, idx[10:20]] = -np.inf
        llr[f, idx[20:25]] = np.nan if f % 3 == 0 else 0.0
        llr[f, idx[25:30]] = -0.0
    T, L = 6, code.layers()
    a = (0.7 + 0.3 * rng.random((T, L))).astype(np.float32)
    b = (0.3 * rng.random((T, L))).astype(np.float32)
    kw = dict(algorithm=g.ALGO_NMS, schedule=g.SCHED_LAYERED, msg_dtype=g.MSG_F16 if msg16 else g.MSG_F32,
              nms_alpha=a, nms_beta=b)
    r = g.LdpcDecoder(code, **kw).decode_arrays(llr, 15, beliefs=True)
    o = ocode.decode(llr, 15, algo=3, sched=1, msg16=msg16, alpha=a, beta=b)
    assert (r["iters"] == o["iters"]).all() and (r["conv"] == o["conv"]).all()
    assert (r["synd_ok"] == o["synd_ok"]).all()
    assert (unpack_msg(r, code.k()) == o["msg"]).all()
    gb, ob = r["beliefs"], o["beliefs"]
    nan = np.isnan(ob)
    assert (np.isnan(gb) == nan).all()
    assert (gb[~nan].view(np.uint32) == ob[~nan].view(np.uint32)).all()
