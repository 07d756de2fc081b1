"""DVB-T2 outer BCH code on the CPU: the oracle restatement pinned by the
reference's own tests (crates/gf2-coding/src/bch/dvb_t2/{params.rs, mod.rs,
generators.rs}), and the library's host-side code construction against it."""
import numpy as np
import pytest

import gf2_b200 as g

# (frame, rate) -> (n, k, t, m), bch/dvb_t2/params.rs:56-85 and its tests
PARAMS = {
    (1, 0): (7200, 7032, 12, 14), (1, 1): (9720, 9552, 12, 14), (1, 2): (10800, 10632, 12, 14),
    (1, 3): (11880, 11712, 12, 14), (1, 4): (12600, 12432, 12, 14), (1, 5): (13320, 13152, 12, 14),
    (0, 0): (32400, 32208, 12, 16), (0, 1): (38880, 38688, 12, 16), (0, 2): (43200, 43040, 10, 16),
    (0, 3): (48600, 48408, 12, 16), (0, 4): (51840, 51648, 12, 16), (0, 5): (54000, 53840, 10, 16),
}


@pytest.mark.parametrize("frame,rate", sorted(PARAMS))
def test_params_and_generator(oracle, frame, rate):
    n, k, t, m = PARAMS[(frame, rate)]
    b = oracle.Bch(frame, rate)
    assert (b.n, b.k, b.t, b.field_m) == (n, k, t, m)
    # generator degree = n - k = t m (mod.rs tests: 168 short, 192 / 160 normal)
    assert b.gen_degree == n - k == t * m
    lib = g.BchCode.dvb_t2(frame, rate)
    assert (lib.n(), lib.k(), lib.t(), lib.field_m) == (n, k, t, m)
    assert (lib.generator() == b.generator()).all()


def test_generator_is_product_of_first_t_factors(oracle):
    # generators.rs: g = g_1 ... g_t; g_1 is the field's primitive polynomial
    b = oracle.Bch(1, 0)
    gen = b.generator()
    assert gen[0] == 1 and gen[-1] == 1
    prim = [0, 1, 3, 5, 14]  # x^14 + x^5 + x^3 + x + 1 (params.rs short frames)
    # g_1 divides g: long division over GF(2) leaves no remainder
    r = gen.copy()
    for d in range(len(r) - 1, 13, -1):
        if r[d]:
            for e in prim:
                r[d - 14 + e] ^= 1
    assert not r[:14].any()


@pytest.mark.parametrize("frame", [1, 0])
def test_roundtrip_all_ones_and_zero(oracle, frame):
    # mod.rs: test_short/normal_frame_encode_decode_roundtrip, test_all_configurations_encodable
    b = oracle.Bch(frame, 0)
    ones = np.ones((1, b.k), np.uint8)
    cw = b.encode(ones)
    assert cw.shape == (1, b.n) and (cw[0, :b.k] == 1).all()
    msg, flips = b.decode(cw)
    assert (msg == ones).all() and flips[0] == 0
    zero = b.encode(np.zeros((1, b.k), np.uint8))
    assert not zero.any()


@pytest.mark.parametrize("frame,rate", [(1, 3), (0, 2)])
def test_codewords_and_t_errors(oracle, frame, rate):
    b = oracle.Bch(frame, rate)
    rng = np.random.default_rng(frame * 10 + rate)
    msg = rng.integers(0, 2, (4, b.k)).astype(np.uint8)
    cw = b.encode(msg)
    assert not b.syndromes(cw).any()  # S_1..S_2t vanish on codewords
    bad = cw.copy()
    for f in range(4):
        bad[f, rng.choice(b.n, size=b.t, replace=False)] ^= 1
    dm, flips = b.decode(bad)
    assert (dm == msg).all() and (flips == b.t).all()
    # Berlekamp-Massey: the locator of t errors has degree t
    assert len(b.berlekamp_massey(b.syndromes(bad[:1])[0])) == b.t + 1
