"""gf2 file formats and the encoder cache on the CPU: byte layouts of the
reference's GF2DATA files (crates/gf2-core/src/io/{format,header,bitvec,matrix,
sparse,formats}.rs and their tests), SipHash-1-3 against CPython's own
SipHash-1-3 (the string hash with hash randomisation off), and the dense parity
part against the oracle encoder."""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

import gf2_b200 as g
from gf2_b200 import gf2io


def header(b):
    assert b[:8] == b"GF2DATA\0"
    version, tag, flags = struct.unpack_from("<HBB", b, 8)
    assert b[12:20] == b"\0" * 8
    mlen, dlen = struct.unpack_from("<IQ", b, 20)
    return version, tag, flags, b[32:32 + mlen], b[32 + mlen:], dlen


def test_bitvec_binary_layout(tmp_path):
    # io/bitvec.rs: test_bitvec_write_has_correct_header; metadata = serde_json of BitVecMetadata
    rng = np.random.default_rng(0)
    bits = rng.integers(0, 2, 100).astype(np.uint8)
    p = tmp_path / "v.gf2"
    gf2io.save_bitvec(p, bits)
    b = p.read_bytes()
    version, tag, flags, meta, payload, dlen = header(b)
    assert (version, tag, flags) == (1, 1, 0)
    assert meta == b'{"type":"BitVec","len_bits":100,"version":1}'
    assert dlen == len(payload) == 16
    w = np.frombuffer(payload, "<u8")
    assert (w == g.pack_bits(bits, 100)[0]).all()
    assert (gf2io.load_bitvec(p) == bits).all()
    assert gf2io.probe(p) == (1, 0, (100, 0, 0))


@pytest.mark.parametrize("n", [0, 1, 64, 100, 1000, 4097])
@pytest.mark.parametrize("fmt", ["binary", "text", "hex"])
def test_bitvec_roundtrip(tmp_path, n, fmt):
    # io/bitvec.rs roundtrip tests (empty, single bit, one word, multiple words, not aligned, large)
    bits = np.random.default_rng(n).integers(0, 2, n).astype(np.uint8)
    p = tmp_path / f"v.{fmt}"
    gf2io.save_bitvec(p, bits, fmt)
    if n:
        assert (gf2io.load_bitvec(p) == bits).all()
        assert gf2io.probe(p)[1] == {"binary": 0, "text": 1, "hex": 2}[fmt] or (fmt == "hex" and n < 128)
    else:
        assert gf2io.load_bitvec(p).size == 0


def test_bitvec_text_and_hex_layout(tmp_path):
    # io/bitvec.rs: test_bitvec_text_format / test_bitvec_hex_format
    bits = np.zeros(100, np.uint8)
    bits[::3] = 1
    gf2io.save_bitvec(tmp_path / "t.txt", bits, "text")
    t = (tmp_path / "t.txt").read_text()
    assert t.startswith("100\n") and t.split("\n")[1] == "".join(map(str, bits[:80]))
    h = np.zeros(128, np.uint8)
    h[5] = h[70] = 1
    gf2io.save_bitvec(tmp_path / "h.hex", h, "hex")
    assert (tmp_path / "h.hex").read_text() == "128\n%016X\n%016X\n" % (1 << 5, 1 << 6)
    assert (gf2io.load_bitvec(tmp_path / "h.hex") == h).all()


def test_bitvec_tail_masking(tmp_path):
    # io/bitvec.rs: test_bitvec_preserves_tail_masking
    w = np.array([~np.uint64(0)], np.uint64)
    gf2io.save_bitvec(tmp_path / "m.gf2", w, len_bits=10)
    got, n = gf2io.load_bitvec_words(tmp_path / "m.gf2")
    assert n == 10 and int(got[0]) == (1 << 10) - 1


def test_bad_files(tmp_path):
    # header.rs: test_header_read_invalid_magic / unsupported_version; bitvec.rs: test_bitvec_read_wrong_type
    p = tmp_path / "bad.gf2"
    p.write_bytes(b"BADMAGIC" + b"\0" * 24)
    with pytest.raises(ValueError):
        gf2io.load_bitmatrix(p)
    p.write_bytes(b"GF2DATA\0" + struct.pack("<H", 99) + b"\0" * 22)
    with pytest.raises(g._capi.Gf2cError):
        gf2io.load_bitmatrix(p)
    gf2io.save_bitvec(p, np.ones(10, np.uint8))
    with pytest.raises(ValueError):
        gf2io.load_bitmatrix(p)


@pytest.mark.parametrize("shape", [(0, 0), (1, 1), (3, 64), (7, 100), (40, 129)])
@pytest.mark.parametrize("fmt", ["binary", "text", "hex"])
def test_bitmatrix_roundtrip_and_layout(tmp_path, shape, fmt):
    m = np.random.default_rng(sum(shape)).integers(0, 2, shape).astype(np.uint8)
    p = tmp_path / f"m.{fmt}"
    gf2io.save_bitmatrix(p, m, fmt)
    assert (gf2io.load_bitmatrix(p, fmt) == m).all()
    rows, cols = shape
    if fmt == "binary":
        version, tag, flags, meta, payload, dlen = header(p.read_bytes())
        assert (version, tag) == (1, 2)
        assert meta == b'{"type":"BitMatrix","rows":%d,"cols":%d,"version":1}' % (rows, cols)
        S = (cols + 63) // 64 if cols else 0
        assert dlen == len(payload) == rows * S * 8
    elif fmt == "text":
        assert p.read_text().split("\n")[0] == f"{rows} {cols}"


def test_sparse_layouts_and_code_files(tmp_path):
    code = g.LdpcCode.dvb_t2_short(0)
    ptr, idx = code.csr()
    m, n, nnz = code.m(), code.n(), code.nnz()
    # SpBitMatrix: COO pairs in CSR order, u32
    gf2io.save_code(tmp_path / "h.gf2", code, dual=False)
    version, tag, flags, meta, payload, dlen = header((tmp_path / "h.gf2").read_bytes())
    assert tag == 3 and meta == (b'{"type":"SpBitMatrix","rows":%d,"cols":%d,"nnz":%d,"format":"coo","version":1}'
                                 % (m, n, nnz))
    pairs = np.frombuffer(payload, "<u4").reshape(-1, 2)
    assert (pairs[:, 1] == idx).all() and (pairs[:, 0] == np.repeat(np.arange(m), np.diff(ptr))).all()
    # SpBitMatrixDual: row offsets, column indices, column offsets, row indices
    gf2io.save_code(tmp_path / "d.gf2", code, dual=True)
    version, tag, flags, meta, payload, dlen = header((tmp_path / "d.gf2").read_bytes())
    assert tag == 4 and meta == b'{"type":"SpBitMatrixDual","rows":%d,"cols":%d,"nnz":%d,"version":1}' % (m, n, nnz)
    a = np.frombuffer(payload, "<u4")
    assert a.size == m + 1 + nnz + n + 1 + nnz
    assert (a[:m + 1] == ptr).all() and (a[m + 1:m + 1 + nnz] == idx).all()
    cptr, cidx = a[m + 1 + nnz:m + 2 + nnz + n], a[m + 2 + nnz + n:]
    rows_of = np.repeat(np.arange(m), np.diff(ptr))
    order = np.lexsort((rows_of, idx))  # CSC, rows ascending in each column
    assert (cidx == rows_of[order]).all() and (np.diff(cptr) == np.bincount(idx, minlength=n)).all()
    for name in ("h.gf2", "d.gf2"):
        c2 = gf2io.load_code(tmp_path / name)
        p2, i2 = c2.csr()
        assert (c2.m(), c2.n(), c2.k()) == (m, n, code.k()) and (p2 == ptr).all() and (i2 == idx).all()
    gf2io.save_code(tmp_path / "h.txt", code, dual=False, format="text")
    r, c, p3, i3 = gf2io.load_sparse(tmp_path / "h.txt")
    assert (r, c) == (m, n) and (p3 == ptr).all() and (i3 == idx).all()


def test_sparse_coo_duplicates_are_dropped(tmp_path):
    # SpBitMatrix::from_coo_deduplicated: sort each row, keep one of repeated edges
    p = tmp_path / "dup.gf2"
    gf2io.save_sparse(p, 3, 5, edges=[(0, 4), (0, 1), (2, 2)])
    b = bytearray(p.read_bytes())
    meta_len = struct.unpack_from("<I", b, 20)[0]
    meta = b[32:32 + meta_len].replace(b'"nnz":3', b'"nnz":4')
    payload = bytes(b[32 + meta_len:]) + struct.pack("<II", 0, 4)
    out = bytes(b[:20]) + struct.pack("<IQ", len(meta), len(payload)) + bytes(meta) + payload
    p.write_bytes(out)
    r, c, ptr, idx = gf2io.load_sparse(p)
    assert (r, c) == (3, 5) and list(ptr) == [0, 2, 2, 3] and list(idx) == [1, 4, 2]


def test_format_detection(tmp_path):
    # io/formats.rs SerializationFormat::detect
    cases = {"3\n101\n": 1, "2 2\n10\n01\n": 1, "128\n0000000000000000\n0000000000000001\n": 1,
             "64\n00000000000000AB\n": 2, "64\n1234567890123456\n": 2}
    for text, fmt in cases.items():
        p = tmp_path / "x"
        p.write_text(text)
        assert gf2io.probe(p)[1] == fmt, text


def cpython_siphash13(data):
    code = f"import sys; sys.stdout.write(str(hash({bytes(data)!r}) & ((1 << 64) - 1)))"
    env = dict(os.environ, PYTHONHASHSEED="0")
    return int(subprocess.check_output([sys.executable, "-c", code], env=env))


def test_siphash13_matches_cpython():
    # CPython hashes bytes with SipHash-1-3; PYTHONHASHSEED=0 zeroes its key, as Rust's DefaultHasher does
    if sys.hash_info.algorithm != "siphash13":
        pytest.skip("this interpreter does not hash with SipHash-1-3")
    rng = np.random.default_rng(5)
    msgs = [bytes(rng.integers(0, 256, L).astype(np.uint8)) for L in (1, 7, 8, 9, 15, 16, 24, 63, 100)]
    msgs.append(struct.pack("<3Q", 9000, 16200, 48599))
    got = [gf2io.siphash13(m) for m in msgs]
    want = [cpython_siphash13(m) for m in msgs]
    assert got == [w if w != (1 << 64) - 1 else w for w in want]


def test_cache_key_is_siphash_of_structure():
    # compute_matrix_hash (cache.rs:461-487): rows, cols, nnz, first 100 (row, col) as usize
    code = g.LdpcCode.dvb_t2_short(2)
    ptr, idx = code.csr()
    rows = np.repeat(np.arange(code.m()), np.diff(ptr))
    stream = struct.pack("<3Q", code.m(), code.n(), code.nnz())
    for r, c in list(zip(rows, idx))[:100]:
        stream += struct.pack("<2Q", r, c)
    n, k, h = gf2io.cache_key(code)
    assert (n, k, h) == (code.n(), code.k(), gf2io.siphash13(stream))
    assert gf2io.cache_filename((n, k, h)) == f"n16200_k{k}_h{h:x}.gf2"
    assert gf2io.parse_cache_filename(f"n16200_k{k}_h{h:x}") == (n, k, h)
    assert gf2io.parse_cache_filename("n1_k2") is None and gf2io.parse_cache_filename("x1_k2_h3") is None


@pytest.mark.parametrize("rate", [0, 3])
def test_parity_part_matches_oracle_encoder(oracle, rate):
    code = g.LdpcCode.dvb_t2_short(rate)
    ocode = oracle.Code.dvbt2(1, rate)
    P = gf2io.parity_part(code)
    k, r = code.k(), code.n() - code.k()
    Pb = g.unpack_bits(P, r)
    rng = np.random.default_rng(rate)
    msg = rng.integers(0, 2, (3, k)).astype(np.uint8)
    cw = ocode.encode(msg)
    par = (msg.astype(np.int64) @ Pb.astype(np.int64)) & 1
    assert (cw[:, k:] == par).all() and (cw[:, :k] == msg).all()


def test_parity_part_generic_qc_code(oracle):
    # parity part: lower bidiagonal identity blocks (invertible), so H has full rank
    base = [[1, 2, 0, 0, -1, -1], [0, -1, 3, 0, 0, -1], [2, 1, -1, -1, 0, 0]]
    qc = g.QuasiCyclicLdpc(np.array(base), 4)
    code = g.LdpcCode.from_quasi_cyclic(qc)
    try:
        P = gf2io.parity_part(code)
    except ValueError:
        pytest.skip("systematic columns of this code are not [0, k)")
    ptr, idx = code.csr()
    H = np.zeros((code.m(), code.n()), np.int64)
    H[np.repeat(np.arange(code.m()), np.diff(ptr)), idx] = 1
    G = np.concatenate([np.eye(code.k(), dtype=np.int64), g.unpack_bits(P, code.n() - code.k())], 1)
    assert not ((G @ H.T) & 1).any()


def test_cache_directory_roundtrip(tmp_path):
    cache = g.EncodingCache()
    code = g.LdpcCode.dvb_t2_short(5)
    P = cache.get_or_compute(code)
    cache.save_to_directory(tmp_path)
    names = os.listdir(tmp_path)
    assert names == [gf2io.cache_filename(gf2io.cache_key(code))]
    tag, fmt, dims = gf2io.probe(tmp_path / names[0])
    assert (tag, fmt, dims[:2]) == (2, 0, (code.k(), code.n() - code.k()))
    (tmp_path / "notes.txt").write_text("ignored")
    (tmp_path / "bad_name.gf2").write_bytes(b"")
    loaded = g.EncodingCache.from_directory(tmp_path)
    assert loaded.stats() == {"entries": 1} and (loaded.get(code) == P).all()
    with pytest.raises(FileNotFoundError):
        g.EncodingCache.from_directory(tmp_path / "missing")
