"""The Rust binding (crates/gf2-cuda) against the C header, on the CPU.

No Rust toolchain exists in this image, so the crate is checked as text: every
function of include/gf2cuda.h has exactly one `extern "C"` declaration in
crates/gf2-cuda/src/ffi.rs with the same name, argument count, argument types
and return type; every status / enum #define has a Rust const of the same
value; the options struct has the same fields in the same order.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gf2cuda.h")
FFI = os.path.join(ROOT, "crates", "gf2-cuda", "src", "ffi.rs")

C_SCALAR = {"int32_t": "i32", "int64_t": "i64", "uint64_t": "u64", "uint16_t": "u16", "uint8_t": "u8",
            "float": "f32", "double": "f64", "int": "i32", "char": "c_char", "void": "c_void"}


def c_type_to_rust(t):
    """Map one C parameter type (without the name) to the Rust spelling."""
    t = " ".join(t.replace("*", " * ").split())
    toks = t.split()
    # pointer levels with constness, read right to left: "const gf2c_code * const *"
    base_const = toks[0] == "const"
    if base_const:
        toks = toks[1:]
    base = toks[0]
    rest = toks[1:]
    rust = C_SCALAR.get(base, base)
    levels = []
    i = 0
    while i < len(rest):
        if rest[i] == "*":
            const_after = i + 1 < len(rest) and rest[i + 1] == "const"
            levels.append(const_after)
            i += 2 if const_after else 1
        else:
            i += 1
    if not levels:
        return rust
    # the innermost pointer's constness is the base's
    quals = [base_const] + levels[:-1]
    for q in quals:
        rust = ("*const " if q else "*mut ") + rust
    return rust


def header_functions():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*([a-z][\w\s\*]*?)\b(gf2c_\w+)\s*\(([^)]*)\)\s*;", src, flags=re.M):
        ret, name, args = m.group(1).strip(), m.group(2), " ".join(m.group(3).split())
        params = []
        if args != "void":
            for a in args.split(","):
                a = a.strip()
                mm = re.match(r"^(.*?)(\w+)$", a)
                params.append(c_type_to_rust(mm.group(1).strip()))
        rret = {"int": "i32", "void": None, "double": "f64", "const char*": "*const c_char"}[ret]
        assert name not in out, name
        out[name] = (params, rret)
    return out


def rust_functions():
    src = open(FFI).read()
    block = src[src.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (gf2c_\w+)\s*\(([^)]*)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        name, args, ret = m.group(1), " ".join(m.group(2).split()), m.group(3)
        params = []
        if args.strip():
            for a in args.split(","):
                a = a.strip()
                if a:
                    params.append(a.split(":", 1)[1].strip())
        assert name not in out, name
        out[name] = (params, ret.strip() if ret else None)
    return out


def test_every_header_function_has_a_matching_rust_declaration():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 40
    assert sorted(h) == sorted(r), (set(h) ^ set(r))
    for name, (params, ret) in h.items():
        rp, rr = r[name]
        assert len(rp) == len(params), f"{name}: {len(rp)} Rust arguments, {len(params)} in C"
        assert rp == params, f"{name}: Rust {rp} vs C {params}"
        assert rr == ret, f"{name}: Rust returns {rr}, C {ret}"


def test_constants_match():
    src = open(HEADER).read()
    defs = dict(re.findall(r"#define (GF2C_[A-Z0-9_]+) (-?\d+)", src))
    rs = dict(re.findall(r"pub const (GF2C_[A-Z0-9_]+): i32 = (-?\d+);", open(FFI).read()))
    assert rs, "no constants in ffi.rs"
    for k, v in rs.items():
        assert k in defs, f"{k} is not defined in the header"
        assert defs[k] == v, f"{k}: Rust {v}, C {defs[k]}"
    for k in defs:
        if k.startswith(("GF2C_ERR_", "GF2C_ALGO_", "GF2C_SCHED_", "GF2C_MSG_", "GF2C_MEM_")) or k == "GF2C_OK":
            assert k in rs, f"{k} missing in ffi.rs"


def test_options_struct_layout_matches():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct \{(.*?)\} gf2c_decoder_opts;", src, flags=re.S).group(1)
    c_fields = [(m.group(2), c_type_to_rust(m.group(1))) for m in
                re.finditer(r"([\w\s\*]+?)\s*\b(\w+);", body)]
    rsrc = open(FFI).read()
    rbody = re.search(r"pub struct gf2c_decoder_opts \{(.*?)\}", rsrc, flags=re.S).group(1)
    r_fields = re.findall(r"pub (\w+): ([^,]+),", rbody)
    assert [(n, t.strip()) for n, t in r_fields] == c_fields


def test_crate_files_present():
    for rel in ("Cargo.toml", "build.rs", "src/lib.rs", "src/ffi.rs"):
        assert os.path.exists(os.path.join(ROOT, "crates", "gf2-cuda", rel)), rel
    lib = open(os.path.join(ROOT, "crates", "gf2-cuda", "src", "lib.rs")).read()
    for trait in ("impl IterativeSoftDecoder for CudaLdpcDecoder", "impl SoftDecoder for CudaLdpcDecoder",
                  "impl BlockEncoder for CudaLdpcEncoder", "pub fn decode_batch("):
        assert trait in lib, trait
