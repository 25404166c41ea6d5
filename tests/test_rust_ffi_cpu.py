"""The Rust binding crate (rblas_b200/rust/rblas-gpu) against the C header.

This image has no Rust toolchain, so the crate's `extern "C"` declarations
are checked here instead: every function the crate declares (directly, or
through its declaration macros) must exist in include/rblas_b200.h with the
same number of parameters, each parameter must have the matching type
(size_t <-> usize, double <-> f64, the enums <-> i32, ...), and each pointer
parameter must agree in mutability (`const T*` <-> `*const`, `T*` <->
`*mut`)."""
from __future__ import annotations

import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rblas_b200.h")
CRATE = os.path.join(ROOT, "rblas_b200", "rust", "rblas-gpu", "src", "lib.rs")


def _split_params(params: str):
    params = params.strip()
    if not params or params == "void":
        return []
    return [p.strip() for p in params.split(",")]


def header_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(rb_\w+)\s*\(([^;{}]*?)\)\s*;", text):
        out[m.group(1)] = _split_params(" ".join(m.group(2).split()))
    return out


def _c_kind(p: str) -> str:
    if "*" not in p:
        return "value"
    return "const" if p.startswith("const ") else "mut"


def _rust_kind(p: str) -> str:
    ty = p.split(":", 1)[1].strip()
    if ty.startswith("*const"):
        return "const"
    if ty.startswith("*mut"):
        return "mut"
    return "value"


# C parameter types and the Rust types that carry them across the ABI
_C_TO_RUST = {
    "size_t": "usize", "float": "f32", "double": "f64", "int": "i32", "int32_t": "i32", "uint32_t": "u32",
    "uint64_t": "u64", "int64_t": "i64", "rb_layout": "i32", "rb_transpose": "i32", "rb_uplo": "i32",
    "rb_side": "i32", "rb_diag": "i32", "rb_precision": "i32", "rb_complex32": "C32", "rb_complex64": "C64",
    "rb_error": "RbError", "void": "c_void", "char": "c_char", "rb_gemm_problem": "RbGemmProblem",
    "rb_request_times": "RbRequestTimes",
}
_RUST_ALIASES = {"Complex<f32>": "C32", "Complex<f64>": "C64"}


def _c_base(p: str) -> str:
    """The element type of a C parameter (`const double* x` -> f64)."""
    words = p.replace("*", " ").split()
    words = [w for w in words if w != "const"]
    return _C_TO_RUST.get(words[0], words[0])


def _rust_base(p: str) -> str:
    ty = p.split(":", 1)[1].strip()
    while ty.startswith(("*const", "*mut")) and " " in ty:
        ty = ty.split(None, 1)[1].strip()
    return _RUST_ALIASES.get(ty, ty)


def _c_depth(p: str) -> int:
    return p.count("*")


def _rust_depth(p: str) -> int:
    return p.split(":", 1)[1].count("*")


def _check_decls(where: str, decls: dict, hdr: dict):
    for name, params in decls.items():
        assert name in hdr, f"{where}: {name} is not declared in the header"
        cp = hdr[name]
        assert len(params) == len(cp), f"{where}: {name}: {len(params)} parameters, {len(cp)} in the header"
        for rp, c in zip(params, cp):
            assert _rust_kind(rp) == _c_kind(c), f"{where}: {name}: `{rp}` against `{c}`"
            assert _rust_depth(rp) == _c_depth(c), f"{where}: {name}: `{rp}` against `{c}`"
            assert _rust_base(rp) == _c_base(c), f"{where}: {name}: `{rp}` against `{c}`"


def crate_functions():
    text = re.sub(r"//[^\n]*", "", open(CRATE).read())
    ffi = text[text.index("pub mod ffi"):]
    out = {}
    # direct declarations: `pub fn rb_x(...) -> ...;`
    for m in re.finditer(r"pub fn (rb_\w+)\s*\(([^)]*)\)", ffi):
        out[m.group(1)] = _split_params(" ".join(m.group(2).split()))
    # declaration macros: `macro_rules! name { ($t:ty, $a:ident, ...) => { extern "C" { pub fn $a(...) ... } } }`
    for mm in re.finditer(r"macro_rules!\s+(\w+)\s*\{\s*\((.*?)\)\s*=>\s*\{(.*?)\n    \}", ffi, re.S):
        name, pattern, body = mm.group(1), mm.group(2), mm.group(3)
        metas = [v.strip().split(":")[0] for v in pattern.split(",")]
        decls = [(d.group(1), d.group(2)) for d in re.finditer(r"pub fn (\$\w+)\s*\(([^)]*)\)", body)]
        for inv in re.finditer(name + r"!\s*\(([^)]*)\)\s*;", ffi):
            args = [a.strip() for a in inv.group(1).split(",")]
            sub = dict(zip(metas, args))
            for meta, params in decls:
                p = " ".join(params.split())
                for k, v in sorted(sub.items(), key=lambda kv: -len(kv[0])):
                    p = p.replace(k, v)
                out[sub[meta]] = _split_params(p)
    return out


def test_crate_declares_functions():
    fns = crate_functions()
    # Level 3, Level 2 and Level 1 entry points are all bound
    for name in ("rb_sgemm_prec", "rb_zgemm", "rb_dtrsm", "rb_daxpy", "rb_zdotc", "rb_dznrm2", "rb_cgemv",
                 "rb_zgerc", "rb_sger"):
        assert name in fns, name


def test_crate_ffi_matches_header():
    _check_decls("crate", crate_functions(), header_functions())


def test_integration_guide_ffi_matches_header():
    """The `extern "C"` snippets of the integration guide, the block a
    maintainer copies into rblas, hold the header's signatures too."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    decls = {}
    for block in re.findall(r"```rust\n(.*?)```", text, re.S):
        block = re.sub(r"//[^\n]*", "", block)
        for m in re.finditer(r"fn (rb_\w+)\s*\(([^)]*)\)", block):
            decls[m.group(1)] = _split_params(" ".join(m.group(2).split()))
    assert len(decls) >= 20
    _check_decls("INTEGRATION.md", decls, header_functions())
