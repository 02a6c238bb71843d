"""The three descriptions of the C ABI agree: the header `include/sbp_b200.h`, the Rust `-sys`
binding given in INTEGRATION.md (the `extern "C"` block and the `#[repr(C)]` structs a Rust
caller of the reference's API would compile), and the ctypes binding the Python host side uses
(`summationbyparts_b200/_capi.py`).  Every exported function must appear in all three with the
same parameter types, and the structs must have the same fields in the same order, so a
mismatch cannot corrupt memory on the other side of the boundary.  CPU only: nothing is loaded.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sbp_b200.h")
INTEGRATION = os.path.join(ROOT, "INTEGRATION.md")

C_BASE_TO_RUST = {
    "int": "c_int", "int64_t": "i64", "int32_t": "i32", "double": "f64", "float": "f32", "void": "c_void",
    "char": "c_char", "unsigned long long": "u64", "sbp_system": "sbp_system", "sbp_cnn": "sbp_cnn",
    "sbp_block_desc": "sbp_block_desc", "sbp_vortex_params": "sbp_vortex_params", "sbp_status": "sbp_status",
}
C_SCALAR_TO_CTYPES = {"int": ctypes.c_int, "sbp_status": ctypes.c_int, "int64_t": ctypes.c_int64,
                      "double": ctypes.c_double, "float": ctypes.c_float,
                      "unsigned long long": ctypes.c_ulonglong}


def _strip_c_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def _c_type(decl: str, has_name: bool = True) -> str:
    """Rust spelling of one C parameter (or, with has_name False, return) declaration.

    levels[0] is the base type's const-ness; every `*` adds a pointer level whose own const-ness
    a following `const` sets; an array parameter decays to one more pointer level.  A pointer
    is `*const` when the level it points to is const."""
    decl = " ".join(decl.split())
    array = re.search(r"\[\s*\d*\s*\]\s*$", decl)
    if array:
        decl = decl[:array.start()].strip()
    if has_name:
        decl = re.sub(r"\b\w+\s*$", "", decl).strip()
    base_words, levels = [], [False]
    for tok in re.findall(r"\*|[A-Za-z_][A-Za-z0-9_]*", decl):
        if tok == "*":
            levels.append(False)
        elif tok == "const":
            levels[-1] = True
        else:
            base_words.append(tok)
    if array:
        levels.append(False)
    out = C_BASE_TO_RUST[" ".join(base_words)]
    for i in range(1, len(levels)):
        out = ("*const " if levels[i - 1] else "*mut ") + out
    return out


def header_functions() -> dict:
    text = _strip_c_comments(open(HEADER).read())
    funcs = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(sbp_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        ret = ret.split("\n")[-1].strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        funcs[name] = (ret, plist)
    return funcs


def header_struct(name: str) -> list:
    """(field, Rust type) of a header struct, in order; `T a, b[4]` declares two fields."""
    text = _strip_c_comments(open(HEADER).read())
    m = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + r"\s*;", text, flags=re.S)
    assert m, name
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        items = decl.split(",")
        first = re.match(r"(.*?)(\**\s*\w+\s*(\[\s*\d+\s*\])?)$", items[0].strip())
        prefix = first.group(1).strip()
        for k, item in enumerate(items):
            item = item.strip() if k else first.group(2).strip()
            stars = "*" * item.count("*")
            item = item.replace("*", "").strip()
            am = re.match(r"(\w+)\s*(\[\s*(\d+)\s*\])?$", item)
            t = _c_type(f"{prefix}{stars} {am.group(1)}")
            fields.append((am.group(1), f"[{t}; {am.group(3)}]" if am.group(3) else t))
    return fields


def rust_block() -> str:
    text = open(INTEGRATION).read()
    blocks = re.findall(r"```rust\n(.*?)```", text, flags=re.S)
    sys_blocks = [b for b in blocks if 'extern "C"' in b]
    assert len(sys_blocks) == 1, "INTEGRATION.md holds exactly one extern \"C\" block"
    return re.sub(r"//[^\n]*", " ", sys_blocks[0])


def rust_functions() -> dict:
    body = rust_block()
    funcs = {}
    for m in re.finditer(r"pub fn (sbp_\w+)\s*\((.*?)\)\s*(->\s*([^;]+))?;", body, flags=re.S):
        name, params, ret = m.group(1), m.group(2), (m.group(4) or "").strip()
        types = []
        for p in [p for p in params.split(",") if p.strip()]:
            _, _, t = p.partition(":")
            types.append(" ".join(t.split()))
        assert name not in funcs, f"{name} declared twice in INTEGRATION.md"
        funcs[name] = (ret, types)
    return funcs


def rust_struct(name: str) -> list:
    body = rust_block()
    m = re.search(r"pub struct " + name + r"\s*\{(.*?)\n\}", body, flags=re.S)
    assert m, f"struct {name} missing from INTEGRATION.md"
    out = []
    for item in re.findall(r"pub (\w+)\s*:\s*([^,\n]+(?:\[[^\]]*\])?)", m.group(1)):
        out.append((item[0], " ".join(item[1].strip().rstrip(",").split())))
    return out


def test_rust_extern_block_matches_header():
    hdr, rust = header_functions(), rust_functions()
    assert sorted(hdr) == sorted(rust), (sorted(set(hdr) - set(rust)), sorted(set(rust) - set(hdr)))
    for name, (ret, params) in hdr.items():
        rret, rtypes = rust[name]
        want = [_c_type(p) for p in params]
        assert rtypes == want, (name, rtypes, want)
        want_ret = _c_type(ret, has_name=False)
        if want_ret == "sbp_status":
            assert rret == "sbp_status", (name, rret)
        else:
            assert rret == want_ret, (name, rret, want_ret)


@pytest.mark.parametrize("name", ["sbp_block_desc", "sbp_vortex_params"])
def test_rust_structs_match_header(name):
    assert rust_struct(name) == header_struct(name)


def test_ctypes_binding_matches_header():
    from summationbyparts_b200 import _capi
    hdr = header_functions()
    assert sorted(hdr) == sorted(_capi.SIGNATURES)
    for name, (ret, params) in hdr.items():
        res, args = _capi.SIGNATURES[name]
        assert len(args) == len(params), name
        for p, a in zip(params, args):
            t = _c_type(p)
            if t.startswith("*"):
                assert a is ctypes.c_void_p or a is ctypes.c_char_p or issubclass(a, ctypes._Pointer), (name, p)
            else:
                base = " ".join(re.sub(r"\b\w+\s*$", "", " ".join(p.split())).split())
                assert a is C_SCALAR_TO_CTYPES[base], (name, p, a)
        rt = _c_type(ret, has_name=False)
        if rt.startswith("*"):
            assert res is ctypes.c_char_p, name
        else:
            assert res is C_SCALAR_TO_CTYPES[" ".join(ret.split())], name
    for cname, cls in (("sbp_block_desc", _capi.BlockDesc), ("sbp_vortex_params", _capi.VortexParams)):
        names = [f for f, _ in header_struct(cname)]
        assert [f for f, _ in cls._fields_] == names, cname
