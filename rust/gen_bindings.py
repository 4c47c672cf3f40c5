"""Generate rust/src/ffi.rs from include/hdc.h.

The role bindgen plays for mwa_hyperdrive's src/gpu headers
(gpu/update_rust_bindings.sh): every #define constant, struct and function
of the C header as Rust FFI declarations, so that the crate and the header
cannot drift apart.  Run after changing include/hdc.h:

    python rust/gen_bindings.py            # rewrite rust/src/ffi.rs
    python rust/gen_bindings.py --check    # exit 1 if ffi.rs is stale

The parser covers the C that include/hdc.h uses (typedef structs of scalars
and pointers, opaque struct typedefs, prototypes with pointer and fixed-size
array parameters, integer #defines) and fails loudly on anything else.
"""

from __future__ import annotations

import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
HEADER = HERE.parent / "include" / "hdc.h"
OUT = HERE / "src" / "ffi.rs"

SCALARS = {"int": "c_int", "unsigned int": "c_uint", "long long": "c_longlong", "unsigned long long": "c_ulonglong",
           "double": "f64", "float": "f32", "size_t": "usize", "char": "c_char", "unsigned char": "c_uchar",
           "void": "c_void", "int64_t": "i64", "uint64_t": "u64", "int32_t": "i32", "uint32_t": "u32"}
RUST_KEYWORDS = {"type", "match", "ref", "move", "fn", "in", "loop", "use", "mod", "impl", "self", "box"}


def strip_comments(txt: str) -> str:
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return re.sub(r"//[^\n]*", "", txt)


def rust_type(ctype: str, opaque: set, structs: set) -> str:
    """C type text (no name) -> Rust FFI type."""
    t = " ".join(ctype.replace("*", " * ").split())
    stars = t.count("*")
    # constness of the pointee: a 'const' before the first '*'
    head = t.split("*")[0].split()
    const = "const" in head
    base = " ".join(w for w in head if w not in ("const", "struct"))
    if base == "hdcStream_t":
        base_r, stars = "*mut CUstream_st", stars
    elif base in SCALARS:
        base_r = SCALARS[base]
    elif base in opaque or base in structs:
        base_r = base
    else:
        raise ValueError(f"unknown C type {ctype!r}")
    if stars == 0:
        if base_r == "c_void":
            return "()"
        return base_r
    r = ("*const " if const else "*mut ") + base_r
    for _ in range(stars - 1):
        r = "*mut " + r
    return r


def split_decl(decl: str):
    """'const JonesF64 *d_beam_jones' -> ('const JonesF64 *', 'd_beam_jones');
    'char name[256]' -> ('char *', 'name')."""
    d = " ".join(decl.replace("*", " * ").split())
    arr = re.search(r"\[\s*\d*\s*\]$", d)
    if arr:
        d = d[: arr.start()].strip()
        m = re.match(r"^(.*?)([A-Za-z_]\w*)$", d)
        return m.group(1).strip() + " *", m.group(2)
    m = re.match(r"^(.*?)([A-Za-z_]\w*)$", d)
    if not m or not m.group(1).strip():
        raise ValueError(f"cannot split declaration {decl!r}")
    return m.group(1).strip(), m.group(2)


def field_name(n: str) -> str:
    return n + "_" if n in RUST_KEYWORDS else n


def parse(header: Path = HEADER):
    txt = strip_comments(header.read_text())
    defines = []
    for m in re.finditer(r"^#define\s+(HDC_\w+)\s+(.+?)\s*$", txt, re.M):
        expr = m.group(2).strip()
        plain = re.sub(r"(\d+)u\b", r"\1", expr)
        if not re.fullmatch(r"[\d\s\*\+\-\(\)]+", plain):
            raise ValueError(f"#define {m.group(1)} is not an integer expression: {expr!r}")
        val = eval(plain, {"__builtins__": {}})  # digits and + - * ( ) only
        defines.append((m.group(1), int(val), "u" in expr))
    opaque = set(re.findall(r"typedef struct (\w+) \1;", txt))
    opaque.add("CUstream_st")
    structs = []
    names = set()
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", txt, re.S):
        names.add(m.group(1))
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", txt, re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            first, *rest = [x.strip() for x in decl.split(",")]
            ctype, name = split_decl(first)
            fields.append((name, rust_type(ctype, opaque, names)))
            for r in rest:  # "double x, y, z"
                fields.append((r, rust_type(ctype, opaque, names)))
        structs.append((m.group(1), fields))
    body = re.sub(r"typedef struct \w+ \{.*?\} \w+;", "", txt, flags=re.S)
    body = re.sub(r"typedef struct \w+ \*?\w+;", "", body)
    body = re.sub(r"^#.*$", "", body, flags=re.M)
    body = body.replace('extern "C" {', "").replace("}", "")
    funcs = []
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b([a-z_][a-z0-9_]*)\s*\(([^)]*)\)\s*;", body, re.S):
        ret = rust_type(m.group(1).strip(), opaque, names)
        params = []
        ptxt = m.group(3).strip()
        if ptxt and ptxt != "void":
            for p in ptxt.split(","):
                ctype, name = split_decl(p.strip())
                params.append((field_name(name), rust_type(ctype, opaque, names)))
        funcs.append((m.group(2), params, ret))
    return defines, sorted(opaque), structs, funcs


def render(header: Path = HEADER) -> str:
    defines, opaque, structs, funcs = parse(header)
    out = ["// Generated by rust/gen_bindings.py from include/hdc.h; do not edit.",
           "#![allow(non_camel_case_types, non_snake_case, dead_code, unused_imports)]", "",
           "use std::os::raw::{c_char, c_int, c_longlong, c_uchar, c_uint, c_ulonglong, c_void};", ""]
    for name, val, unsigned in defines:
        out.append(f"pub const {name}: {'c_uint' if unsigned else 'c_int'} = {val};")
    out.append("")
    for name in opaque:
        out += [f"#[repr(C)]", f"pub struct {name} {{", "    _private: [u8; 0],", "}", ""]
    for name, fields in structs:
        out += ["#[repr(C)]", "#[derive(Debug, Clone, Copy)]", f"pub struct {name} {{"]
        out += [f"    pub {field_name(f)}: {t}," for f, t in fields]
        out += ["}", ""]
    out.append('extern "C" {')
    for name, params, ret in funcs:
        args = ", ".join(f"{n}: {t}" for n, t in params)
        tail = "" if ret == "()" else f" -> {ret}"
        out.append(f"    pub fn {name}({args}){tail};")
    out.append("}")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    text = render()
    if "--check" in sys.argv:
        sys.exit(0 if OUT.exists() and OUT.read_text() == text else 1)
    OUT.write_text(text)
    print(f"wrote {OUT}")
