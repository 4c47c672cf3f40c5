"""Struct layouts of the drop-in FFI types, measured by compiling a probe.

The drop-in layer is only a drop-in if every struct the reference's Rust
binds through bindgen (gpu/types.h:33-287, FP64 build) has the same size and
field offsets in include/hdc.h.  `probe(header)` writes a small C program that
includes `header` and prints sizeof and offsetof of every field of those
structs, compiles it with the host C compiler and returns the numbers.  The
field names are taken from include/hdc.h, so a renamed field in either header
fails to compile.

make_golden.py runs it on the reference's types.h and commits the result as
ref_struct_layouts.json; tests/test_abi.py runs it on include/hdc.h and
compares.
"""

from __future__ import annotations

import json
import re
import subprocess
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
STRUCTS = ["RADec", "HADec", "XYZ", "UVW", "LmnRime", "GaussianParams", "ShapeletCoeff", "ShapeletUV", "JonesF32",
           "JonesF64", "Addresses", "Points", "Gaussians", "Shapelets", "IonoConsts"]


def fields(header: Path = ROOT / "include" / "hdc.h") -> dict:
    """Field names of every struct in STRUCTS, in declaration order."""
    txt = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    out = {}
    for name in STRUCTS:
        m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), txt, re.S)
        assert m, f"struct {name} not found in {header}"
        names = []
        for decl in m.group(1).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "double x, y, z" or "const JonesF64 *power_law_fds"
            head, *rest = [d.strip() for d in decl.split(",")]
            names.append(re.findall(r"[A-Za-z_]\w*", head)[-1])
            names.extend(re.findall(r"[A-Za-z_]\w*", r)[-1] for r in rest)
        out[name] = names
    return out


def probe(header: Path, cc: str = "gcc") -> dict:
    """{struct: {"size": n, "offsets": {field: offset}}} for `header`."""
    flds = fields()
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{Path(header).resolve()}"', "int main(void) {",
             '  printf("{\\n");']
    for i, (s, names) in enumerate(flds.items()):
        lines.append(f'  printf("\\"{s}\\": {{\\"size\\": %zu, \\"offsets\\": {{", sizeof({s}));')
        for j, f in enumerate(names):
            sep = ", " if j else ""
            lines.append(f'  printf("{sep}\\"{f}\\": %zu", offsetof({s}, {f}));')
        lines.append(f'  printf("}}}}{"," if i + 1 < len(flds) else ""}\\n");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = Path(d) / "probe.c", Path(d) / "probe"
        src.write_text("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c11", "-o", str(exe), str(src)], check=True, capture_output=True, text=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


DROPIN = ["model_points", "model_gaussians", "model_shapelets", "model_autos", "xyzs_to_uvws", "rotate", "average",
          "iono_loop", "subtract_iono", "add_model", "get_gpu_device_info"]


def _norm_type(decl: str) -> str:
    """ABI-relevant type of one parameter declaration: no parameter name, no
    top-level const, arrays as pointers, the FP64 build's FLOAT/JONES."""
    d = re.sub(r"\s+", " ", decl.strip())
    d = re.sub(r"\bFLOAT\b", "double", d)
    d = re.sub(r"\bJONES\b", "JonesF64", d)
    arr = re.search(r"\[\s*\d*\s*\]$", d)
    if arr:
        d = d[: arr.start()].strip() + " *"
    m = re.match(r"^(.*?)([A-Za-z_]\w*)$", d)
    if m and m.group(1).strip() and not m.group(1).strip().endswith(("struct", "const")):
        d = m.group(1)
    d = d.replace("*", " * ")
    toks = d.split()
    if toks and toks[0] == "const" and "*" not in toks:
        toks = toks[1:]  # a by-value const is the same type for the ABI
    # "const int * const" -> drop a trailing const on the pointer itself
    while toks and toks[-1] == "const":
        toks = toks[:-1]
    return " ".join(toks)


def prototypes(text: str, names=DROPIN) -> dict:
    """{name: [return type, [parameter types]]} of the C functions `names`
    declared or defined in `text`."""
    txt = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    txt = re.sub(r"//[^\n]*", "", txt)
    out = {}
    for n in names:
        m = re.search(r"(const\s+char\s*\*)\s*%s\s*\(([^)]*)\)\s*[;{]" % n, txt, re.S)
        if not m:
            continue
        params = [p for p in m.group(2).split(",") if p.strip()]
        out[n] = ["const char *", [_norm_type(p) for p in params]]
    return out
