"""The Rust binding (rust/, not compiled here: no cargo) against the C header
it binds: rust/src/ffi.rs must be exactly what rust/gen_bindings.py makes
from the current include/hdc.h, declare every function of the header with
the same number of parameters, and lay out every FFI struct with the
header's fields in the header's order."""

import importlib.util
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def load(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_ffi_rs_is_generated_from_the_current_header():
    gen = load(ROOT / "rust" / "gen_bindings.py", "gen_bindings")
    assert (ROOT / "rust" / "src" / "ffi.rs").read_text() == gen.render(), "run python rust/gen_bindings.py"


def c_prototypes():
    txt = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "hdc.h").read_text(), flags=re.S)
    txt = re.sub(r"typedef struct \w+ \{.*?\} \w+;", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(([^)]*)\)\s*;", txt, re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_every_function_declared_with_its_arity():
    rs = (ROOT / "rust" / "src" / "ffi.rs").read_text()
    decl = {m.group(1): (0 if not m.group(2).strip() else m.group(2).count(",") + 1)
            for m in re.finditer(r"pub fn (\w+)\(([^)]*)\)", rs)}
    c = c_prototypes()
    assert set(decl) == set(c)
    for name, n in c.items():
        assert decl[name] == n, name
    # the reference's drop-in FFI is all there
    for ref in ["model_points", "model_gaussians", "model_shapelets", "model_autos", "xyzs_to_uvws", "rotate",
                "average", "iono_loop", "subtract_iono", "add_model", "get_gpu_device_info"]:
        assert ref in decl


def test_struct_fields_in_header_order():
    lp = load(ROOT / "tests" / "golden" / "layout_probe.py", "layout_probe")
    rs = (ROOT / "rust" / "src" / "ffi.rs").read_text()
    for name, fields in lp.fields().items():
        m = re.search(r"#\[repr\(C\)\]\n#\[derive\(Debug, Clone, Copy\)\]\npub struct %s \{(.*?)\n\}" % name, rs,
                      re.S)
        assert m, name
        got = re.findall(r"pub (\w+):", m.group(1))
        assert got == fields, name


def test_safe_wrappers_call_declared_functions_only():
    rs = (ROOT / "rust" / "src" / "ffi.rs").read_text()
    lib = (ROOT / "rust" / "src" / "lib.rs").read_text()
    declared = set(re.findall(r"pub fn (\w+)\(", rs))
    # calls (not the wrappers' own `fn` definitions)
    called = set(re.findall(r"(?<!fn )\b(hdc_\w+|model_\w+)\(", lib))
    assert called and called <= declared, called - declared
