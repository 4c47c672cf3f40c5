"""The C-ABI library loads and exports every entry point include/hdc.h
declares, the drop-in structs and functions have the reference's layouts and
parameter types, and kernel error words decode to static messages (no GPU
needed: no compute call is made)."""

import ctypes
import importlib.util
import json
import re
import shutil
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def layout_probe():
    spec = importlib.util.spec_from_file_location("layout_probe", GOLDEN / "layout_probe.py")
    lp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(lp)
    return lp


def declared_functions():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", txt, re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.append(name)
    return sorted(set(names))


def test_header_declares_the_reference_ffi():
    names = declared_functions()
    # every C symbol the reference's Rust binds (gpu/model.h:33-56,
    # gpu/peel.h:13-35, gpu/utils.h:28)
    for ref in ["model_points", "model_gaussians", "model_shapelets", "model_autos", "xyzs_to_uvws", "rotate",
                "average", "iono_loop", "subtract_iono", "add_model", "get_gpu_device_info"]:
        assert ref in names


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_struct_layouts_equal_the_reference():
    """sizeof and every field offset of the FFI structs, include/hdc.h against
    the reference's gpu/types.h (FP64 build; fixture made by make_golden.py)."""
    ref = json.loads((GOLDEN / "ref_struct_layouts.json").read_text())["layouts"]
    ours = layout_probe().probe(ROOT / "include" / "hdc.h")
    assert set(ours) == set(ref)
    for name in ref:
        assert ours[name] == ref[name], name


def test_dropin_prototypes_equal_the_reference():
    """Parameter types (after the FP64 build's macros) of every drop-in
    function, include/hdc.h against the reference's definitions."""
    lp = layout_probe()
    ref = json.loads((GOLDEN / "ref_struct_layouts.json").read_text())["prototypes"]
    ours = lp.prototypes((ROOT / "include" / "hdc.h").read_text())
    assert set(ref) == set(lp.DROPIN)
    for name in ref:
        assert ours.get(name) == ref[name], name


def test_kernel_error_words_decode_to_static_messages():
    from mwa_hyperdrive_b200 import _lib, build

    if not _lib.LIB_PATH.exists():
        build.build()
    lib = _lib.lib()
    assert lib.hdc_kernel_error_string(0) is None
    timeout = lib.hdc_kernel_error_string(1)
    index = lib.hdc_kernel_error_string(2)
    assert b"bounded wait ran out" in timeout and b"unchanged" in timeout
    assert b"index outside" in index
    # a timeout wins over an index error when both bits are set
    assert lib.hdc_kernel_error_string(3) == timeout


def test_library_exports_every_declared_symbol():
    from mwa_hyperdrive_b200 import _lib, build

    if not _lib.LIB_PATH.exists():
        build.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    from mwa_hyperdrive_b200 import _lib

    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from mwa_hyperdrive_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "libhdc.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.HdcError):
        _lib.lib()
