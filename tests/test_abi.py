"""The C-ABI library loads and exports every entry point include/hdc.h
declares (no GPU needed: nothing is called)."""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


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
    for ref in ["model_points", "model_gaussians", "model_shapelets", "model_autos", "xyzs_to_uvws", "rotate",
                "average", "iono_loop", "subtract_iono", "add_model"]:
        assert ref in names


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
