"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares."""
import ctypes
import glob
import os
import re

from conftest import REPO


def _declared():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        names |= set(re.findall(r"TP_API\s+[\w\s\*]+?\b(tp_\w+)\s*\(", open(h).read()))
    return names


def _lib_path():
    from dissolve_tp.build import LIB, build

    if not os.path.exists(LIB):
        build()
    return LIB


def test_header_declares_entry_points():
    names = _declared()
    assert {"tp_assemble_csr", "tp_cg_create", "tp_matfree_apply", "tp_pattern"} <= names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib_path())
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from dissolve_tp import _lib

    assert _declared() <= set(_lib.SIGNATURES)
    assert _lib.lib.tp_version() >= 10000
    assert _lib.status_string(_lib.TP_ERR_BREAKDOWN).startswith("Krylov breakdown")


def test_no_cpu_fallback_when_library_missing(tmp_path, monkeypatch):
    """the binding refuses to load without the shared library"""
    import dissolve_tp.build as b
    import dissolve_tp._lib as L

    monkeypatch.setattr(b, "LIB", str(tmp_path / "missing.so"))
    monkeypatch.setattr(L, "LIB", str(tmp_path / "missing.so"))
    try:
        L._load()
    except ImportError as e:
        assert "no CPU fallback" in str(e)
    else:
        raise AssertionError("loaded a missing library")
