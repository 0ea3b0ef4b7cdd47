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


def test_zero_size_and_null_arguments_need_no_device():
    """Zero-length calls return TP_OK and null operands are rejected with ValueError, both
    before any device work: nothing here needs a GPU, so the placeholder addresses are
    never dereferenced."""
    import pytest

    from dissolve_tp import _lib

    one = (ctypes.c_double * 4)(1.0, 1.0, 1.0, 1.0)
    P = 4096  # placeholder address, never read
    zero_calls = [
        ("tp_cell_average", 0, P, P, P, None),
        ("tp_axpby", 0, 2.0, P, 3.0, P, None),
        ("tp_advance_state", 0, P, P, P, P, None),
        ("tp_pack_columns", 0, 3, 4, P, P, None),
        ("tp_unpack_columns", 0, 3, 4, P, P, None),
        ("tp_o2_alpha", 0, P, P, 0.1, 2.0, P, None),
        ("tp_lumped_rhs", 0, 3, 4, P, P, None, 50.0, 0, None, one, P, None),
    ]
    for name, *args in zero_calls:
        assert _lib.call(name, *args) == _lib.TP_OK, name
    null_calls = [
        ("tp_axpby", 8, 2.0, None, 3.0, P, None),
        ("tp_cell_average", 8, P, None, P, None),
        ("tp_pack_columns", 8, 3, 2, P, P, None),  # ld < S
        ("tp_lumped_rhs", 8, 5, 5, P, P, None, 50.0, 0, None, one, P, None),  # S > 4
    ]
    for name, *args in null_calls:
        with pytest.raises(ValueError):
            _lib.call(name, *args)
