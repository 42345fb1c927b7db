"""The C ABI: librumb.so loads and exports every entry point include/rumb.h declares, and its
error convention holds without a GPU (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"RUMB_API\s+int\s+(rumb_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from rumb import _lib
    L = _lib.load()
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    # and the binding covers every declaration
    assert set(declared) <= set(_lib.exported_symbols())


def test_version_and_error_convention():
    from rumb import _lib
    L = _lib.load()
    assert L.rumb_version() == 100
    # NULL context -> RUMB_E_INVAL with a message, no crash
    assert L.rumb_ctx_sync(None) == _lib.E_INVAL
    assert "NULL" in _lib.last_error()
    assert L.rumb_cancel(None) == _lib.E_INVAL


def test_context_without_gpu_reports_nodev_or_works():
    from rumb import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    st = L.rumb_ctx_create(0, ctypes.byref(h))
    if st == _lib.OK:
        assert L.rumb_ctx_destroy(h) == _lib.OK
    else:
        assert st == _lib.E_NODEV, _lib.last_error()
        with pytest.raises(_lib.RumbError):
            _lib.Context(0)
