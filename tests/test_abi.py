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


def test_bm_plan_counts_the_solve_buffers_without_a_gpu():
    """rumb_bm_plan sizes a solve from (n, mp, dtype) alone: the state and scratch slabs, the
    snapshot slab, the float64 certificate, the masks and the rows; bad sizes are refused."""
    from rumb import _lib
    n, mp = 18, 23650
    m2, N = n << (n - 1), 1 << n
    cert = 16 * m2 + 24 * N + 32 * mp + 64 + 4 * N + 16 * mp
    work = lambda e: 10 * m2 * e + (m2 + 31) // 32 * 4 + 4 * N + 64 * e + 16
    assert _lib.bm_plan(n, mp, "float64") == work(8) + cert
    assert _lib.bm_plan(n, mp, "float32") == work(4) + cert
    assert _lib.bm_plan(n, mp, "mixed") == work(4) + work(8) + cert
    for bad in ((1, mp, "float64"), (31, mp, "float64"), (n, 0, "float64")):
        with pytest.raises(_lib.RumbError):
            _lib.bm_plan(*bad)
