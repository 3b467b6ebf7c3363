"""The C-ABI library loads and exports every entry point that include/a43g.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from angstromcube_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"\b(a43g_\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    assert len(declared()) >= 14


@pytest.mark.parametrize("name", declared())
def test_symbol_exported(name):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(declared()) <= set(_lib.EXPORTED)


def test_errors_are_returned_not_fatal():
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.a43g_plan_build(None, ctypes.byref(h))
    assert rc == _lib.A43G_ERR_ARGUMENT
    assert b"null" in L.a43g_last_error()
    assert L.a43g_version().startswith(b"a43g")
