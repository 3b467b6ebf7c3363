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


def test_argument_errors_of_the_newer_entry_points():
    """Argument and state errors are reported before any device work: the traced solve without a
    reference solution or before the energy is set, the density matrices without G, the
    Hamiltonian reader on a missing file."""
    import numpy as np
    from angstromcube_b200 import green_function as gf, workloads
    L = _lib.lib()
    w = workloads.make("periodic4_1atom")
    p = gf.construct_Green_function(w.geometry)
    o = _lib.SolveOptions()
    st = _lib.SolveStats()
    count = ctypes.c_int32(-1)
    rc = L.a43g_solve_traced(p.handle, ctypes.byref(o), None, None, ctypes.byref(st), None, None, 10, None, 0,
                             ctypes.byref(count))
    assert rc == _lib.A43G_ERR_ARGUMENT and b"null" in L.a43g_last_error()
    ref = np.zeros(16)
    rc = L.a43g_solve_traced(p.handle, ctypes.byref(o), None, None, ctypes.byref(st), None,
                             ref.ctypes.data_as(ctypes.c_void_p), 10, None, 0, ctypes.byref(count))
    assert rc == _lib.A43G_ERR_STATE and b"energy" in L.a43g_last_error()
    out = np.zeros(16)
    rc = L.a43g_projection_coefficients(p.handle, None, out.ctypes.data_as(ctypes.c_void_p), None)
    assert rc == _lib.A43G_ERR_ARGUMENT
    h = ctypes.c_void_p()
    rc = L.a43g_hamiltonian_load(b"/nonexistent/Hmt.xml", ctypes.byref(h))
    assert rc != 0 and not h.value
