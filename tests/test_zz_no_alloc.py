"""The allocation-free action (a43g_action_multiply_noalloc), for callers that cannot let the
library allocate device memory (hosts whose own pool owns the GPU's memory, loops that cannot
take the synchronization of cudaMalloc): two calls in a
row agree with a43g_action_multiply on the same inputs, within the tolerances of the action
tests (1e-12 relative in FP64, 3e-5 in FP32); plans needing more than the fixed scratch, and
plans not yet current on the device, are refused with an error.  This file is collected last."""
import ctypes

import numpy as np
import pytest

from helpers import GEOMETRIES, inputs_for, product_plan, rel_err
from angstromcube_b200 import _lib, green_action

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-12, np.float32: 3e-5}


def noalloc(plan, y, x, ci, dtype_code):
    flops = ctypes.c_double(0)
    rc = _lib.lib().a43g_action_multiply_noalloc(plan.handle, _lib.ptr(y), _lib.ptr(x), _lib.ptr(ci), plan.nnzb,
                                                 plan.nCols, None, dtype_code, ctypes.byref(flops))
    return rc, flops.value


@pytest.mark.parametrize("name", ["wrap8", "peri_xy_wrap_z"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_matches_multiply_twice(name, dtype):
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    p.upload()
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    code = _lib.A43G_F64 if dtype == np.float64 else _lib.A43G_F32
    ci = torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()
    op = green_action.action_t(p, "float64" if dtype == np.float64 else "float32")
    gen = torch.Generator(device="cuda").manual_seed(17)
    for _ in range(2):                               # two calls in a row on fresh inputs
        x = torch.randn((p.nnzb, 2, 64, 64), device="cuda", dtype=tdt, generator=gen)
        y_ref = torch.empty_like(x)
        f_ref = op.multiply(y_ref, x, ci, p.nnzb, p.nCols)
        y = torch.full_like(x, float("nan"))
        rc, f = noalloc(p, y, x, ci, code)
        torch.cuda.synchronize()
        assert rc == 0, _lib.lib().a43g_last_error()
        assert f == f_ref
        assert rel_err(y.double().cpu().numpy(), y_ref.double().cpu().numpy()) < TOL[dtype]


def test_noalloc_allocates_nothing():
    """After a first call (which loads the library's device code and looks up the array), further
    calls leave the device's free memory and the torch caching allocator's reservation unchanged."""
    g = GEOMETRIES["wrap8"]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    p.upload()
    ci = torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()
    x = torch.randn((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    x32, y32 = x.float(), torch.empty((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float32)
    for xx, yy, code in ((x, y, _lib.A43G_F64), (x32, y32, _lib.A43G_F32)):
        assert noalloc(p, yy, xx, ci, code)[0] == 0, _lib.lib().a43g_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(3):
        for xx, yy, code in ((x, y, _lib.A43G_F64), (x32, y32, _lib.A43G_F32)):
            assert noalloc(p, yy, xx, ci, code)[0] == 0, _lib.lib().a43g_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == reserved0


def test_noalloc_refuses_large_and_stale_plans():
    g = GEOMETRIES["wrap8_fd16_numax5"]()            # about 74 MB of FP64 projector scratch
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    ci = torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()
    rc, _ = noalloc(p, y, x, ci, _lib.A43G_F64)      # not uploaded yet: refused before any work
    assert rc == _lib.A43G_ERR_STATE
    assert b"a43g_plan_upload" in _lib.lib().a43g_last_error()
    p.upload()
    rc, _ = noalloc(p, y, x, ci, _lib.A43G_F64)
    assert rc == _lib.A43G_ERR_UNSUPPORTED
    assert b"scratch" in _lib.lib().a43g_last_error()
