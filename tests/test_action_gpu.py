"""Parity of the sm_100a action (through the C ABI) with the oracle.

FP64: within 1e-12 relative (max norm) of the restated oracle, which itself matches the
reference's CPU build to 1e-13.  FP32: within 3e-5 relative (rounding of the FP32 stencil
and projector sums; the FP32 reference build shows the same order).  Full-size plans are
checked through size-independent properties: linearity and complex symmetry at k = 0.
"""
import numpy as np
import pytest

import oracle
from helpers import GEOMETRIES, inputs_for, product_plan, rel_err
from angstromcube_b200 import green_action, green_function as gf, workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 3e-5


def apply(plan, x_np, dtype):
    x = torch.from_numpy(x_np.astype(dtype)).cuda()
    y = torch.empty_like(x)
    ci = torch.from_numpy(plan.export()["colindx"].astype(np.int16)).cuda()
    op = green_action.action_t(plan, "float64" if dtype == np.float64 else "float32")
    flops = op.multiply(y, x, ci, plan.nnzb, plan.nCols)
    torch.cuda.synchronize()
    assert flops > 0
    return y.cpu().numpy()


@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_action_fp64_fp32_vs_oracle(name):
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    o = oracle.RestatedOracle(p.export(), Vc, E)
    x = np.random.default_rng(2).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = o.action(x)
    y64 = apply(p, x, np.float64)
    assert rel_err(y64, y_ref) < FP64_TOL
    y32 = apply(p, x, np.float32)
    assert rel_err(y32, y_ref) < FP32_TOL


@pytest.mark.parametrize("variant", ["rows", "plain", "pencils", "staged"])
@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_action_fp32_local_variants_vs_oracle(name, variant, monkeypatch):
    """Every FP32 local kernel (rows with loads ahead; plain rows; y-pencils, the default;
    y-pencils with staged neighbour cubes) matches the oracle on every boundary condition, with
    Bloch phases (k != 0)."""
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    monkeypatch.setenv("A43G_LOCAL", variant)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = np.random.default_rng(3).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = oracle.RestatedOracle(p.export(), Vc, E).action(x)
    assert rel_err(apply(p, x, np.float32), y_ref) < FP32_TOL


@pytest.mark.parametrize("variant", ["rows", "pencils", "rolled", "chain3"])
@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_action_fp64_local_variants_vs_oracle(name, variant, monkeypatch):
    """Both FP64 local kernels (rows; pencils with the two planes on two threads, the default),
    both FP64 additions (z-orders unrolled, the default; "rolled": one at a time) and both
    atom-matrix chains (one kernel, the default; "chain3": collect, multiply, broadcast) match the
    oracle (FP64 to 1e-12, FP32 to 3e-5) on every boundary condition, with Bloch phases (k != 0)."""
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    if variant == "rolled":
        monkeypatch.setenv("A43G_ADD64", "rolled")
    elif variant == "chain3":
        monkeypatch.setenv("A43G_ATOM_CHAIN", "three")
    else:
        monkeypatch.setenv("A43G_LOCAL64", variant)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = np.random.default_rng(4).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = oracle.RestatedOracle(p.export(), Vc, E).action(x)
    assert rel_err(apply(p, x, np.float64), y_ref) < FP64_TOL
    if variant == "chain3":
        assert rel_err(apply(p, x, np.float32), y_ref) < FP32_TOL


def test_action_matches_reference_build():
    """Directly against the reference's action_t on the same plan inputs (FP64 and FP32)."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    from helpers import reference_plan
    g = GEOMETRIES["mixed_iso_peri_vac"]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    r = reference_plan(g, Vc, mats, offs, E, k, dVol)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = np.random.default_rng(4).standard_normal((p.nnzb, 2, 64, 64))
    assert rel_err(apply(p, x, np.float64), r.action(x)) < FP64_TOL
    assert rel_err(apply(p, x, np.float32), r.action(x.astype(np.float32)).astype(np.float64)) < FP32_TOL


@pytest.mark.parametrize("kpoint", [(0.0, 0.0, 0.0), (0.125, -0.25, 1 / 3.0)])
def test_benchmark_cell_matches_reference_build(kpoint):
    """The benchmark cell itself (periodic 16^3 cubes, 64 atoms numax 5 sigma 0.6, its potential,
    atom matrices and energy E = -0.2 + 0.02i) with one source cube (4,096 blocks), against the
    reference's action_t<double,2,1>::multiply on identical inputs: FP64 and FP32 actions."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    w = workloads.make("periodic16_64atoms_s1x1x1")
    k = np.array(kpoint)
    r = oracle.RefGreen(w.geometry)
    r.set_potential(w.Vcell)
    r.set_atom_matrices(w.mats, w.offsets)
    r.set_energy(w.E, w.dVol)
    r.set_kpoint(k)
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, w.E, w.dVol)
    gf.update_phases(p, k)
    assert p.nnzb == r.sizes["nnzb"] == 4096
    x = np.random.default_rng(21).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = r.action(x)
    assert rel_err(apply(p, x, np.float64), y_ref) < FP64_TOL
    assert rel_err(apply(p, x, np.float32), y_ref) < FP32_TOL


def test_action_mid_size_workload():
    w = workloads.make("periodic8_8atoms_s2x2x1")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, w.E, w.dVol)
    o = oracle.RestatedOracle(p.export(), w.Vcell, w.E)
    x = np.random.default_rng(3).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = o.action(x)
    assert rel_err(apply(p, x, np.float64), y_ref) < FP64_TOL
    assert rel_err(apply(p, x, np.float32), y_ref) < FP32_TOL


def _complex_columns(y):
    # [nnzb, 2, 64, 64] -> complex [nnzb*64 rows, 64 columns]
    return (y[:, 0] + 1j * y[:, 1]).reshape(-1, 64)


@pytest.mark.parametrize("name", ["periodic16_64atoms"])
def test_full_size_linearity_and_symmetry(name):
    """At the benchmark size: A(a x + b z) = a A x + b A z, and u^T A v = v^T A u per column
    at k = 0 (H real symmetric, the truncated operator complex symmetric)."""
    w = workloads.make(name)
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, w.E, w.dVol)
    ci = torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()
    op = green_action.action_t(p, "float64")
    gen = torch.Generator(device="cuda").manual_seed(0)
    shape = (p.nnzb, 2, 64, 64)
    x = torch.randn(shape, device="cuda", dtype=torch.float64, generator=gen)
    z = torch.randn(shape, device="cuda", dtype=torch.float64, generator=gen)
    Ax, Az, As = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    op.multiply(Ax, x, ci, p.nnzb, p.nCols)
    op.multiply(Az, z, ci, p.nnzb, p.nCols)
    op.multiply(As, 0.75 * x - 1.25 * z, ci, p.nnzb, p.nCols)
    torch.cuda.synchronize()
    lin = (As - (0.75 * Ax - 1.25 * Az)).abs().max().item() / As.abs().max().item()
    assert lin < 1e-13
    # bilinear symmetry per column: sum over rows of x * (A z) == z * (A x), complex arithmetic
    xc = torch.complex(x[:, 0], x[:, 1]); zc = torch.complex(z[:, 0], z[:, 1])
    Axc = torch.complex(Ax[:, 0], Ax[:, 1]); Azc = torch.complex(Az[:, 0], Az[:, 1])
    ci64 = ci.long()
    s1 = torch.zeros((p.nCols, 64), dtype=torch.complex128, device="cuda")
    s2 = torch.zeros_like(s1)
    s1.index_add_(0, ci64, (xc * Azc).sum(dim=1))
    s2.index_add_(0, ci64, (zc * Axc).sum(dim=1))
    sym = (s1 - s2).abs().max().item() / s1.abs().max().item()
    assert sym < 1e-11
    # FP32 operator on the same input
    op32 = green_action.action_t(p, "float32")
    x32 = x.float(); Ax32 = torch.empty_like(x32)
    op32.multiply(Ax32, x32, ci, p.nnzb, p.nCols)
    torch.cuda.synchronize()
    assert ((Ax32.double() - Ax).abs().max() / Ax.abs().max()).item() < FP32_TOL


@pytest.mark.parametrize("name", ["wrap8", "peri_xy_wrap_z", "repeat_aniso"])
def test_projector_tensor_cores_vs_simt(name, monkeypatch):
    """The FP32 projector on the tensor cores (3xTF32) and on the SIMT cores (default) agree, and
    both match the FP64 oracle; no kernel recorded a wait timeout."""
    from angstromcube_b200 import _lib
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    monkeypatch.setenv("A43G_PROJECTOR", "tc")
    p_tc = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = np.random.default_rng(9).standard_normal((p_tc.nnzb, 2, 64, 64))
    y_tc = apply(p_tc, x, np.float32)
    _lib.check(_lib.lib().a43g_plan_device_status(p_tc.handle), "device status")
    monkeypatch.setenv("A43G_PROJECTOR", "simt")
    p_simt = product_plan(g, Vc, mats, offs, E, k, dVol)
    y_simt = apply(p_simt, x, np.float32)
    y_ref = oracle.RestatedOracle(p_tc.export(), Vc, E).action(x)
    assert rel_err(y_simt, y_ref) < FP32_TOL
    assert rel_err(y_tc, y_ref) < FP32_TOL
    assert rel_err(y_tc, y_simt) < FP32_TOL


def test_action_fp32_unaligned_input():
    """x that is only 4-byte aligned (an offset view) takes the generic projector kernels and
    gives the same result as an aligned copy."""
    g = GEOMETRIES["wrap8"]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    xn = np.random.default_rng(5).standard_normal((p.nnzb, 2, 64, 64)).astype(np.float32)
    n = xn.size
    buf = torch.zeros(n + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(xn.ravel()).cuda()
    x_off = buf[1:].view(p.nnzb, 2, 64, 64)
    assert x_off.data_ptr() % 16 != 0
    ci = torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()
    op = green_action.action_t(p, "float32")
    y_off = torch.empty((p.nnzb, 2, 64, 64), dtype=torch.float32, device="cuda")
    op.multiply(y_off, x_off, ci, p.nnzb, p.nCols)
    torch.cuda.synchronize()
    # and a y that is only 4-byte aligned
    ybuf = torch.zeros(n + 1, dtype=torch.float32, device="cuda")
    y_off2 = ybuf[1:].view(p.nnzb, 2, 64, 64)
    op.multiply(y_off2, x_off.contiguous().clone(), ci, p.nnzb, p.nCols)
    torch.cuda.synchronize()
    y_al = apply(p, xn, np.float32)
    assert rel_err(y_off2.cpu().numpy(), y_al) < FP32_TOL
    y_ref = oracle.RestatedOracle(p.export(), Vc, E).action(xn.astype(np.float64))
    assert rel_err(y_off.cpu().numpy(), y_ref) < FP32_TOL
    assert rel_err(y_al, y_ref) < FP32_TOL


def test_action_rejects_bad_sizes():
    g = GEOMETRIES["no_atoms"]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    x = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    ci = torch.zeros(p.nnzb, device="cuda", dtype=torch.int16)
    op = green_action.action_t(p, "float64")
    with pytest.raises(RuntimeError, match="nnzb"):
        op.multiply(torch.empty_like(x), x, ci, p.nnzb + 1, p.nCols)
    with pytest.raises(RuntimeError, match="alias"):
        op.multiply(x, x, ci, p.nnzb, p.nCols)


@pytest.mark.parametrize("name", ["wrap8", "peri_xy_wrap_z"])
def test_autotune_keeps_parity(name):
    """The autotuner only changes the schedule: after it the FP32 and FP64 actions still match
    the oracle."""
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    report = green_action.autotune(p, "float32")
    assert "chosen" in report, report
    x = np.random.default_rng(12).standard_normal((p.nnzb, 2, 64, 64))
    y_ref = oracle.RestatedOracle(p.export(), Vc, E).action(x)
    assert rel_err(apply(p, x, np.float32), y_ref) < FP32_TOL
    assert "chosen" in green_action.autotune(p, "float64")
    assert rel_err(apply(p, x, np.float64), y_ref) < FP64_TOL
