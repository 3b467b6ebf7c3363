"""Atomic density matrices Im <p_i|G|p_j> (a43g_projection_coefficients) against the reference's
own get_projection_coefficients (include/green_dyadic.hxx:1062-1088, CPU build in oracle/_ref) on
the same plan and block vector: within 1e-12 relative.  Plans with periodic atom images are
refused, as the reference refuses them."""
import numpy as np
import pytest

import oracle
from helpers import GEOMETRIES, inputs_for, product_plan, reference_plan
from angstromcube_b200 import green_action

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["iso6_fd16", "mixed_iso_peri_vac", "repeat_aniso"])
def test_density_matrices_match_reference(name):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    r = reference_plan(g, Vc, mats, offs, E, k, dVol)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    G = np.random.default_rng(7).standard_normal((p.nnzb, 2, 64, 64))
    ref = r.projection_coefficients(G)
    if ref is None:
        with pytest.raises(RuntimeError, match="periodic atom images"):
            green_action.get_projection_coefficients(p, torch.from_numpy(G).cuda())
        return
    ours = green_action.get_projection_coefficients(p, torch.from_numpy(G).cuda())
    assert len(ours) == len(ref) > 0
    scale = max(np.abs(m).max() for m in ref)
    for a, b in zip(ours, ref):
        assert np.abs(a - b).max() <= 1e-12 * scale


def test_density_matrices_refuse_periodic_images():
    g = GEOMETRIES["peri_xy_wrap_z"]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    assert p.sizes["nAtomImages"] > p.sizes["nAtoms"]
    G = torch.zeros((p.nnzb, 2, 64, 64), dtype=torch.float64, device="cuda")
    with pytest.raises(RuntimeError, match="periodic atom images"):
        green_action.get_projection_coefficients(p, G)
