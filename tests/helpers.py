"""Shared set-up of the parity tests: geometries, plans on both sides, seeded inputs."""
import numpy as np

from angstromcube_b200 import green_function as gf
from angstromcube_b200 import workloads

H = (0.25, 0.25, 0.25)


def geometry(nb, bc, r, src, nFD, natoms, seed=3, h=H, sigma=0.5, numax=3):
    """Random atoms in a cell of nb cubes (atom ids = indices)."""
    rng = np.random.default_rng(seed)
    ng = tuple(4 * n for n in nb)
    L = np.array(ng) * np.array(h)
    atoms = np.zeros((natoms, 8))
    atoms[:, :3] = rng.uniform(-L / 2, L / 2, size=(natoms, 3))
    atoms[:, 3] = 1
    atoms[:, 4] = np.arange(natoms)
    atoms[:, 5] = numax
    atoms[:, 6] = sigma
    return workloads.Geometry(ng, bc, h, r, src, nFD, 6.0, atoms)


# geometries covering every boundary condition, both stencils and both projector cases
GEOMETRIES = {
    "wrap8": lambda: geometry((8, 8, 8), (1, 1, 1), 3.0, (2, 2, 2), 4, 3),
    "iso6_fd16": lambda: geometry((6, 6, 6), (0, 0, 0), 2.5, (2, 1, 1), 8, 2),
    "mixed_iso_peri_vac": lambda: geometry((6, 5, 7), (0, 1, 2), 2.0, (1, 2, 2), 4, 3),
    "repeat_aniso": lambda: geometry((5, 6, 4), (3, 1, 0), 2.2, (2, 2, 1), 4, 2, h=(0.25, 0.3, 0.2)),
    "wrap8_fd16_numax5": lambda: geometry((8, 8, 8), (1, 1, 1), 2.9, (3, 3, 3), 8, 4, sigma=0.4, numax=5),
    "peri_xy_wrap_z": lambda: geometry((4, 4, 8), (1, 1, 1), 3.0, (1, 1, 2), 4, 2),
    "no_atoms": lambda: geometry((4, 4, 4), (1, 1, 1), 6.0, (1, 1, 1), 4, 0),
}


def inputs_for(g, seed=5):
    """Cell potential, atom matrices, energy, k-point and dVol for a geometry."""
    rng = np.random.default_rng(seed)
    ncell = int(np.prod(np.array(g.ng) // 4))
    Vc = rng.standard_normal((ncell, 64)) * 0.3
    na = len(g.xyzZinso)
    mats, offs = workloads._atom_matrices([int(v) for v in g.xyzZinso[:, 5]], list(g.xyzZinso[:, 6]), rng)
    E = complex(-0.3, 0.05)
    k = np.array([0.1, 0.2, -0.15])
    dVol = float(np.prod(g.hg))
    return Vc, mats, offs, E, k, dVol, na


def product_plan(g, Vc, mats, offs, E, k, dVol):
    p = gf.construct_Green_function(g)
    gf.update_potential(p, Vc, mats if len(offs) else None, offs if len(offs) else None, layout="cells")
    gf.update_energy_parameter(p, E, dVol)
    gf.update_phases(p, k)
    return p


def reference_plan(g, Vc, mats, offs, E, k, dVol):
    import oracle
    r = oracle.RefGreen(g)
    r.set_potential(Vc)
    if len(offs):
        r.set_atom_matrices(mats, offs)
    r.set_energy(E, dVol)
    r.set_kpoint(k)
    return r


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
