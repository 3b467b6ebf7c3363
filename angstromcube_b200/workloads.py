"""Seeded synthetic workloads of the Green-function action and solver.

Every workload is a cell of 4x4x4-point cubes with a local potential made of Gaussian wells
plus small uniform noise, SHO-projector atoms with random symmetric atom matrices, an energy
parameter and a k-point.  The numbers follow the workloads the benchmarks are quoted on:

  periodic4_1atom      4^3 cubes (16^3 points, h = 0.25 Bohr), periodic, 4 Gaussians, one atom
                       numax 3 sigma 0.5 at the centre, 1 source cube, r_trunc 6, E = -0.3 + 0.05i
  periodic16_64atoms   16^3 cubes, periodic, 64 Gaussians, 64 atoms on a 4^3 lattice with
                       +-0.3 Bohr jitter, numax 5 sigma 0.6, 4x4x1 source cubes, r_trunc 12,
                       E = -0.2 + 0.02i
  wrapped32_256atoms   32^3 cubes, truncation sphere fits (wrapped), 256 atoms on an 8x8x4
                       lattice over the whole cell with +-0.3 Bohr jitter, 4x4x2 sources, r_trunc 12
plus scaled-down variants used by the tests.  Potentials are periodic sums over minimum
images; atom matrices are real symmetric with N(0, 0.1) entries, the overlap part shifted to
be positive definite, then multiplied by the SHO prefactors (the caller-side rescaling of
src/energy_contour.cxx:307-323).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Geometry:
    ng: tuple
    bc: tuple
    hg: tuple
    r_trunc: float
    sources: tuple
    nFD: int = 4
    proj_radius: float = 6.0
    xyzZinso: np.ndarray = field(default_factory=lambda: np.zeros((0, 8)))


@dataclass
class Workload:
    name: str
    geometry: Geometry
    Vcell: np.ndarray          # [ncells, 64]
    mats: np.ndarray           # concatenated [natoms][2][nc][nc]
    offsets: np.ndarray        # [natoms]
    E: complex
    k: np.ndarray
    dVol: float
    tolerance: float
    max_iterations: int

    @property
    def natoms(self):
        return len(self.geometry.xyzZinso)


def nsho(numax):
    return (numax + 1) * (numax + 2) * (numax + 3) // 6


def sho_prefactors(numax, sigma):
    """sqrt(2^nx/(nx! sqrt(pi) sigma)) * (same for y, z) in zyx order (include/sho_projection.hxx:181-209)."""
    from math import factorial, pi, sqrt
    f1 = [sqrt(2.0 ** n / (factorial(n) * sqrt(pi) * sigma)) for n in range(numax + 1)]
    out = []
    for nz in range(numax + 1):
        for ny in range(numax + 1 - nz):
            for nx in range(numax + 1 - nz - ny):
                out.append(f1[nx] * f1[ny] * f1[nz])
    return np.array(out)


def _potential_cells(ng, hg, centres, depth, width, noise, rng):
    """Sum of periodic Gaussian wells on the grid (minimum image), returned as [ncells][64]."""
    ng = np.asarray(ng); hg = np.asarray(hg, dtype=np.float64)
    L = ng * hg
    axes = [(np.arange(ng[d]) - ng[d] / 2 + 0.5) * hg[d] for d in range(3)]
    # the Gaussians are separable: per centre and direction the 1D factor of the minimum-image
    # distance, then V[z, y, x] = depth * sum_c gz[c, z] gy[c, y] gx[c, x] as one matrix product
    c = np.asarray(centres, dtype=np.float64).reshape(-1, 3)
    g = []
    for d in range(3):
        dd = axes[d][None, :] - c[:, d:d + 1]
        dd -= L[d] * np.round(dd / L[d])
        g.append(np.exp(-(dd * dd) / (2 * width * width)))
    gzy = (g[2][:, :, None] * g[1][:, None, :]).reshape(len(c), -1)          # [c, z*y]
    V = depth * (gzy.T @ g[0]).reshape(ng[2], ng[1], ng[0])
    V += rng.uniform(-noise, noise, size=V.shape)
    nb = ng // 4
    # [iz, iy, ix] -> [bz, i4z, by, i4y, bx, i4x] -> cells (bz, by, bx) x points (i4z, i4y, i4x)
    Vc = V.reshape(nb[2], 4, nb[1], 4, nb[0], 4).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 64)
    return np.ascontiguousarray(Vc), V


def _atom_matrices(numaxes, sigmas, rng):
    mats, offsets, off = [], [], 0
    for numax, sigma in zip(numaxes, sigmas):
        n = nsho(numax)
        A = rng.normal(0.0, 0.1, size=(n, n)); dH = np.triu(A) + np.triu(A, 1).T
        B = rng.normal(0.0, 0.1, size=(n, n)); dS = np.triu(B) + np.triu(B, 1).T
        dS += (-np.linalg.eigvalsh(dS)[0] + 0.1) * np.eye(n)
        f = sho_prefactors(numax, sigma)
        F = np.outer(f, f)
        mats.append(np.concatenate([(F * dH).ravel(), (F * dS).ravel()]))
        offsets.append(off); off += 2 * n * n
    if not mats:
        return np.zeros(1), np.zeros(0, np.int64)
    return np.concatenate(mats), np.array(offsets, np.int64)


def make(name, seed=0):
    """Build one of the named workloads (see the module docstring)."""
    rng = np.random.default_rng(seed)
    h = 0.25
    if name in ("periodic4_1atom", "periodic4_1atom_iso", "periodic4_noatom"):
        nb = 4
        ng = (4 * nb,) * 3
        L = ng[0] * h
        centres = rng.uniform(-L / 2, L / 2, size=(4, 3))
        Vc, _ = _potential_cells(ng, (h,) * 3, centres, -1.0, 1.5, 1e-3, rng)
        atoms = np.zeros((0 if name == "periodic4_noatom" else 1, 8))
        if len(atoms):
            atoms[0] = [0, 0, 0, 1, 0, 3, 0.5, 0]
        mats, offs = _atom_matrices([3] * len(atoms), [0.5] * len(atoms), rng)
        bc = (0, 0, 0) if name.endswith("_iso") else (1, 1, 1)
        geo = Geometry(ng, bc, (h,) * 3, 6.0, (1, 1, 1), 4, 6.0, atoms)
        return Workload(name, geo, Vc, mats, offs, complex(-0.3, 0.05), np.zeros(3), h ** 3, 1e-9, 500)
    if name.startswith("periodic") and "_" in name:
        # periodicN_Matoms[_sSx_Sy_Sz]: N^3 cubes, M atoms on a cubic lattice, sources box
        parts = name.split("_")
        nb = int(parts[0][len("periodic"):])
        natoms = int(parts[1][:-len("atoms")])
        src = (4, 4, 1)
        if len(parts) > 2 and parts[2].startswith("s"):
            src = tuple(int(v) for v in parts[2][1:].split("x"))
        ng = (4 * nb,) * 3
        L = ng[0] * h
        centres = rng.uniform(-L / 2, L / 2, size=(64, 3))
        Vc, _ = _potential_cells(ng, (h,) * 3, centres, -1.0, 1.5, 1e-3, rng)
        m = int(round(natoms ** (1 / 3)))
        assert m ** 3 == natoms
        a = L / m
        grid = (np.arange(m) + 0.5) * a - L / 2
        pos = np.array(np.meshgrid(grid, grid, grid, indexing="ij")).reshape(3, -1).T[:, ::-1]
        pos = pos + rng.uniform(-0.3, 0.3, size=pos.shape)
        atoms = np.zeros((natoms, 8))
        atoms[:, :3] = pos; atoms[:, 3] = 1; atoms[:, 4] = np.arange(natoms); atoms[:, 5] = 5; atoms[:, 6] = 0.6
        mats, offs = _atom_matrices([5] * natoms, [0.6] * natoms, rng)
        geo = Geometry(ng, (1, 1, 1), (h,) * 3, 12.0, src, 4, 6.0, atoms)
        return Workload(name, geo, Vc, mats, offs, complex(-0.2, 0.02), np.zeros(3), h ** 3, 1e-8, 2000)
    if name == "wrapped32_256atoms":
        nb = 32
        ng = (4 * nb,) * 3
        L = ng[0] * h
        centres = rng.uniform(-L / 2, L / 2, size=(256, 3))
        Vc, _ = _potential_cells(ng, (h,) * 3, centres, -1.0, 1.5, 1e-3, rng)
        # 8 x 8 x 4 sites over the whole cell (4 Bohr apart in x and y, 8 Bohr in z)
        gxy = (np.arange(8) + 0.5) * (L / 8) - L / 2
        gz = (np.arange(4) + 0.5) * (L / 4) - L / 2
        pos = np.array(np.meshgrid(gxy, gxy, gz, indexing="ij")).reshape(3, -1).T
        pos = pos + rng.uniform(-0.3, 0.3, size=pos.shape)
        natoms = len(pos)
        atoms = np.zeros((natoms, 8))
        atoms[:, :3] = pos; atoms[:, 3] = 1; atoms[:, 4] = np.arange(natoms); atoms[:, 5] = 5; atoms[:, 6] = 0.6
        mats, offs = _atom_matrices([5] * natoms, [0.6] * natoms, rng)
        geo = Geometry(ng, (1, 1, 1), (h,) * 3, 12.0, (4, 4, 2), 4, 6.0, atoms)
        return Workload(name, geo, Vc, mats, offs, complex(-0.2, 0.02), np.zeros(3), h ** 3, 1e-10, 2000)
    raise KeyError(name)


def random_blocks(nnzb, rng, dtype=np.float64):
    """Random block vector [nnzb, 2, 64, 64]."""
    return rng.standard_normal((nnzb, 2, 64, 64)).astype(dtype)


def contour_semicircle(n=32, e_bottom=-1.0, e_top=0.0):
    """Energy points and complex weights of a semicircular contour from e_bottom to e_top in the
    upper half plane, Gauss-Legendre in the angle: E(theta) = c + R exp(i theta), theta from pi
    to 0 (c the midpoint, R the radius).  With 32 points the imaginary parts run from about
    1.1e-3 to 0.5 Ha for the interval [-1, 0]."""
    x, wx = np.polynomial.legendre.leggauss(n)
    c, R = 0.5 * (e_bottom + e_top), 0.5 * (e_top - e_bottom)
    theta = 0.5 * np.pi * (1.0 - x)                     # x = -1 -> pi (bottom), x = 1 -> 0 (top)
    E = c + R * np.exp(1j * theta)
    # dE = i R exp(i theta) dtheta, dtheta = -pi/2 dx
    w = 1j * R * np.exp(1j * theta) * (-0.5 * np.pi) * wx
    return E, w


def truncation_radius(E, scale=8.0, lo=8.0, hi=16.0):
    """r_trunc = clamp(8 / sqrt(Im E / 0.5), 8, 16) Bohr: longer-ranged Green functions close to
    the real axis."""
    return float(np.clip(scale / np.sqrt(np.imag(E) / 0.5), lo, hi))


def contour_kpoints(n=4, seed=7):
    """Gamma and n-1 seeded points in the irreducible wedge of the cubic Brillouin zone
    (0 <= k_z <= k_y <= k_x < 0.5, units of 2 pi / cell), equal weights."""
    rng = np.random.default_rng(seed)
    ks = [np.zeros(3)]
    while len(ks) < n:
        k = np.sort(rng.uniform(0.0, 0.5, size=3))[::-1]
        ks.append(k)
    return np.array(ks), np.full(n, 1.0 / n)


def batched_contour(name="periodic16_64atoms_s2x2x2", nE=32, nk=4):
    """The batched contour workload: the 16^3-cube cell with 64 atoms and 8 source cubes, nE
    energy points on the semicircle from -1 to 0 Ha, nk k-points.  Returns the workload, the
    (E, k) pairs in the reference's loop order (energies outer), their weights and truncation
    radii."""
    w = make(name)
    E, wE = contour_semicircle(nE)
    K, wK = contour_kpoints(nk)
    pairs = [(complex(e), k.copy(), complex(we) * wk, truncation_radius(e))
             for e, we in zip(E, wE) for k, wk in zip(K, wK)]
    return w, pairs
