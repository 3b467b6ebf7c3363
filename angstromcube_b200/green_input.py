"""The grid Hamiltonian file (Hmt.xml / Hmt.json), mirroring green_input::load_Hamiltonian
(src/green_input.cxx:29-221) and grid_operators::write_to_file (include/grid_operators.hxx:
460-613).  Parsing and writing happen in libangstromcube_b200.so (a43g_hamiltonian_*).

    ng, bc, hg, Veff, natoms, xyzZinso, atom_mat = load_Hamiltonian("Hmt.xml")
    write_to_file("Hmt.json", ng, bc, hg, Veff, xyzZinso, atom_mat, fileformat="json")
    geometry, Vcell_grid, mats, offsets = geometry_from_file("Hmt.xml", r_trunc=..., sources=...)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr


def load_Hamiltonian(filename):
    """(ng[3], bc[3], hg[3], Veff [nz, ny, nx], natoms, xyzZinso [natoms, 8], atom_mat list of
    [2, nSHO, nSHO]) as the reference's loader returns them."""
    h = ctypes.c_void_p()
    check(_lib.lib().a43g_hamiltonian_load(str(filename).encode(), ctypes.byref(h)), "a43g_hamiltonian_load")
    try:
        ng = np.zeros(3, np.uint32); bc = np.zeros(3, np.int32); hg = np.zeros(3)
        na = ctypes.c_int32(0); nm = ctypes.c_int64(0)
        check(_lib.lib().a43g_hamiltonian_info(h, ptr(ng), ptr(bc), ptr(hg), ctypes.byref(na), ctypes.byref(nm)),
              "a43g_hamiltonian_info")
        V = np.zeros((int(ng[2]), int(ng[1]), int(ng[0])))
        xyz = np.zeros((na.value, 8))
        mats = np.zeros(max(nm.value, 1))
        offs = np.zeros(max(na.value, 1), np.int64)
        check(_lib.lib().a43g_hamiltonian_get(h, ptr(V), ptr(xyz), ptr(mats), ptr(offs)), "a43g_hamiltonian_get")
    finally:
        _lib.lib().a43g_hamiltonian_destroy(h)
    atom_mat = []
    for a in range(na.value):
        numax = int(xyz[a, 5])
        n = (numax + 1) * (numax + 2) * (numax + 3) // 6
        atom_mat.append(mats[offs[a]:offs[a] + 2 * n * n].reshape(2, n, n).copy())
    return ng.astype(int), bc.astype(int), hg, V, na.value, xyz, atom_mat


def write_to_file(filename, ng, bc, hg, Veff, xyzZinso, atom_mat, fileformat="xml", spectrum=None):
    """Write a grid Hamiltonian in the reference's XML or JSON layout."""
    ng = np.ascontiguousarray(ng, np.uint32); bc = np.ascontiguousarray(bc, np.int32)
    hg = np.ascontiguousarray(hg, np.float64)
    V = np.ascontiguousarray(Veff, np.float64).reshape(-1)
    xyz = np.ascontiguousarray(xyzZinso, np.float64).reshape(-1, 8)
    mats = np.concatenate([np.ascontiguousarray(m, np.float64).ravel() for m in atom_mat]) if atom_mat else np.zeros(1)
    offs = np.cumsum([0] + [np.asarray(m).size for m in atom_mat[:-1]]).astype(np.int64) if atom_mat else np.zeros(1, np.int64)
    h = ctypes.c_void_p()
    check(_lib.lib().a43g_hamiltonian_create(ptr(ng), ptr(bc), ptr(hg), ptr(V), len(xyz), ptr(xyz), ptr(mats), ptr(offs),
                                             ctypes.byref(h)), "a43g_hamiltonian_create")
    sp = None if spectrum is None else np.ascontiguousarray(spectrum, np.float64)
    try:
        check(_lib.lib().a43g_hamiltonian_save(h, str(filename).encode(), 1 if fileformat == "json" else 0, ptr(sp)),
              "a43g_hamiltonian_save")
    finally:
        _lib.lib().a43g_hamiltonian_destroy(h)


def geometry_from_file(filename, r_trunc, sources=(1, 1, 1), nFD=4, proj_radius=6.0):
    """The plan geometry of a Hamiltonian file (the cell, boundary conditions, spacing and atoms
    the reference's construct_Green_function receives from load_Hamiltonian), the potential on
    the full grid and the atom matrices concatenated with their offsets (per atom id) for
    green_function.update_potential(..., layout="grid")."""
    from .workloads import Geometry
    ng, bc, hg, V, natoms, xyz, mats = load_Hamiltonian(filename)
    # the plan takes atom ids as indices into the matrix list: renumber in file order
    xyz = xyz.copy()
    xyz[:, 4] = np.arange(natoms)
    geo = Geometry(tuple(int(n) for n in ng), tuple(int(b) for b in bc), tuple(float(h) for h in hg), float(r_trunc),
                   tuple(sources), nFD, proj_radius, xyz)
    flat = np.concatenate([m.ravel() for m in mats]) if mats else np.zeros(1)
    offs = np.cumsum([0] + [m.size for m in mats[:-1]]).astype(np.int64) if mats else np.zeros(0, np.int64)
    return geo, V, flat, offs
