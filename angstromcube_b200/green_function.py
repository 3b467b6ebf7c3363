"""Plan construction and updates, mirroring the reference's green_function namespace
(src/green_function.cxx): construct_Green_function, update_potential, update_energy_parameter
and update_phases.  All work happens in the C++ plan builder behind include/a43g.h.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr

# boundary conditions (include/boundary_condition.hxx:17-30)
Isolated_Boundary, Periodic_Boundary, Vacuum_Boundary, Repeat_Boundary = 0, 1, 2, 3


class ActionPlan:
    """Owns an a43g plan handle (the counterpart of action_plan_t, include/action_plan.hxx:32-114)."""

    def __init__(self, geometry, on_device=False):
        g = _lib.Geometry()
        for d in range(3):
            g.ng[d] = int(geometry.ng[d]); g.bc[d] = int(geometry.bc[d]); g.hg[d] = float(geometry.hg[d])
            g.sources[d] = float(geometry.sources[d])
        g.r_trunc = float(geometry.r_trunc); g.nFD = int(geometry.nFD); g.proj_radius = float(geometry.proj_radius)
        self._xyz = np.ascontiguousarray(np.asarray(geometry.xyzZinso, dtype=np.float64).reshape(-1))
        g.natoms = len(self._xyz) // 8
        g.xyzZinso = self._xyz.ctypes.data if g.natoms else None
        h = ctypes.c_void_p()
        if on_device:
            check(_lib.lib().a43g_plan_build_device(ctypes.byref(g), ctypes.byref(h)), "a43g_plan_build_device")
        else:
            check(_lib.lib().a43g_plan_build(ctypes.byref(g), ctypes.byref(h)), "a43g_plan_build")
        self.handle = h
        s = _lib.PlanSizes()
        check(_lib.lib().a43g_plan_get_sizes(self.handle, ctypes.byref(s)), "a43g_plan_get_sizes")
        self.sizes = {"nnzb": s.nnzb, "nRows": s.nRows, "nCols": s.nCols, "nAtoms": s.nAtoms,
                      "nAtomImages": s.nAtomImages, "ncoeff_images": s.ncoeff_images, "ncoeffs": s.ncoeffs,
                      "SHOadd_nnz": s.SHOadd_nnz, "SHOprj_nnz": s.SHOprj_nnz, "SHOsum_nnz": s.SHOsum_nnz,
                      "ncells": s.ncells}
        for d in range(3):
            self.sizes["nlists%d" % d] = s.nlists[d]
            self.sizes["lists_nnz%d" % d] = s.lists_nnz[d]
            self.sizes["FD_range%d" % d] = s.FD_range[d]
        self.geometry = geometry

    @property
    def nnzb(self):
        return self.sizes["nnzb"]

    @property
    def nCols(self):
        return self.sizes["nCols"]

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().a43g_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        """Host copies of all plan arrays (same names and layouts as the reference's members)."""
        s = self.sizes
        nnzb, nR, nC, nA, nAI = s["nnzb"], s["nRows"], s["nCols"], s["nAtoms"], s["nAtomImages"]
        a = {
            "rowstart": np.zeros(nR + 1, np.uint32), "colindx": np.zeros(nnzb, np.uint16),
            "rowindx": np.zeros(nnzb, np.uint32), "veff_index": np.zeros(nnzb, np.int32),
            "subset": np.zeros(nC, np.uint32), "rowCubePos": np.zeros((nR, 4), np.float32),
            "colCubePos": np.zeros((nC, 4), np.float32), "target_minus_source": np.zeros((nnzb, 4), np.int16),
            "grid_spacing_trunc": np.zeros(3), "kinetic_prefactor": np.zeros(3),
            "AtomStarts": np.zeros(nA + 1, np.uint32), "AtomLmax": np.zeros(nA, np.int8), "AtomSigma": np.zeros(nA),
            "global_atom_ids": np.zeros(nA, np.int64), "AtomImageIndex": np.zeros(nAI, np.uint32),
            "AtomImageStarts": np.zeros(nAI + 1, np.uint32), "AtomImagePos": np.zeros((nAI, 4)),
            "AtomImageLmax": np.zeros(nAI, np.int8), "AtomImageShift": np.zeros((nAI, 4), np.int8),
            "AtomImagePhase": np.zeros((nAI, 4)), "grid_spacing_dyadic": np.zeros(4),
            "SHOadd_start": np.zeros(nnzb + 1, np.uint32), "SHOadd_col": np.zeros(s["SHOadd_nnz"], np.uint32),
            "SHOprj_start": np.zeros(nC * (nAI + 1), np.uint32), "SHOprj_col": np.zeros(s["SHOprj_nnz"], np.uint32),
            "SHOsum_start": np.zeros(nA + 1, np.uint32), "SHOsum_col": np.zeros(s["SHOsum_nnz"], np.uint32),
            "phase": np.zeros((3, 2, 2)),
        }
        lm = a["AtomLmax"]
        e = _lib.PlanExport()
        for k, v in a.items():
            setattr(e, k, v.ctypes.data if v.size else None)
        for d in range(3):
            a["lists_start%d" % d] = np.zeros(s["nlists%d" % d] + 1, np.uint32)
            a["lists%d" % d] = np.zeros(s["lists_nnz%d" % d], np.int32)
            e.lists_start[d] = a["lists_start%d" % d].ctypes.data
            e.lists[d] = a["lists%d" % d].ctypes.data if a["lists%d" % d].size else None
        check(_lib.lib().a43g_plan_export(self.handle, ctypes.byref(e)), "a43g_plan_export")
        lm = a["AtomLmax"].astype(np.int64)
        nc = (lm + 1) * (lm + 2) * (lm + 3) // 6
        mats = np.zeros(max(int(np.sum(2 * nc * nc)), 1))
        e2 = _lib.PlanExport()
        e2.AtomMatrices = mats.ctypes.data
        check(_lib.lib().a43g_plan_export(self.handle, ctypes.byref(e2)), "a43g_plan_export")
        a["AtomMatrices"] = mats[:int(np.sum(2 * nc * nc))]
        a["FD_range"] = np.array([s["FD_range%d" % d] for d in range(3)], np.int32)
        return a

    def upload(self):
        check(_lib.lib().a43g_plan_upload(self.handle), "a43g_plan_upload")


def construct_Green_function(geometry, on_device=False):
    """Build the plan (src/green_function.cxx:357-1068); on_device: the atom-image x target-row
    test of the dyadic plan on the current CUDA device (same arrays)."""
    return ActionPlan(geometry, on_device)


def update_potential(plan, V, atom_matrices=None, atom_offsets=None, layout="grid"):
    """Set the local potential (full grid, natural order, or cell cubes [ncells][64]) and
    optionally the atom matrices (src/green_function.cxx:114-211)."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    lay = {"grid": 0, "cells": 1}[layout]
    check(_lib.lib().a43g_plan_set_potential(plan.handle, ptr(V), lay), "a43g_plan_set_potential")
    if atom_matrices is not None:
        m = np.ascontiguousarray(atom_matrices, dtype=np.float64)
        o = np.ascontiguousarray(atom_offsets, dtype=np.int64)
        check(_lib.lib().a43g_plan_set_atom_matrices(plan.handle, ptr(m), ptr(o), len(o)),
              "a43g_plan_set_atom_matrices")


def update_energy_parameter(plan, E, dVol):
    """M_a = dVol (dH_a - E dS_a) and the local E (src/green_function.cxx:64-109)."""
    check(_lib.lib().a43g_plan_set_energy(plan.handle, float(np.real(E)), float(np.imag(E)), float(dVol)),
          "a43g_plan_set_energy")


def update_phases(plan, k_point):
    """Bloch phases of the finite-difference halos and the atom images (src/green_function.cxx:218-251)."""
    k = np.ascontiguousarray(k_point, dtype=np.float64)
    check(_lib.lib().a43g_plan_set_kpoint(plan.handle, ptr(k)), "a43g_plan_set_kpoint")
