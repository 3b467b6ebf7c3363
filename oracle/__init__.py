"""TEST INFRASTRUCTURE ONLY -- the oracle.

Two CPU implementations of the reference's Green-function action, used as checkers:

* ``RefGreen``  -- the reference's own sources (real-space/AngstromCube) compiled as a CPU
  build into ``oracle/_ref/libref_green.so`` by ``oracle/Makefile`` plus ``ref_shim.cxx``.
  Plans, potential, atom matrices and the action come straight from the reference code.
* ``restated_action`` -- ``green_oracle.c``, a plain-C restatement of the action that takes
  the plan arrays; it is pinned against ``RefGreen`` and the reference's analytic
  finite-difference known answers.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
package.  The product (``angstromcube_b200``) never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_green.so")
RESTATED_LIB = os.path.join(HERE, "liboracle_green.so")

_c_int64_p = ctypes.POINTER(ctypes.c_int64)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class _RefGeometry(ctypes.Structure):
    _fields_ = [("ng", ctypes.c_int32 * 3), ("bc", ctypes.c_int32 * 3), ("hg", ctypes.c_double * 3),
                ("r_trunc", ctypes.c_double), ("sources", ctypes.c_double * 3), ("nFD", ctypes.c_int32),
                ("proj_radius", ctypes.c_double), ("natoms", ctypes.c_int32),
                ("xyzZinso", ctypes.c_void_p), ("echo", ctypes.c_int32)]


_EXPORT_FIELDS = [
    "rowstart", "colindx", "rowindx", "veff_index", "subset", "rowCubePos", "colCubePos",
    "target_minus_source", "grid_spacing_trunc", "kinetic_prefactor",
    "lists_start0", "lists_start1", "lists_start2", "lists0", "lists1", "lists2",
    "AtomStarts", "AtomLmax", "AtomSigma", "global_atom_ids", "AtomImageIndex", "AtomImageStarts",
    "AtomImagePos", "AtomImageLmax", "AtomImageShift", "AtomImagePhase", "grid_spacing_dyadic",
    "SHOadd_start", "SHOadd_col", "SHOprj_start", "SHOprj_col", "SHOsum_start", "SHOsum_col",
    "AtomMatrices", "phase"]


class _RefExport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in _EXPORT_FIELDS]


def ref_available():
    return os.path.exists(REF_LIB)


_ref_lib = None


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_plan_build.restype = ctypes.c_void_p
        lib.ref_plan_build.argtypes = [ctypes.POINTER(_RefGeometry)]
        lib.ref_plan_free.argtypes = [ctypes.c_void_p]
        lib.ref_plan_sizes.argtypes = [ctypes.c_void_p, _c_int64_p]
        lib.ref_plan_export.argtypes = [ctypes.c_void_p, ctypes.POINTER(_RefExport)]
        lib.ref_set_potential.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_set_atom_matrices.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_set_energy.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.ref_set_kpoint.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_projection_coefficients.restype = ctypes.c_int
        lib.ref_projection_coefficients.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_action_f64.restype = ctypes.c_double
        lib.ref_action_f64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_action_f32.restype = ctypes.c_double
        lib.ref_action_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_set_phase.restype = ctypes.c_double
        lib.ref_set_phase.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ref_sho_prefactors.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        _ref_lib = lib
    return _ref_lib


SIZE_KEYS = ["nnzb", "nRows", "nCols", "nAtoms", "nAtomImages", "ncoeff_images", "ncoeffs",
             "nlists0", "nlists1", "nlists2", "lists_nnz0", "lists_nnz1", "lists_nnz2",
             "SHOadd_nnz", "SHOprj_nnz", "SHOsum_nnz", "FD_range0", "FD_range1", "FD_range2", "ncells"]


class RefGreen:
    """The reference's own CPU build: plan construction and action_t::multiply."""

    def __init__(self, geometry, echo=0):
        """geometry: angstromcube_b200 Geometry-like object with ng, bc, hg, r_trunc, sources,
        nFD, proj_radius and atoms (xyzZinso rows)."""
        self.lib = _load_ref()
        g = _RefGeometry()
        for d in range(3):
            g.ng[d] = int(geometry.ng[d]); g.bc[d] = int(geometry.bc[d]); g.hg[d] = float(geometry.hg[d])
            g.sources[d] = float(geometry.sources[d])
        g.r_trunc = float(geometry.r_trunc); g.nFD = int(geometry.nFD)
        g.proj_radius = float(geometry.proj_radius)
        self._xyz = np.ascontiguousarray(np.asarray(geometry.xyzZinso, dtype=np.float64).reshape(-1))
        g.natoms = len(self._xyz) // 8
        g.xyzZinso = self._xyz.ctypes.data if g.natoms else None
        g.echo = echo
        self.h = self.lib.ref_plan_build(ctypes.byref(g))
        if not self.h:
            raise RuntimeError("reference construct_Green_function failed")
        s = np.zeros(20, dtype=np.int64)
        self.lib.ref_plan_sizes(self.h, s.ctypes.data_as(_c_int64_p))
        self.sizes = dict(zip(SIZE_KEYS, (int(v) for v in s)))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_plan_free(self.h)
            self.h = None

    def export(self):
        s = self.sizes
        nnzb, nR, nC, nA, nAI = s["nnzb"], s["nRows"], s["nCols"], s["nAtoms"], s["nAtomImages"]
        a = {
            "rowstart": np.zeros(nR + 1, np.uint32), "colindx": np.zeros(nnzb, np.uint16),
            "rowindx": np.zeros(nnzb, np.uint32), "veff_index": np.zeros(nnzb, np.int32),
            "subset": np.zeros(nC, np.uint32), "rowCubePos": np.zeros((nR, 4), np.float32),
            "colCubePos": np.zeros((nC, 4), np.float32),
            "target_minus_source": np.zeros((nnzb, 4), np.int16),
            "grid_spacing_trunc": np.zeros(3), "kinetic_prefactor": np.zeros(3),
            "AtomStarts": np.zeros(nA + 1, np.uint32), "AtomLmax": np.zeros(nA, np.int8),
            "AtomSigma": np.zeros(nA), "global_atom_ids": np.zeros(nA, np.int64),
            "AtomImageIndex": np.zeros(nAI, np.uint32), "AtomImageStarts": np.zeros(nAI + 1, np.uint32),
            "AtomImagePos": np.zeros((nAI, 4)), "AtomImageLmax": np.zeros(nAI, np.int8),
            "AtomImageShift": np.zeros((nAI, 4), np.int8), "AtomImagePhase": np.zeros((nAI, 4)),
            "grid_spacing_dyadic": np.zeros(4),
            "SHOadd_start": np.zeros(nnzb + 1, np.uint32), "SHOadd_col": np.zeros(s["SHOadd_nnz"], np.uint32),
            "SHOprj_start": np.zeros(nC * (nAI + 1), np.uint32), "SHOprj_col": np.zeros(s["SHOprj_nnz"], np.uint32),
            "SHOsum_start": np.zeros(nA + 1, np.uint32), "SHOsum_col": np.zeros(s["SHOsum_nnz"], np.uint32),
            "phase": np.zeros((3, 2, 2)),
        }
        nmat = 0
        e = _RefExport()
        for k, v in a.items():
            setattr(e, k, v.ctypes.data if v.size else None)
        for dd in range(3):
            a["lists_start%d" % dd] = np.zeros(s["nlists%d" % dd] + 1, np.uint32)
            a["lists%d" % dd] = np.zeros(s["lists_nnz%d" % dd], np.int32)
            setattr(e, "lists_start%d" % dd, a["lists_start%d" % dd].ctypes.data)
            setattr(e, "lists%d" % dd, a["lists%d" % dd].ctypes.data if a["lists%d" % dd].size else None)
        self.lib.ref_plan_export(self.h, ctypes.byref(e))
        lm = a["AtomLmax"].astype(np.int64)
        nc = (lm + 1) * (lm + 2) * (lm + 3) // 6
        nmat = int(np.sum(2 * nc * nc))
        mats = np.zeros(max(nmat, 1))
        e2 = _RefExport()
        e2.AtomMatrices = mats.ctypes.data
        self.lib.ref_plan_export(self.h, ctypes.byref(e2))
        a["AtomMatrices"] = mats[:nmat]
        a["FD_range"] = np.array([s["FD_range%d" % d] for d in range(3)], np.int32)
        return a

    def set_potential(self, Vcell):
        V = np.ascontiguousarray(Vcell, dtype=np.float64)
        assert V.shape == (self.sizes["ncells"], 64)
        self.lib.ref_set_potential(self.h, _ptr(V))

    def set_atom_matrices(self, mats, offsets):
        m = np.ascontiguousarray(mats, dtype=np.float64)
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        self.lib.ref_set_atom_matrices(self.h, _ptr(m), _ptr(o))

    def set_energy(self, E, dVol):
        self.lib.ref_set_energy(self.h, float(np.real(E)), float(np.imag(E)), float(dVol))

    def set_kpoint(self, k):
        kk = np.ascontiguousarray(k, dtype=np.float64)
        self.lib.ref_set_kpoint(self.h, _ptr(kk))

    def projection_coefficients(self, G):
        """green_dyadic::get_projection_coefficients: Im <p_i|G|p_j> of every plan atom for an FP64
        block vector G [nnzb, 2, 64, 64]; a list of [nSHO, nSHO] arrays, or None where the
        reference refuses (plans with periodic atom images)."""
        e = self.export()
        ns = [((int(l) + 1) * (int(l) + 2) * (int(l) + 3)) // 6 for l in e["AtomLmax"]]
        out = np.zeros(max(1, sum(n * n for n in ns)))
        G = np.ascontiguousarray(G, dtype=np.float64)
        if self.lib.ref_projection_coefficients(self.h, _ptr(G), _ptr(out)) != 0:
            return None
        res, o = [], 0
        for n in ns:
            res.append(out[o:o + n * n].reshape(n, n).copy())
            o += n * n
        return res

    def action(self, x):
        """y = (H - E S) x for x of shape [nnzb, 2, 64, 64], float64 or float32."""
        x = np.ascontiguousarray(x)
        y = np.zeros_like(x)
        if x.dtype == np.float64:
            self.lib.ref_action_f64(self.h, _ptr(y), _ptr(x))
        elif x.dtype == np.float32:
            self.lib.ref_action_f32(self.h, _ptr(y), _ptr(x))
        else:
            raise TypeError(x.dtype)
        return y


def ref_set_phase(angle):
    lib = _load_ref()
    ph = np.zeros((2, 2))
    dev = lib.ref_set_phase(_ptr(ph), float(angle))
    return ph, dev


def ref_sho_prefactors(numax, sigma):
    lib = _load_ref()
    n = (numax + 1) * (numax + 2) * (numax + 3) // 6
    out = np.zeros(n)
    lib.ref_sho_prefactors(_ptr(out), int(numax), float(sigma))
    return out


def ref_quadrature(kind, n):
    """The reference's quadrature tables (src/energy_contour.cxx:456, :2156): kind "legendre"
    or "fermi_dirac"; nodes ascending and weights."""
    lib = _load_ref()
    x = np.zeros(256); w = np.zeros(256)
    f = lib.ref_gauss_legendre if kind == "legendre" else lib.ref_gauss_fermi_dirac
    m = f(_ptr(x), _ptr(w), ctypes.c_uint(int(n)))
    o = np.argsort(x[:m])
    return x[:m][o], w[:m][o]


def ref_energy_mesh(kBT, eBot, nBot, nPar, nFer, nPol):
    """energy_contour::get_energy_mesh (src/energy_contour.cxx:139-240): points and weights."""
    lib = _load_ref()
    E = np.zeros(2 * 512); W = np.zeros(2 * 512)
    lib.ref_energy_mesh.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_int]
    n = lib.ref_energy_mesh(_ptr(E), _ptr(W), 512, kBT, eBot, nBot, nPar, nFer, nPol)
    return E[:2 * n:2] + 1j * E[1:2 * n:2], W[:2 * n:2] + 1j * W[1:2 * n:2]


# ---------------------------------------------------------------- restated oracle (plain C)

class _OraclePlan(ctypes.Structure):
    _fields_ = [
        ("nnzb", ctypes.c_uint32), ("nRows", ctypes.c_uint32), ("nCols", ctypes.c_uint32),
        ("colindx", ctypes.c_void_p), ("rowindx", ctypes.c_void_p), ("veff_index", ctypes.c_void_p),
        ("Vcell", ctypes.c_void_p), ("E_re", ctypes.c_double), ("E_im", ctypes.c_double),
        ("nlists", ctypes.c_uint32 * 3), ("lists_start", ctypes.c_void_p * 3), ("lists", ctypes.c_void_p * 3),
        ("kinetic_prefactor", ctypes.c_double * 3), ("FD_range", ctypes.c_int32 * 3),
        ("phase", ctypes.c_double * 12),
        ("nAtoms", ctypes.c_uint32), ("nAtomImages", ctypes.c_uint32),
        ("AtomStarts", ctypes.c_void_p), ("AtomLmax", ctypes.c_void_p), ("AtomMatrices", ctypes.c_void_p),
        ("AtomImageStarts", ctypes.c_void_p), ("AtomImagePos", ctypes.c_void_p),
        ("AtomImageLmax", ctypes.c_void_p), ("AtomImagePhase", ctypes.c_void_p),
        ("grid_spacing", ctypes.c_void_p), ("rowCubePos", ctypes.c_void_p),
        ("SHOprj_start", ctypes.c_void_p), ("SHOprj_col", ctypes.c_void_p), ("SHOprj_coloff", ctypes.c_void_p),
        ("SHOadd_start", ctypes.c_void_p), ("SHOadd_col", ctypes.c_void_p),
        ("SHOsum_start", ctypes.c_void_p), ("SHOsum_col", ctypes.c_void_p)]


_restated = None


def restated_available():
    return os.path.exists(RESTATED_LIB)


def _load_restated():
    global _restated
    if _restated is None:
        lib = ctypes.CDLL(RESTATED_LIB)
        for name in ("oracle_potential", "oracle_action"):
            getattr(lib, name).argtypes = [ctypes.POINTER(_OraclePlan), ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_kinetic.argtypes = [ctypes.POINTER(_OraclePlan), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_dyadic.argtypes = [ctypes.POINTER(_OraclePlan), ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_set_phase.restype = ctypes.c_double
        lib.oracle_set_phase.argtypes = [ctypes.c_void_p, ctypes.c_double]
        _restated = lib
    return _restated


class RestatedOracle:
    """Wraps the plain-C restatement around a dict of plan arrays (as exported by RefGreen or
    by the product's plan builder), a cell potential, atom matrices and an energy."""

    def __init__(self, arrays, Vcell, E):
        self.lib = _load_restated()
        self.keep = []
        a = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
        self.a = a
        p = _OraclePlan()
        p.nnzb = len(a["colindx"]); p.nRows = len(a["rowstart"]) - 1; p.nCols = len(a["subset"])
        V = np.ascontiguousarray(Vcell, dtype=np.float64)
        self.keep.append(V)
        p.colindx = _ptr(a["colindx"]); p.rowindx = _ptr(a["rowindx"]); p.veff_index = _ptr(a["veff_index"])
        p.Vcell = _ptr(V); p.E_re = float(np.real(E)); p.E_im = float(np.imag(E))
        for dd in range(3):
            p.nlists[dd] = len(a["lists_start%d" % dd]) - 1
            p.lists_start[dd] = _ptr(a["lists_start%d" % dd]); p.lists[dd] = _ptr(a["lists%d" % dd])
            p.kinetic_prefactor[dd] = float(a["kinetic_prefactor"][dd]); p.FD_range[dd] = int(a["FD_range"][dd])
        ph = np.ascontiguousarray(a["phase"], dtype=np.float64).reshape(-1)
        for i in range(12):
            p.phase[i] = ph[i]
        p.nAtoms = len(a["AtomLmax"]); p.nAtomImages = len(a["AtomImageLmax"])
        for k in ("AtomStarts", "AtomLmax", "AtomMatrices", "AtomImageStarts", "AtomImagePos", "AtomImageLmax",
                  "AtomImagePhase", "rowCubePos", "SHOprj_start", "SHOprj_col", "SHOadd_start", "SHOadd_col",
                  "SHOsum_start", "SHOsum_col"):
            setattr(p, k, _ptr(a[k]) if a[k].size else None)
        p.grid_spacing = _ptr(a["grid_spacing_dyadic"])
        nAI = p.nAtomImages
        starts = a["SHOprj_start"].reshape(p.nCols, nAI + 1) if nAI else np.zeros((p.nCols, 1), np.uint32)
        coloff = np.zeros(p.nCols, np.uint64)
        if p.nCols > 1:
            coloff[1:] = np.cumsum(starts[:, -1].astype(np.uint64))[:-1]
        self.keep.append(coloff)
        p.SHOprj_coloff = _ptr(coloff)
        self.p = p

    def action(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.oracle_action(ctypes.byref(self.p), _ptr(y), _ptr(x))
        return y

    def potential(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.oracle_potential(ctypes.byref(self.p), _ptr(y), _ptr(x))
        return y

    def kinetic(self, x, dd):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.oracle_kinetic(ctypes.byref(self.p), int(dd), _ptr(y), _ptr(x))
        return y

    def dyadic(self, x, want_coefficients=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        ncI = int(self.a["AtomImageStarts"][-1]) if self.p.nAtomImages else 0
        apc = np.zeros((max(ncI, 1) * self.p.nCols, 2, 64)) if want_coefficients else None
        cad = np.zeros_like(apc) if want_coefficients else None
        self.lib.oracle_dyadic(ctypes.byref(self.p), _ptr(y), _ptr(x), _ptr(apc), _ptr(cad))
        return (y, apc, cad) if want_coefficients else y


def restated_set_phase(angle):
    lib = _load_restated()
    ph = np.zeros((2, 2))
    dev = lib.oracle_set_phase(_ptr(ph), float(angle))
    return ph, dev
