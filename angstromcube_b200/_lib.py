"""ctypes binding of include/a43g.h (libangstromcube_b200.so).

Loading fails loudly when the library has not been built: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libangstromcube_b200.so")

A43G_OK, A43G_ERR_ARGUMENT, A43G_ERR_CUDA, A43G_ERR_STATE, A43G_ERR_MEMORY, A43G_ERR_UNSUPPORTED = range(6)
A43G_F64, A43G_F32 = 0, 1

# every entry point declared in include/a43g.h
EXPORTED = [
    "a43g_last_error", "a43g_version", "a43g_plan_build", "a43g_plan_build_device", "a43g_plan_destroy", "a43g_plan_get_sizes",
    "a43g_plan_export", "a43g_plan_set_potential", "a43g_plan_set_atom_matrices", "a43g_plan_set_energy",
    "a43g_plan_set_kpoint", "a43g_plan_upload", "a43g_action_multiply", "a43g_action_part", "a43g_vjp", "a43g_plan_autotune", "a43g_action_multiply_noalloc",
    "a43g_kernel_launches", "a43g_plan_device_status", "a43g_solve", "a43g_solve_traced", "a43g_solve_batched",
    "a43g_hamiltonian_load", "a43g_hamiltonian_info", "a43g_hamiltonian_get", "a43g_hamiltonian_create",
    "a43g_hamiltonian_save", "a43g_hamiltonian_destroy", "a43g_projection_coefficients",
]


class Geometry(ctypes.Structure):
    _fields_ = [("ng", ctypes.c_uint32 * 3), ("bc", ctypes.c_int32 * 3), ("hg", ctypes.c_double * 3),
                ("r_trunc", ctypes.c_double), ("sources", ctypes.c_double * 3), ("nFD", ctypes.c_int32),
                ("proj_radius", ctypes.c_double), ("natoms", ctypes.c_int32), ("xyzZinso", ctypes.c_void_p)]


class PlanSizes(ctypes.Structure):
    _fields_ = [("nnzb", ctypes.c_int64), ("nRows", ctypes.c_int64), ("nCols", ctypes.c_int64),
                ("nAtoms", ctypes.c_int64), ("nAtomImages", ctypes.c_int64), ("ncoeff_images", ctypes.c_int64),
                ("ncoeffs", ctypes.c_int64), ("nlists", ctypes.c_int64 * 3), ("lists_nnz", ctypes.c_int64 * 3),
                ("SHOadd_nnz", ctypes.c_int64), ("SHOprj_nnz", ctypes.c_int64), ("SHOsum_nnz", ctypes.c_int64),
                ("FD_range", ctypes.c_int64 * 3), ("ncells", ctypes.c_int64)]


_EXPORT_NAMES = ["rowstart", "colindx", "rowindx", "veff_index", "subset", "rowCubePos", "colCubePos",
                 "target_minus_source", "grid_spacing_trunc", "kinetic_prefactor"]
_EXPORT_NAMES2 = ["AtomStarts", "AtomLmax", "AtomSigma", "global_atom_ids", "AtomImageIndex", "AtomImageStarts",
                  "AtomImagePos", "AtomImageLmax", "AtomImageShift", "AtomImagePhase", "grid_spacing_dyadic",
                  "SHOadd_start", "SHOadd_col", "SHOprj_start", "SHOprj_col", "SHOsum_start", "SHOsum_col",
                  "AtomMatrices", "phase"]


class PlanExport(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_void_p) for n in _EXPORT_NAMES] +
                [("lists_start", ctypes.c_void_p * 3), ("lists", ctypes.c_void_p * 3)] +
                [(n, ctypes.c_void_p) for n in _EXPORT_NAMES2])


A43G_SOLVE_NO_RETIRE = 1
A43G_SOLVE_PRECONDITION = 2


class SolveOptions(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("max_iterations", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("update_factor", ctypes.c_double), ("update_gap", ctypes.c_int32),
                ("check_every", ctypes.c_int32), ("seed", ctypes.c_uint64), ("echo", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("batch", ctypes.c_int32), ("pad", ctypes.c_int32)]


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("refinements", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("breakdowns", ctypes.c_int32), ("residual_max", ctypes.c_double),
                ("residual_estimate", ctypes.c_double), ("operator_applications", ctypes.c_double),
                ("seconds", ctypes.c_double), ("fp64_sources", ctypes.c_int32), ("pad", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """The loaded library (raises if it is missing: build it with python -m angstromcube_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libangstromcube_b200.so is not built (run python -m angstromcube_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, u32, f64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_double
        L.a43g_last_error.restype = ctypes.c_char_p
        L.a43g_version.restype = ctypes.c_char_p
        L.a43g_plan_build.argtypes = [ctypes.POINTER(Geometry), ctypes.POINTER(vp)]
        L.a43g_plan_build_device.argtypes = [ctypes.POINTER(Geometry), ctypes.POINTER(vp)]
        L.a43g_plan_destroy.argtypes = [vp]
        L.a43g_plan_get_sizes.argtypes = [vp, ctypes.POINTER(PlanSizes)]
        L.a43g_plan_export.argtypes = [vp, ctypes.POINTER(PlanExport)]
        L.a43g_plan_set_potential.argtypes = [vp, vp, i32]
        L.a43g_plan_set_atom_matrices.argtypes = [vp, vp, vp, ctypes.c_int64]
        L.a43g_plan_set_energy.argtypes = [vp, f64, f64, f64]
        L.a43g_plan_set_kpoint.argtypes = [vp, vp]
        L.a43g_plan_upload.argtypes = [vp]
        L.a43g_action_multiply.argtypes = [vp, vp, vp, vp, u32, u32, ctypes.c_uint, vp, i32, ctypes.POINTER(f64)]
        L.a43g_action_part.argtypes = [vp, i32, vp, vp, vp, i32]
        L.a43g_vjp.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.a43g_plan_autotune.argtypes = [vp, i32, vp, ctypes.c_char_p, ctypes.c_size_t]
        L.a43g_action_multiply_noalloc.argtypes = [vp, vp, vp, vp, u32, u32, vp, i32, ctypes.POINTER(f64)]
        L.a43g_kernel_launches.restype = ctypes.c_uint64
        L.a43g_plan_device_status.argtypes = [vp]
        L.a43g_solve.argtypes = [vp, ctypes.POINTER(SolveOptions), vp, vp, ctypes.POINTER(SolveStats), vp]
        L.a43g_solve_traced.argtypes = [vp, ctypes.POINTER(SolveOptions), vp, vp, ctypes.POINTER(SolveStats), vp,
                                        vp, i32, vp, i32, ctypes.POINTER(i32)]
        L.a43g_solve_batched.argtypes = [vp, ctypes.POINTER(SolveOptions), i32, vp, vp, f64, vp,
                                         ctypes.POINTER(SolveStats), vp]
        L.a43g_hamiltonian_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        L.a43g_hamiltonian_info.argtypes = [vp, vp, vp, vp, vp, vp]
        L.a43g_hamiltonian_get.argtypes = [vp, vp, vp, vp, vp]
        L.a43g_hamiltonian_create.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp, ctypes.POINTER(vp)]
        L.a43g_hamiltonian_save.argtypes = [vp, ctypes.c_char_p, i32, vp]
        L.a43g_hamiltonian_destroy.argtypes = [vp]
        L.a43g_projection_coefficients.argtypes = [vp, vp, vp, vp]
        for name in EXPORTED:
            if name not in ("a43g_last_error", "a43g_version", "a43g_kernel_launches"):
                getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


class A43GError(RuntimeError):
    def __init__(self, code, where):
        msg = lib().a43g_last_error().decode(errors="replace")
        super().__init__("%s failed with status %d: %s" % (where, code, msg))
        self.code = code


def check(code, where):
    if code != A43G_OK:
        raise A43GError(code, where)


def ptr(a):
    """ctypes address of a numpy array (host) or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p)
    return ctypes.c_void_p(a.data_ptr())
