"""The operator, mirroring green_action::action_t<real_t,R1C2=2,Noco=1,64>
(include/green_action.hxx:57-299): multiply(y, x, colIndex, nnzb, nCols, l2nX, stream) over
R1C2 64-column blocks, returning the reference's flop count.  x, y and colIndex are CUDA
tensors (or raw device addresses); the arithmetic runs in libangstromcube_b200.so.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr


def _dtype_code(real_t):
    name = str(real_t)
    if "float64" in name or "double" in name:
        return _lib.A43G_F64
    if "float32" in name or "float" in name:
        return _lib.A43G_F32
    raise TypeError("real_t must be float64 or float32, got %s" % name)


class action_t:
    """Implicit linear operator (H - E S) on block-sparse R1C2 data of one plan."""

    def __init__(self, plan, real_t="float64"):
        self.plan = plan
        self.real_t = real_t
        self.dtype = _dtype_code(real_t)
        self.LM = self.LN = 64

    def multiply(self, y, x, colIndex, nnzb, nCols=1, l2nX=0, stream=0):
        """y = (H - E S) x; returns the number of floating point operations (reference count)."""
        flops = ctypes.c_double(0)
        st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        check(_lib.lib().a43g_action_multiply(self.plan.handle, ptr(y), ptr(x), ptr(colIndex), int(nnzb), int(nCols),
                                              int(l2nX), st, self.dtype, ctypes.byref(flops)),
              "a43g_action_multiply")
        return flops.value

    def has_preconditioner(self):
        return False

    def get_plan(self):
        return self.plan


def solve_options(tolerance=1e-9, max_iterations=500, precision="float64", update_factor=0.0, update_gap=0,
                  check_every=10, seed=1, echo=0, retire=True, batch=0, precondition=False):
    """Options of a43g_solve (include/a43g.h): precision "float64" is plain FP64 tfQMR,
    "float32" the FP32 recurrences with the FP64 solution and residual replacement (a
    replacement when a source's estimate fell by update_factor or after update_gap iterations;
    0 takes the library defaults 0.1 and 10); retire=False keeps computing on finished source
    cubes (as the reference's solver library does); batch: pairs per wave of solve_batched;
    precondition: right preconditioning by the cube-diagonal local operator (A43G_SOLVE_PRECONDITION)."""
    o = _lib.SolveOptions()
    o.tolerance = tolerance
    o.max_iterations = max_iterations
    o.precision = _dtype_code(precision)
    o.update_factor = update_factor
    o.update_gap = update_gap
    o.check_every = check_every
    o.seed = seed
    o.echo = echo
    o.flags = (0 if retire else _lib.A43G_SOLVE_NO_RETIRE) | (_lib.A43G_SOLVE_PRECONDITION if precondition else 0)
    o.batch = batch
    return o


def solve(plan, X=None, want_rho=True, stream=0, **kw):
    """tfQMR solve of (H - E S) X = B (B: unit diagonal blocks).  X: optional CUDA tensor
    [nnzb, 2, 64, 64] receiving the solution (float64).  Returns (stats dict, rho) with
    rho complex [nCols, 64] = diag(G_diag)/pi as action_t::solve exports it."""
    opts = solve_options(**kw)
    stats = _lib.SolveStats()
    rho = np.zeros((plan.nCols, 64, 2)) if want_rho else None
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_solve(plan.handle, ctypes.byref(opts), ptr(X), ptr(rho), ctypes.byref(stats), st),
          "a43g_solve")
    return stats.as_dict(), (rho[..., 0] + 1j * rho[..., 1] if want_rho else None)


def solve_traced(plan, X_reference, every=10, X=None, want_rho=False, stream=0, capacity=100000, **kw):
    """solve() recording every `every` iterations the relative error of the current solution
    against X_reference (CUDA float64 tensor [nnzb, 2, 64, 64]).  Returns (stats, rho, trace) with
    trace a float64 array of rows [iteration, |X - X_reference| / |X_reference|, active sources]."""
    opts = solve_options(**kw)
    stats = _lib.SolveStats()
    rho = np.zeros((plan.nCols, 64, 2)) if want_rho else None
    tr = np.zeros((capacity, 3))
    count = ctypes.c_int32(0)
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_solve_traced(plan.handle, ctypes.byref(opts), ptr(X), ptr(rho), ctypes.byref(stats), st,
                                       ptr(X_reference), int(every), ptr(tr), int(capacity), ctypes.byref(count)),
          "a43g_solve_traced")
    return (stats.as_dict(), (rho[..., 0] + 1j * rho[..., 1] if want_rho else None),
            tr[:min(count.value, capacity)].copy())


def solve_batched(plan, energies, kpoints, dVol, want_rho=False, stream=0, **kw):
    """Solves for every (energy, k-point) pair on the plan's geometry."""
    E = np.ascontiguousarray(np.stack([np.real(energies), np.imag(energies)], axis=-1), dtype=np.float64)
    K = np.ascontiguousarray(kpoints, dtype=np.float64).reshape(-1, 3)
    n = len(E)
    assert len(K) == n
    opts = solve_options(**kw)
    stats = (_lib.SolveStats * n)()
    rho = np.zeros((n, plan.nCols, 64, 2)) if want_rho else None
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_solve_batched(plan.handle, ctypes.byref(opts), n, ptr(E), ptr(K), float(dVol), ptr(rho),
                                        stats, st), "a43g_solve_batched")
    out = [stats[i].as_dict() for i in range(n)]
    return out, (rho[..., 0] + 1j * rho[..., 1] if want_rho else None)


def vjp(plan, L, G, potential=True, matrices=True, positions=True, stream=0):
    """Derivatives of F = sum over blocks and columns of L^T (H - E S) G (complex, no
    conjugation) for CUDA float64 tensors L, G [nnzb, 2, 64, 64].  Returns a dict with
      "V": complex [ncells, 64]        dF/dV in cell-cube layout,
      "M": list of complex [nc, nc]    dF/dM_A per plan atom (order of export()["global_atom_ids"]),
      "R": complex [nAtoms, 3]         dF/dR_A (atom positions)."""
    e = plan.export()
    nat = len(e["AtomLmax"])
    ncs = [((int(l) + 1) * (int(l) + 2) * (int(l) + 3)) // 6 for l in e["AtomLmax"]]   # int8 in the export
    dV = np.zeros((plan.sizes["ncells"], 64, 2)) if potential else None
    dM = np.zeros(max(1, sum(2 * n * n for n in ncs))) if matrices else None
    dR = np.zeros((max(nat, 1), 3, 2)) if positions else None
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_vjp(plan.handle, ptr(L), ptr(G), ptr(dV), ptr(dM), ptr(dR), st), "a43g_vjp")
    out = {}
    if potential:
        out["V"] = dV[..., 0] + 1j * dV[..., 1]
    if matrices:
        mats, o = [], 0
        for n in ncs:
            mats.append(dM[o:o + n * n].reshape(n, n) + 1j * dM[o + n * n:o + 2 * n * n].reshape(n, n))
            o += 2 * n * n
        out["M"] = mats
    if positions:
        out["R"] = (dR[..., 0] + 1j * dR[..., 1])[:nat]
    return out


def get_projection_coefficients(plan, G, stream=0):
    """Atomic density matrices Im <p_i|G|p_j> (green_dyadic::get_projection_coefficients) of a
    CUDA float64 Green function G [nnzb, 2, 64, 64]: a list of [nSHO, nSHO] arrays in the order of
    export()["global_atom_ids"]."""
    e = plan.export()
    ns = [((int(l) + 1) * (int(l) + 2) * (int(l) + 3)) // 6 for l in e["AtomLmax"]]
    out = np.zeros(max(1, sum(n * n for n in ns)))
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_projection_coefficients(plan.handle, ptr(G), ptr(out), st), "a43g_projection_coefficients")
    res, o = [], 0
    for n in ns:
        res.append(out[o:o + n * n].reshape(n, n).copy())
        o += n * n
    return res


def autotune(plan, precision="float32", stream=0):
    """Chooses the action's schedule for this plan by timing (a43g_plan_autotune); returns the
    report text."""
    buf = ctypes.create_string_buffer(4096)
    st = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    check(_lib.lib().a43g_plan_autotune(plan.handle, _dtype_code(precision), st, buf, len(buf)), "a43g_plan_autotune")
    return buf.value.decode()


def solve_concurrent(geometry, V, atom_matrices, atom_offsets, energies, kpoints, dVol, workers=4,
                     layout="cells", **kw):
    """Batched solves of many (energy, k-point) pairs of one geometry, several at a time: one plan
    and one CUDA stream per worker thread (plans are independent, so their solves overlap on the
    GPU; small cells leave most of the GPU idle in a single solve).  Returns [(stats, rho)] in the
    order of the pairs."""
    import threading
    import torch
    from . import green_function as gf
    pairs = list(zip(energies, kpoints))
    out = [None] * len(pairs)
    errors = []

    def work(w):
        try:
            plan = gf.construct_Green_function(geometry)
            gf.update_potential(plan, V, atom_matrices, atom_offsets, layout=layout)
            stream = torch.cuda.Stream()
            for i in range(w, len(pairs), workers):
                E, k = pairs[i]
                gf.update_energy_parameter(plan, E, dVol)
                gf.update_phases(plan, k)
                out[i] = solve(plan, stream=stream, **kw)
            stream.synchronize()
            plan.close()
        except Exception as e:          # reported after all workers ended
            errors.append(e)

    threads = [threading.Thread(target=work, args=(w,)) for w in range(max(1, min(workers, len(pairs))))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out
