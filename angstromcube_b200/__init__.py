"""angstromcube_b200: B200-native (sm_100a) Green-function action (H - E S) X of AngstromCube
and its tfQMR solver, behind the C ABI of include/a43g.h.

    from angstromcube_b200 import green_function, green_action, workloads
    w = workloads.make("periodic4_1atom")
    plan = green_function.construct_Green_function(w.geometry)
    green_function.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    green_function.update_energy_parameter(plan, w.E, w.dVol)
    op = green_action.action_t(plan, "float64")
    op.multiply(y, x, colIndex, plan.nnzb, plan.nCols)      # CUDA tensors
"""
from . import _lib, green_action, green_function, workloads  # noqa: F401

__all__ = ["green_action", "green_function", "workloads"]
