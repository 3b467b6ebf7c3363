"""Distribution of Green-function solves over ranks (one process per GPU).

The solves of different (energy, k-point) pairs and of disjoint source-cube sets are
independent: the action never couples them (the reference distributes source cubes over MPI
ranks, src/green_function.cxx:262-307, and loops over (E, k) serially,
src/energy_contour.cxx:355-386).  A contour integration therefore shards its (E, k) points over
ranks and sums the weighted densities once at the end with one all-reduce.
"""
import numpy as np


def shard(n_items, world, rank):
    """Contiguous, balanced share [start, stop) of n_items for a rank."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def contour_points(energies, weights, kpoints, kweights):
    """All (E, k) pairs with their combined weights, in the reference's loop order
    (energies outer, k-points inner)."""
    pts = []
    for E, wE in zip(energies, weights):
        for k, wk in zip(kpoints, kweights):
            pts.append((complex(E), complex(wE) * wk, np.asarray(k, float)))
    return pts


def reduce_density(rho_local, group=None):
    """Sum the complex densities [nCols, 64] of all ranks (torch.distributed all-reduce)."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.stack([rho_local.real, rho_local.imag], axis=-1))
    if dist.is_available() and dist.is_initialized():
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, group=group)
    t = t.cpu().numpy()
    return t[..., 0] + 1j * t[..., 1]


def integrate(points, solve_point, world=1, rank=0, group=None):
    """Weighted density sum over the (E, k) points assigned to this rank, reduced over ranks.
    solve_point(E, k) returns the density [nCols, 64] of one solve."""
    start, stop = shard(len(points), world, rank)
    acc = None
    for E, w, k in points[start:stop]:
        rho = solve_point(E, k) * w
        acc = rho if acc is None else acc + rho
    if acc is None:
        acc = np.zeros_like(solve_point.zero()) if hasattr(solve_point, "zero") else None
    return reduce_density(acc, group)
