"""Multi-rank host logic on CPU: world size 2 with the gloo backend (127.0.0.1).  The solve of
one (E, k) point is replaced by a deterministic function of (E, k) so that the sharded,
all-reduced contour sum can be compared with the serial sum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from angstromcube_b200 import parallel


def fake_solve(E, k):
    x = np.arange(4 * 64, dtype=float).reshape(4, 64)
    return (np.cos(x * E.real + k.sum()) + 1j * np.sin(x * E.imag)) / (1 + abs(E))


def points():
    E = np.linspace(-1, 0, 5) + 0.1j
    w = np.linspace(0.1, 0.5, 5) + 0.01j
    ks = [np.zeros(3), np.array([0.25, 0, 0]), np.array([0.25, 0.25, 0])]
    return parallel.contour_points(E, w, ks, [0.5, 0.25, 0.25])


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rho = parallel.integrate(points(), fake_solve, world, rank)
        out[rank] = rho
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _free_port():
    s = socket.socket(); s.bind(("127.0.0.1", 0)); p = s.getsockname()[1]; s.close()
    return p


def test_shard_covers_everything():
    for n in range(0, 23):
        for world in range(1, 5):
            parts = [parallel.shard(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_contour_sum_two_ranks_gloo():
    serial = sum(w * fake_solve(E, k) for E, w, k in points())
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    for r in range(2):
        assert np.allclose(out[r], serial, rtol=1e-12, atol=1e-12)
