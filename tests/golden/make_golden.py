"""Generates the golden fixtures of tests/golden from the reference's own CPU build
(oracle/_ref/libref_green.so, built by oracle/Makefile from the reference sources).

    python tests/golden/make_golden.py

plan_wrap6.npz     plan arrays of a wrapped 6^3-cube cell with 4 sources and 3 atoms
action_p2.npz      reference action_t<double,2,1>::multiply on a seeded x for a periodic
                   2^3-cube cell with one atom at k = (0.25, -1/3, 0.1): two full blocks of y and
                   per-block checksums (sum and weighted sum of squares) of all blocks
phase.npz          kinetic_plan::set_phase at every 5 degrees
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from helpers import geometry, inputs_for, reference_plan  # noqa: E402


def block_checksums(y):
    w = np.arange(1, 8193, dtype=np.float64).reshape(2, 64, 64) / 8192.0
    return np.stack([y.sum(axis=(1, 2, 3)), (w * y * y).sum(axis=(1, 2, 3))], axis=1)


def main():
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    g = geometry((6, 6, 6), (1, 1, 1), 2.4, (2, 2, 1), 4, 3, seed=11)
    r = oracle.RefGreen(g)
    a = r.export()
    np.savez_compressed(os.path.join(HERE, "plan_wrap6.npz"), **{"plan_" + k: v for k, v in a.items()})

    g = geometry((2, 2, 2), (1, 1, 1), 6.0, (1, 1, 1), 4, 1, seed=12, sigma=0.5, numax=2)
    Vc, mats, offs, E, _, dVol, _ = inputs_for(g, seed=13)
    k = np.array([0.25, -1 / 3.0, 0.1])
    r = reference_plan(g, Vc, mats, offs, E, k, dVol)
    x = np.random.default_rng(14).standard_normal((r.sizes["nnzb"], 2, 64, 64))
    y = r.action(x)
    np.savez_compressed(os.path.join(HERE, "action_p2.npz"), Vc=Vc, mats=mats, offs=offs, E=E, k=k, dVol=dVol,
                        x_seed=14, y_blocks=y[:2], checksums=block_checksums(y))

    angles = np.arange(-180, 181, 5) / 360.0
    ph = np.array([oracle.ref_set_phase(a)[0] for a in angles])
    np.savez_compressed(os.path.join(HERE, "phase.npz"), angles=angles, phase=ph)


if __name__ == "__main__":
    main()
