"""Host logic of bench.py that needs no GPU: the DRAM traffic table under profiles/ and the
naming of the local kernel the autotuner chose."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_traffic_table_has_the_local_kernels():
    b = load_bench()
    assert b.read_traffic("local_pencil_kernel_f32") == 66275
    assert b.read_traffic("local_fused_pf_kernel_f32") == 70326
    assert b.read_traffic("local_pencil64_kernel_f64") == 159058
    assert b.read_traffic("no_such_kernel") is None


def test_local_kernel_named_from_the_autotuner_choice():
    b = load_bench()
    line = ["chosen: projector chunk 32, addition 8 blocks per CTA, local %s, CUDA-core projector"]
    name, key = b.local_kernel_of([line[0] % "pencils"])
    assert name.startswith("local_pencil_kernel") and key == "local_pencil_kernel_f32"
    name, key = b.local_kernel_of([line[0] % "rows with loads ahead"])
    assert name.startswith("local_fused_pf_kernel") and key == "local_fused_pf_kernel_f32"
    name, key = b.local_kernel_of([line[0] % "plain rows"])
    assert name.startswith("local_fused_kernel") and key is None


def test_pair_walk_is_a_permutation_spread_over_the_contour():
    b = load_bench()
    order = b.pair_order(128)
    assert sorted(order) == list(range(128))
    # consecutive solves are far apart on the contour (energies are the outer loop, 4 k-points)
    assert all(abs(order[i + 1] // 4 - order[i] // 4) >= 8 for i in range(20))


def test_contour_workload():
    """32 Gauss-Legendre energies on the semicircle from -1 to 0 Ha (imaginary parts 2.1e-3 to
    0.5 Ha), 4 k-points, truncation radii clamp(8/sqrt(Im E/0.5), 8, 16); the weights integrate
    a constant and a linear function of E along the semicircle exactly."""
    import numpy as np
    from angstromcube_b200 import workloads
    w, pairs = workloads.batched_contour()
    assert len(pairs) == 128 and w.geometry.sources == (2, 2, 2)
    E = np.array([p[0] for p in pairs[::4]])
    assert 2e-3 < E.imag.min() < 2.2e-3 and 0.498 < E.imag.max() <= 0.5
    Es, ws = workloads.contour_semicircle(32)
    assert abs(ws.sum() - (0.0 - (-1.0))) < 1e-13          # integral of dE from -1 to 0
    assert abs((ws * Es).sum() - (0.0 - 1.0) / 2) < 1e-13  # integral of E dE
    rs = [p[3] for p in pairs]
    assert min(rs) > 8.0 and max(rs) == 16.0
    K, wk = workloads.contour_kpoints()
    assert np.all(K[0] == 0) and np.all(K[1:] < 0.5) and np.all(K[1:, 0] >= K[1:, 1]) and abs(wk.sum() - 1) < 1e-15
