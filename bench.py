"""Benchmark of the Green-function solver: solves/s at 1e-8 relative residual.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--wave P]
    python bench.py --full-contour [--nk K]     (every pair of the contour; a long run)

Workload (the batched contour): the periodic 16^3-cube cell (h = 0.25 Bohr) with 64 atoms
(numax 5, sigma 0.6) on a jittered 4^3 lattice and 64 Gaussian wells, 8 source cubes (512
right-hand-side columns), 32 energies on a semicircular Gauss-Legendre contour from -1 to 0 Ha
(imaginary parts 2.1e-3 to 0.5 Ha), each with its truncation radius clamp(8/sqrt(Im E/0.5), 8,
16) Bohr, times 4 k-points (Gamma and 3 seeded points of the irreducible wedge): 128 (E, k)
solves.  Every radius above 8 Bohr leaves the 16 Bohr cell untruncated, so all 128 share one
plan of 32,768 blocks (checked at set-up).  A solve is one (E, k) pair with all 512 columns at a
true FP64 relative residual below 1e-8.

A step solves one wave of --wave pairs (default 1) with a43g_solve_batched: FP32 recurrences and
operator, FP64 solution and residual replacement, finished source cubes retired, sources whose
FP32 recurrences stall continued in FP64.  The steps walk through the 128 pairs in a fixed order
that spreads them over the contour (pair 37*i mod 128 for the i-th solve), so a run of K steps
times a sample of K*P pairs of the whole contour; `value` counts the converged solves per second
of device time.  Reported beside it on the same pairs: the plain FP64 solver (the reference's
algorithm: FP64 tfQMR, no retirement, one pair at a time) on the first pairs of the sample, per
pair status and iterations, the fused local kernel and the projector against their rooflines,
and the reference's CPU action (oracle/_ref) timed on the host cores on a bounded sample and
extrapolated to a solve.  Each rank of a multi-GPU run solves its own pairs (weak scaling) and
the weighted densities of all ranks are summed with one NCCL all-reduce per step, as the
contour integration does.  --impl reference prints the reference CPU arm only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "periodic16_64atoms_s2x2x2"
PRECONDITION = True          # right preconditioning by the cube-diagonal local operator
TOLERANCE = 1e-8
MAX_ITERATIONS = 1500
STRIDE = 37            # walk of the 128 pairs: 37*i mod 128 (37 is coprime with 128)
METRIC = "Solves/s at 1e-8 resid (mixed+batched vs plain FP64); action % HBM peak"
# plain FP64 tfQMR iterations to 1e-8 of the 32 contour energies at Gamma, one source cube of this
# cell, measured with this repository's FP64 solver on a B200 (1500 = no convergence within 1500
# iterations); the reference arm, which runs without a GPU, extrapolates its action time to solves
# with them
FP64_ITERATIONS_GAMMA = [430, 387, 379, 361, 343, 300, 284, 242, 221, 209, 199, 195, 191, 184, 194, 198,
                         205, 211, 217, 242, 267, 292, 353, 408, 505, 646, 876, 1247, 1500, 1500, 1500, 1500]


def _json_default(o):
    """numpy scalars and arrays in the result line"""
    if hasattr(o, "tolist"):
        return o.tolist()
    return str(o)


def emit(obj):
    sys.stdout.write(json.dumps(obj, default=_json_default) + "\n")
    sys.stdout.flush()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--wave", type=int, default=1, help="(E, k) pairs per step")
    ap.add_argument("--fp64-pairs", type=int, default=2, help="pairs of the sample also solved in plain FP64")
    ap.add_argument("--full-contour", action="store_true", help="solve all pairs (mixed+batched and plain FP64)")
    ap.add_argument("--convergence-scan", action="store_true",
                    help="FP64 iterations over the contour energies and the residual history at -0.2+0.02i")
    ap.add_argument("--profile-case", choices=["action", "solve"], default=None,
                    help="small case for ncu captures on the one-source 16^3 cell (4096 blocks, 134 MB per FP32 "
                         "vector): 'action' applies the FP32 action with the CUDA-core and the tensor-core "
                         "projector and the FP64 action, 4 times each; 'solve' runs 40 iterations of the mixed "
                         "and of the FP64 solver")
    ap.add_argument("--wrapped32", action="store_true",
                    help="the wrapped 32^3-cube cell (256 atoms, 32 source cubes, 300,960 blocks) at "
                         "E = -0.2 + 0.02i to 1e-10: plain FP64 solve, then the mixed solve with the error of "
                         "G against it every 10 iterations")
    ap.add_argument("--wrapped32-iterations", type=int, default=2000, help="iteration limit of --wrapped32")
    ap.add_argument("--wrapped32-energy", type=complex, default=complex(-0.2, 0.02),
                    help="energy of --wrapped32 (Python complex literal, e.g. -0.2+0.1j)")
    ap.add_argument("--nk", type=int, default=4, help="k-points of the contour")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), p.get("bf16_tflops", 1590.0), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.rows)}


def pair_order(npairs):
    """The fixed walk through the pairs: 37 i mod npairs (a permutation when npairs is a power of
    two), spreading consecutive solves over the contour."""
    from math import gcd
    stride = STRIDE if gcd(STRIDE, npairs) == 1 else 1
    return [(stride * i) % npairs for i in range(npairs)]


# ------------------------------------------------------------------ reference CPU leg

def _ref_worker(args):
    """One process: the reference's action_t<double,2,1>::multiply (its CPU build in
    oracle/_ref) on the contour cell with ONE source cube; returns seconds per action."""
    workload, seed, reps, E = args
    # the reference's plan builder prints warnings on stdout: keep the JSON line alone there
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    import tempfile
    import numpy as np
    os.chdir(tempfile.mkdtemp())                 # the reference plan builder writes an SVG file
    sys.path.insert(0, ROOT)
    import oracle
    from angstromcube_b200 import workloads
    w = workloads.make(workload)
    g = w.geometry
    g.sources = (1, 1, 1)
    r = oracle.RefGreen(g)
    r.set_potential(w.Vcell)
    r.set_atom_matrices(w.mats, w.offsets)
    r.set_energy(E, w.dVol)
    x = np.random.default_rng(seed).standard_normal((r.sizes["nnzb"], 2, 64, 64))
    best = None
    for _ in range(reps):
        t = time.perf_counter()
        r.action(x)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return best


def cpu_action_seconds(workload, E, procs=None, reps=1):
    """Reference CPU action of one source cube, one process per host core in parallel; returns
    (seconds per single-source action (slowest process), processes)."""
    import multiprocessing as mp
    procs = procs or min(os.cpu_count() or 1, 32)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_worker, [(workload, i, reps, E) for i in range(procs)])
    return max(times), procs


def _ref_small_cell_solve(_):
    """The CPU-runnable configuration solved for real: the reference's CPU action inside the
    numpy restatement of tfQMR (oracle/tfqmr.py), FP64 to 1e-9.  Returns (iterations, seconds)."""
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    import tempfile
    os.chdir(tempfile.mkdtemp())
    sys.path.insert(0, ROOT)
    import oracle
    from oracle import tfqmr
    from angstromcube_b200 import workloads
    w = workloads.make("periodic4_1atom")
    r = oracle.RefGreen(w.geometry)
    r.set_potential(w.Vcell)
    r.set_atom_matrices(w.mats, w.offsets)
    r.set_energy(w.E, w.dVol)
    e = r.export()
    t = time.perf_counter()
    X, info = tfqmr.solve_blocks(r.action, e["subset"], e["colindx"], r.sizes["nnzb"], r.sizes["nCols"],
                                 tol=w.tolerance, maxiter=w.max_iterations)
    return info["iterations"], time.perf_counter() - t, bool(info["converged"])


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_available
    if not ref_available():
        emit({"impl": "reference", "unavailable": "reference CPU build oracle/_ref not built"})
        return
    import multiprocessing as mp
    import numpy as np
    from angstromcube_b200 import workloads
    w, pairs = workloads.batched_contour(WORKLOAD, nk=a.nk)
    nsrc = 8
    order = pair_order(len(pairs))
    nE = len(pairs) // a.nk
    # a step is one wave of the same pairs as our arm; a pair's solve = 8 sources x 2 actions x its
    # FP64 iteration count (measured at Gamma on the GPU, the table above) x the action time
    E_mid = pairs[order[0]][0]
    cpu_action_seconds(WORKLOAD, E_mid, procs=2)              # warm-up: page in, build plans
    vals, t_all = [], time.perf_counter()
    t1, cores = 0.0, 1
    for step in range(a.steps):
        t1, cores = cpu_action_seconds(WORKLOAD, pairs[order[(step * a.wave) % len(pairs)]][0])
        its = [FP64_ITERATIONS_GAMMA[order[(step * a.wave + i) % len(pairs)] // a.nk * 32 // nE]
               for i in range(a.wave)]
        seconds = sum(t1 * nsrc * 2 * n for n in its) / cores
        vals.append(a.wave / seconds)
    elapsed = time.perf_counter() - t_all
    value = sum(vals) / len(vals)
    # the CPU-runnable configuration solved for real on every core
    with mp.get_context("spawn").Pool(min(cores, 8)) as pool:
        sol = pool.map(_ref_small_cell_solve, range(min(cores, 8)))
    it0, s0, ok0 = sol[0]
    sample = ("reference action_t<double,2,1>::multiply (oracle/_ref CPU build, -O3 x86-64-v3) of the contour "
              "cell with one source cube per process, %d processes, %.2f s per action; a solve = 8 sources x 2 x "
              "FP64 tfQMR iterations of its energy (GPU-measured table), extrapolated" % (cores, t1))
    emit({
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * elapsed / max(a.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "batched contour: %s, %d energies x %d k-points, tolerance %g" % (
            WORKLOAD, nE, a.nk, TOLERANCE), "wave": a.wave},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "small_cell_cpu_solve": {"iterations": it0, "seconds": s0, "converged": ok0, "processes": len(sol),
                               "solves_per_s": len(sol) / max(s[1] for s in sol),
                               "what": "periodic 4^3-cube cell, one atom: reference CPU action inside the numpy "
                                       "tfQMR restatement, FP64 to 1e-9, one solve per process"},
    })


# ------------------------------------------------------------------ our arm

def time_part(lib_mod, plan, part, dtype_code, x, y, reps, stream):
    """Average duration of one part of the action, CUDA events on the launching stream."""
    import torch
    for _ in range(3):
        lib_mod.check(lib_mod.lib().a43g_action_part(plan.handle, part, lib_mod.ptr(y), lib_mod.ptr(x),
                                                     stream.cuda_stream, dtype_code), "a43g_action_part")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        lib_mod.check(lib_mod.lib().a43g_action_part(plan.handle, part, lib_mod.ptr(y), lib_mod.ptr(x),
                                                     stream.cuda_stream, dtype_code), "a43g_action_part")
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


def read_traffic(kernel):
    """DRAM bytes per block of a kernel from the committed ncu summary (profiles/traffic.txt: one
    line per kernel, name and bytes per block, measured on a smaller case and scaled by blocks)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return float(parts[1])
    except Exception:
        pass
    return None


def local_kernel_of(tune_lines):
    """Name of the FP32 local kernel the autotuner chose (from its "chosen: ..." line) and the key
    of its DRAM traffic in profiles/traffic.txt (None where no capture exists)."""
    chosen = " ".join(tune_lines)
    if "local pencils" in chosen:
        return "local_pencil_kernel (FP32 y-pencils: potential + 8th-order kinetic, one pass)", "local_pencil_kernel_f32"
    if "local plain rows" in chosen:
        return "local_fused_kernel<float,16> (potential + 8th-order kinetic, one pass)", None
    return "local_fused_pf_kernel<float,16> (potential + 8th-order kinetic, one pass)", "local_fused_pf_kernel_f32"


def check_one_plan(w, pairs):
    """Every truncation radius of the contour gives the same plan (the dense one): the plans of
    the smallest and the largest radius have identical arrays."""
    import copy
    import numpy as np
    from angstromcube_b200 import green_function as gf
    rs = [p[3] for p in pairs]
    exports = []
    for r in (min(rs), max(rs)):
        g = copy.copy(w.geometry)
        g.r_trunc = r
        exports.append(gf.construct_Green_function(g).export())
    a, b = exports
    return all(np.array_equal(a[k], b[k]) for k in a if k not in ("AtomMatrices", "phase"))


def our_arm(a):
    import numpy as np
    import torch
    import torch.distributed as dist
    from angstromcube_b200 import _lib, green_action, green_function as gf, workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", init_method="env://", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    hbm, bf16, peak_kind = peaks()
    w, pairs = workloads.batched_contour(WORKLOAD, nk=a.nk)
    one_plan = check_one_plan(w, pairs)
    g = w.geometry
    g.r_trunc = pairs[0][3]
    plan = gf.construct_Green_function(g)
    gf.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(plan, pairs[0][0], w.dVol)
    plan.upload()
    stream = torch.cuda.Stream()
    # schedule of the FP32 action chosen by timing, outside the timed region
    tune_report = green_action.autotune(plan, "float32", stream)
    opts = dict(tolerance=TOLERANCE, max_iterations=MAX_ITERATIONS, precision="float32", check_every=1,
                precondition=PRECONDITION)
    order = pair_order(len(pairs))
    nsteps_total = a.warmup + a.steps

    def wave_of(step):
        # rank r takes the waves r, r + world, ... of the walk (distinct pairs on every rank)
        base = (step * world + rank) * a.wave
        return [order[(base + i) % len(pairs)] for i in range(a.wave)]

    rho_all = torch.zeros((plan.nCols, 64, 2), dtype=torch.float64, device="cuda")

    def step(idx):
        sel = wave_of(idx)
        Es = [pairs[i][0] for i in sel]
        Ks = [pairs[i][1] for i in sel]
        stats, rho = green_action.solve_batched(plan, Es, Ks, w.dVol, want_rho=True, stream=stream,
                                                batch=a.wave, **opts)
        acc = sum(pairs[i][2] * rho[n] for n, i in enumerate(sel))
        rho_all.copy_(torch.from_numpy(np.stack([acc.real, acc.imag], axis=-1)))
        if world > 1:
            dist.all_reduce(rho_all)
        return sel, stats

    for i in range(a.warmup):
        step(i)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.lib().a43g_kernel_launches()
    records = []
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(a.warmup, nsteps_total):
            records.append(step(i))
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        wall = time.perf_counter() - t0
    launches = _lib.lib().a43g_kernel_launches() - launches0
    dev = e0.elapsed_time(e1) * 1e-3
    t = torch.tensor([max(dev, 1e-9)], dtype=torch.float64, device="cuda")
    conv = torch.tensor([sum(s["converged"] for _, st in records for s in st)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(conv)
    tmax = float(t.item())
    value = float(conv.item()) / tmax
    per_pair = []
    for sel, st in records:
        for i, s in zip(sel, st):
            E, k = pairs[i][0], pairs[i][1]
            per_pair.append({"pair": i, "E": [E.real, E.imag], "k": list(np.round(k, 4)),
                             "converged": bool(s["converged"]), "iterations": s["iterations"],
                             "fp64_sources": s["fp64_sources"], "replacements": s["refinements"],
                             "residual": s["residual_max"]})

    # end to end through the public API: host potential and matrices in (pinned), host energies and
    # k-points in, the pairs' densities out; one wave per step, timed on the host around synchronized work
    Vpin = torch.from_numpy(w.Vcell).pin_memory().numpy()
    Mpin = torch.from_numpy(w.mats).pin_memory().numpy()
    ke2e = 0 if a.no_e2e else a.steps              # the same pairs as the timed steps
    torch.cuda.synchronize()
    te = time.perf_counter()
    conv_e2e = 0
    for i in range(ke2e):
        gf.update_potential(plan, Vpin, Mpin, w.offsets, layout="cells")
        sel = wave_of(a.warmup + i)
        st_e, rho_e = green_action.solve_batched(plan, [pairs[j][0] for j in sel], [pairs[j][1] for j in sel],
                                                 w.dVol, want_rho=True, stream=stream, batch=a.wave, **opts)
        conv_e2e += sum(s["converged"] for s in st_e)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - te
    h2d = w.Vcell.nbytes + w.mats.nbytes + a.wave * 5 * 8
    d2h = a.wave * plan.nCols * 64 * 16

    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": 1e3 * tmax / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32 recurrences and operator, f64 solution and residual replacement",
               "data": "synthetic (seeded)",
               "config": {"workload": "batched contour: %s, 32 Gauss-Legendre energies on the semicircle "
                                      "-1..0 Ha x %d k-points, 8 source cubes, tolerance %g" % (WORKLOAD, a.nk, TOLERANCE),
                          "cell_cubes": [16, 16, 16], "sources": plan.nCols, "rhs_columns": plan.nCols * 64,
                          "atoms": w.natoms, "numax": 5, "nnzb_per_pair": plan.nnzb, "one_plan_for_all_radii": one_plan,
                          "wave": a.wave, "pairs_timed": len(per_pair), "max_iterations": MAX_ITERATIONS,
                          "preconditioner": "cube-diagonal local operator, from the right" if PRECONDITION else None,
                          "parallelism": "dp%d ((E, k) pairs per rank)" % world,
                          "l2": "inputs larger than L2 (%.2f GB per FP32 vector and pair)" % (plan.nnzb * 32768 / 1e9)},
               "solve": {"converged": int(conv.item()), "pairs": len(per_pair) * world, "wall_s_per_step": wall / a.steps,
                         "per_pair": per_pair},
               "e2e": None if 0 == ke2e else {"value": conv_e2e * world / e2e_s, "unit": "solves/s",
                                               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
               "gpu_launches": int(launches), "clocks": clocks.summary(),
               "autotune": [l for l in tune_report.splitlines() if l.startswith("chosen")]}
    return plan, w, pairs, stream, opts, out, hbm, bf16, peak_kind, world, rank, records


def measure_kernels(plan, stream, out, hbm, bf16, peak_kind):
    """Rooflines of the fused local kernel (HBM) and of the projector (TF32 tensor peak)."""
    import torch
    from angstromcube_b200 import _lib
    nnzb = plan.nnzb
    x = torch.randn((nnzb, 2, 64, 64), device="cuda", dtype=torch.float32)
    y = torch.empty_like(x)
    t_local = time_part(_lib, plan, 0, _lib.A43G_F32, x, y, 20, stream)
    bytes_local = 2 * nnzb * 8192 * 4 + plan.sizes["ncells"] * 64 * 4 + nnzb * (7 * 4) + plan.sizes["lists_nnz2"] * 4
    ach = bytes_local / t_local / 1e9
    kname, tkey = local_kernel_of(out.get("autotune", []))
    traffic = read_traffic(tkey) if tkey else None
    out["roofline"] = {"kernel": kname,
                       "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                       "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_local,
                       "ms_per_launch": t_local * 1e3,
                       "traffic": traffic * nnzb if traffic is not None else None}
    t_dyadic = time_part(_lib, plan, 1, _lib.A43G_F32, x, y, 10, stream)
    nsho = 56
    L = 5
    sf_flops = 2.0 * 2 * (64 * (L + 1) + 16 * (L + 1) * (L + 2) // 2 + 4 * nsho) * 128 * plan.sizes["SHOadd_nnz"]
    fma_peak = 148 * 128 * 2 * 1.965 / 1e3    # TFLOP/s: SMs x FP32 lanes x 2 flops x GHz
    flops = 4.0 * nsho * 64 * 128 * plan.sizes["SHOadd_nnz"]
    tf32_peak = bf16 / 2
    tc = os.environ.get("A43G_PROJECTOR", "") == "tc"
    out["roofline_projector"] = {"kernel": ("sho_project_tc + sho_add_tc (tcgen05 kind::tf32, 3xTF32)" if tc else
                                            "sho_project_simt + sho_add_simt (FP32 CUDA cores, sum-factorized)")
                                 + " + atom matrices",
                                 "bound": "tensor", "achieved": flops / t_dyadic / 1e12, "peak": tf32_peak,
                                 "unit": "TFLOP/s", "frac": flops / t_dyadic / 1e12 / tf32_peak,
                                 "peak_kind": "dense TF32 = half of the %s bf16 peak" % peak_kind,
                                 "algorithmic_flops_per_launch": flops, "ms_per_launch": t_dyadic * 1e3,
                                 "note": "flops of the dense contraction P (64 x 64 per block and image) x X (64 x 128)",
                                 # the kernels do the sum-factorized work: 64 (L+1) + 16 (L+1)(L+2)/2 + 4 nSHO
                                 # FMAs per column and (image, block) pair, for the projection and the addition
                                 "sum_factorized_flops_per_launch": sf_flops,
                                 "sum_factorized_tflops": sf_flops / t_dyadic / 1e12,
                                 "fp32_fma_peak_tflops": fma_peak,
                                 "fp32_fma_frac": sf_flops / t_dyadic / 1e12 / fma_peak}
    x64 = torch.randn((nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    y64 = torch.empty_like(x64)
    del x, y
    out["action_ms"] = {"fp32_local": t_local * 1e3, "fp32_projector": t_dyadic * 1e3,
                        "fp64_local": time_part(_lib, plan, 0, _lib.A43G_F64, x64, y64, 10, stream) * 1e3,
                        "fp64_projector": time_part(_lib, plan, 1, _lib.A43G_F64, x64, y64, 3, stream) * 1e3}
    del x64, y64
    torch.cuda.empty_cache()


def fp64_plain(plan, w, pairs, sel, stream, opts):
    """The plain FP64 solver on the given pairs one after the other: FP64 tfQMR without
    retirement (the reference's algorithm).  Returns per-pair (converged, iterations, seconds)."""
    from angstromcube_b200 import green_action, green_function as gf
    o64 = dict(opts)
    o64["precision"] = "float64"
    o64["precondition"] = False               # the reference's solver has no preconditioner
    res = []
    for i in sel:
        E, k = pairs[i][0], pairs[i][1]
        gf.update_energy_parameter(plan, E, w.dVol)
        gf.update_phases(plan, k)
        s, _ = green_action.solve(plan, stream=stream, want_rho=False, retire=False, **o64)
        res.append((bool(s["converged"]), s["iterations"], s["seconds"]))
    return res


def mixed_single(plan, w, pairs, sel, stream, opts):
    """The same pairs with the mixed solver, one pair per wave (a43g_solve_batched with batch 1)."""
    from angstromcube_b200 import green_action
    res = []
    for i in sel:
        st, _ = green_action.solve_batched(plan, [pairs[i][0]], [pairs[i][1]], w.dVol, stream=stream,
                                           batch=1, **opts)
        res.append((bool(st[0]["converged"]), st[0]["iterations"], st[0]["seconds"]))
    return res


def full_contour(a):
    """Every pair of the contour with the mixed batched solver (waves as large as memory allows)
    and with the plain FP64 solver; prints one JSON line per solver and a summary."""
    import numpy as np
    import torch
    from angstromcube_b200 import green_action, green_function as gf, workloads
    torch.cuda.set_device(0)
    w, pairs = workloads.batched_contour(WORKLOAD, nk=a.nk)
    g = w.geometry
    g.r_trunc = pairs[0][3]
    plan = gf.construct_Green_function(g)
    gf.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(plan, pairs[0][0], w.dVol)
    plan.upload()
    stream = torch.cuda.Stream()
    green_action.autotune(plan, "float32", stream)
    opts = dict(tolerance=TOLERANCE, max_iterations=MAX_ITERATIONS, precision="float32", check_every=1,
                precondition=PRECONDITION)
    Es = [p[0] for p in pairs]
    Ks = [p[1] for p in pairs]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st, rho = green_action.solve_batched(plan, Es, Ks, w.dVol, want_rho=True, stream=stream, batch=a.wave, **opts)
    e1.record(stream)
    torch.cuda.synchronize()
    t_mixed = e0.elapsed_time(e1) * 1e-3
    emit({"solver": "mixed+batched", "pairs": len(pairs), "wave": a.wave, "seconds": t_mixed,
          "converged": sum(s["converged"] for s in st),
          "per_pair": [[i, pairs[i][0].real, pairs[i][0].imag, s["converged"], s["iterations"], s["fp64_sources"],
                        s["residual_max"]] for i, s in enumerate(st)]})
    res64 = fp64_plain(plan, w, pairs, range(len(pairs)), stream, opts)
    t64 = sum(r[2] for r in res64)
    emit({"solver": "plain fp64", "pairs": len(pairs), "seconds": t64, "converged": sum(r[0] for r in res64),
          "per_pair": [[i, pairs[i][0].real, pairs[i][0].imag, r[0], r[1]] for i, r in enumerate(res64)]})
    cm, c64 = sum(s["converged"] for s in st), sum(r[0] for r in res64)
    emit({"summary": {"mixed_batched_solves_per_s": cm / t_mixed, "fp64_plain_solves_per_s": c64 / t64,
                      "speedup": (cm / t_mixed) / (c64 / t64) if c64 else None,
                      "seconds": [t_mixed, t64], "converged": [cm, c64], "pairs": len(pairs)}})


def convergence_scan(a):
    """Convergence of the plain FP64 solver on the one-source version of the contour cell: the
    iterations to 1e-8 at the 32 contour energies (Gamma, at most 1500 iterations), and the true
    relative residual at E = -0.2 + 0.02i (the energy of the cell's single-energy configuration)
    after 100, 200, ... 2000 iterations.  The solver is deterministic, so the solve capped at n
    iterations is the first n iterations of the uncapped one."""
    import numpy as np
    import torch
    from angstromcube_b200 import green_action, green_function as gf, workloads
    torch.cuda.set_device(0)
    w = workloads.make("periodic16_64atoms_s1x1x1")
    plan = gf.construct_Green_function(w.geometry)
    gf.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    stream = torch.cuda.Stream()
    E, _ = workloads.contour_semicircle(32)
    scan = []
    for e in E:
        gf.update_energy_parameter(plan, e, w.dVol)
        st, _ = green_action.solve(plan, stream=stream, want_rho=False, precision="float64", tolerance=1e-8,
                                   max_iterations=1500, check_every=1, retire=False)
        scan.append({"E": [e.real, e.imag], "iterations": st["iterations"], "converged": bool(st["converged"]),
                     "residual": st["residual_max"], "seconds": st["seconds"]})
        emit({"scan": scan[-1]})
    gf.update_energy_parameter(plan, complex(-0.2, 0.02), w.dVol)
    hist = []
    for n in range(100, 2001, 100):
        st, _ = green_action.solve(plan, stream=stream, want_rho=False, precision="float64", tolerance=1e-8,
                                   max_iterations=n, check_every=1, retire=False)
        hist.append({"iterations": st["iterations"], "residual": st["residual_max"],
                     "estimate": st["residual_estimate"]})
        emit({"history": hist[-1]})
    emit({"convergence_scan": {"cell": "periodic16_64atoms_s1x1x1", "tolerance": 1e-8, "scan": scan,
                               "history_E": [-0.2, 0.02], "history": hist}})


def profile_case(a):
    """The small case of the ncu captures: the one-source version of the benchmark cell at
    E = -0.2 + 0.02i (Gamma), above L2 per vector, a few launches of every kernel of the path."""
    import torch
    from angstromcube_b200 import _lib, green_action, green_function as gf, workloads
    torch.cuda.set_device(0)
    w = workloads.make("periodic16_64atoms_s1x1x1")
    stream = torch.cuda.Stream()

    def plan_for(projector):
        os.environ["A43G_PROJECTOR"] = projector
        p = gf.construct_Green_function(w.geometry)
        gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
        gf.update_energy_parameter(p, complex(-0.2, 0.02), w.dVol)
        return p

    if a.profile_case == "action":
        g = torch.Generator(device="cuda").manual_seed(5)
        for projector in ("simt", "tc"):
            p = plan_for(projector)
            x = torch.randn((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float32, generator=g)
            y = torch.empty_like(x)
            t0 = time_part(_lib, p, 0, _lib.A43G_F32, x, y, 4, stream)
            t1 = time_part(_lib, p, 1, _lib.A43G_F32, x, y, 4, stream)
            emit({"case": "action", "precision": "float32", "projector": projector, "local_ms": t0 * 1e3,
                  "projector_ms": t1 * 1e3})
        x = x.double()
        y = torch.empty_like(x)
        for name, env in (("pencils, addition unrolled", {}), ("rows, addition rolled",
                                                               {"A43G_LOCAL64": "rows", "A43G_ADD64": "rolled"})):
            for k in ("A43G_LOCAL64", "A43G_ADD64"):
                os.environ.pop(k, None)
            os.environ.update(env)
            p = plan_for("simt")
            t0 = time_part(_lib, p, 0, _lib.A43G_F64, x, y, 4, stream)
            t1 = time_part(_lib, p, 1, _lib.A43G_F64, x, y, 4, stream)
            emit({"case": "action", "precision": "float64", "kernels": name, "local_ms": t0 * 1e3,
                  "projector_ms": t1 * 1e3})
        for k in ("A43G_LOCAL64", "A43G_ADD64"):
            os.environ.pop(k, None)
    else:
        p = plan_for("simt")
        for precision in ("float32", "float64"):
            st, _ = green_action.solve(p, stream=stream, want_rho=False, precision=precision, tolerance=1e-8,
                                       max_iterations=40, check_every=10)
            emit({"case": "solve", "precision": precision, "iterations": st["iterations"],
                  "residual": st["residual_max"], "seconds": st["seconds"]})


def wrapped32(a):
    """Mixed precision on the large cell: the wrapped 32^3-cube cell (128^3 points, h = 0.25 Bohr)
    with 256 atoms on a jittered 8x8x4 lattice (numax 5, sigma 0.6), 32 source cubes (2048
    columns), truncation radius 12 Bohr, E = -0.2 + 0.02i (or --wrapped32-energy), tolerance
    1e-10.  First the plain FP64
    solve (no retirement, the reference's algorithm), whose solution is kept on the device, then
    the mixed solve traced against it: the relative error of G every 10 iterations (the
    residual-replacement gap) and at the end.  One FP64 block vector is 19.7 GB; the FP64 solve
    holds 8 of them and the FP64 solution of the mixed solve's continuation 8 plus the reference."""
    import torch
    from angstromcube_b200 import green_action, green_function as gf, workloads
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    w = workloads.make("wrapped32_256atoms")
    t1 = time.perf_counter()
    plan = gf.construct_Green_function(w.geometry)
    t2 = time.perf_counter()
    E = complex(a.wrapped32_energy)
    gf.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(plan, E, w.dVol)
    plan.upload()
    stream = torch.cuda.Stream()
    tune = green_action.autotune(plan, "float32", stream)
    out = {"cell": "wrapped32_256atoms", "nnzb": plan.nnzb, "columns": 64 * plan.nCols,
           "atoms": plan.sizes["nAtoms"], "atom_images": plan.sizes["nAtomImages"], "E": [E.real, E.imag],
           "tolerance": 1e-10, "max_iterations": a.wrapped32_iterations,
           "seconds_inputs": t1 - t0, "seconds_host_plan": t2 - t1, "autotune": tune.strip().splitlines()[-1:]}
    emit({"setup": out})
    Xref = torch.empty((plan.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    st, _ = green_action.solve(plan, X=Xref, stream=stream, want_rho=False, precision="float64", tolerance=1e-10,
                               max_iterations=a.wrapped32_iterations, check_every=10, retire=False)
    out["fp64"] = {k: st[k] for k in ("iterations", "converged", "residual_max", "residual_estimate", "seconds")}
    emit({"fp64": out["fp64"]})
    st3, _, tr = green_action.solve_traced(plan, Xref, every=10, stream=stream, precision="float32",
                                           tolerance=1e-10, max_iterations=a.wrapped32_iterations, check_every=10)
    out["mixed"] = {k: st3[k] for k in ("iterations", "converged", "residual_max", "residual_estimate", "seconds",
                                       "fp64_sources", "refinements")}
    out["mixed"]["error_of_G"] = [[int(r[0]), float(r[1]), int(r[2])] for r in tr]
    out["speedup_mixed_vs_fp64"] = st["seconds"] / max(st3["seconds"], 1e-12)
    emit({"wrapped32": out})


def launch_ranks(a):
    """--gpus N without a launcher: start N ranks with torch.distributed.run (one process per GPU,
    NCCL over 127.0.0.1) and return its exit code."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(a.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    a = parse()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(a))
    if a.impl == "reference":
        reference_arm(a)
        return
    if a.full_contour:
        full_contour(a)
        return
    if a.convergence_scan:
        convergence_scan(a)
        return
    if a.profile_case:
        profile_case(a)
        return
    if a.wrapped32:
        wrapped32(a)
        return
    plan, w, pairs, stream, opts, out, hbm, bf16, peak_kind, world, rank, records = our_arm(a)
    if rank == 0:
        measure_kernels(plan, stream, out, hbm, bf16, peak_kind)
        # plain FP64 on the first pairs of the timed sample, and the mixed solver on the same
        # pairs one at a time: the metric's comparison on matched solves
        sel = [i for s, _ in records for i in s][:max(1, a.fp64_pairs)]
        r64 = fp64_plain(plan, w, pairs, sel, stream, opts)
        if a.wave == 1:
            # the timed solves of these pairs (one pair per wave, device-timed by the solver)
            timed = {i: st for s_, sts in records for i, st in zip(s_, sts)}
            rmx = [(bool(timed[i]["converged"]), timed[i]["iterations"], timed[i]["seconds"]) for i in sel]
        else:
            rmx = mixed_single(plan, w, pairs, sel, stream, opts)
        t64, tmx = sum(r[2] for r in r64), sum(r[2] for r in rmx)
        c64, cmx = sum(r[0] for r in r64), sum(r[0] for r in rmx)
        out["fp64_plain"] = {"pairs": sel, "solves_per_s": c64 / t64, "seconds": t64, "converged": c64,
                             "iterations": [r[1] for r in r64],
                             "mixed_same_pairs": {"solves_per_s": cmx / tmx, "seconds": tmx, "converged": cmx,
                                                  "iterations": [r[1] for r in rmx]},
                             "speedup_mixed_vs_fp64": (cmx / tmx) / (c64 / t64) if c64 and cmx else None,
                             "what": "the same (E, k) pairs: plain FP64 tfQMR without retirement or preconditioner "
                                     "(the reference's algorithm), one pair at a time, against our solver (mixed "
                                     "precision, retirement%s) one pair per wave" % (
                                         ", cube-diagonal preconditioner" if PRECONDITION else "")}
        if world == 1 and not a.no_cpu:
            from oracle import ref_available
            if ref_available():
                t1, cores = cpu_action_seconds(WORKLOAD, pairs[sel[0]][0])
                its = [r[1] for r in r64]
                sec = sum(t1 * 8 * 2 * n for n in its) / cores
                out["cpu_baseline"] = {"value": len(its) / sec, "unit": "solves/s", "cores": cores, "kind": "reference",
                                       "sample": "reference CPU action (oracle/_ref) of the cell with one source cube "
                                                 "per process, %d processes, %.2f s per action; a solve = 8 sources x 2 x "
                                                 "the FP64 iteration count this run measured for the pair (%s), "
                                                 "extrapolated" % (cores, t1, its)}
        emit(out)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
