"""Benchmark of the Green-function solver: solves/s at 1e-8 relative residual.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one solve of the periodic 16^3-cube cell with 64 atoms (numax 5), 16 source cubes
(1024 right-hand-side columns), truncation radius 12 Bohr, to 1e-8 relative residual per
column, with the mixed-precision solver: FP32 tfQMR sweeps (FP32 finite-difference stencil,
potential and projectors) inside FP64 residual refinement.  The energy is E = -0.2 + 0.5i Ha,
the largest imaginary part of the energy contour over this cell: at E = -0.2 + 0.02i tfQMR
stagnates (4000 FP32 iterations leave a relative residual of 0.33, 700 FP64 iterations 0.07),
so no solver reaches 1e-8 there in a bounded time.  Each rank solves its own energy point
(weak scaling); the complex densities of all ranks are summed with one NCCL all-reduce per
step, as the energy-contour integration does.

Reported beside the solver throughput: the fused local-action kernel against the measured HBM
peak, the tensor-core projector, the plain FP64 solver on the same point, and the reference's
CPU action (oracle/_ref) timed on the host cores on a bounded sample and extrapolated to a
solve.  --impl reference prints the reference CPU arm only.
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

WORKLOAD = "periodic16_64atoms"
ENERGY = complex(-0.2, 0.5)
TOLERANCE = 1e-8
# tfQMR iterations of the plain FP64 solver at this workload, energy and tolerance (measured
# with this code on a B200); the reference arm, which runs without a GPU, extrapolates its
# action time to a solve with it.  The main arm uses the count of its own FP64 solve.
FP64_ITERATIONS = 240
METRIC = "Solves/s at 1e-8 resid (mixed+batched vs plain FP64); action % HBM peak"


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
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison solve")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
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


# ------------------------------------------------------------------ reference CPU leg

def _ref_worker(args):
    """One process: the reference's action_t<double,2,1>::multiply (its CPU build in
    oracle/_ref) on the benchmark cell with ONE source cube; returns seconds per action."""
    workload, seed, reps = args
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
    r.set_energy(ENERGY, w.dVol)
    x = np.random.default_rng(seed).standard_normal((r.sizes["nnzb"], 2, 64, 64))
    best = None
    for _ in range(reps):
        t = time.perf_counter()
        r.action(x)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return best


def cpu_reference_sample(workload, nsources, procs=None, reps=1, iterations=FP64_ITERATIONS):
    """Reference CPU action on a bounded sample: one single-source action per process, all host
    cores in parallel.  Returns (solves/s extrapolated, cores, seconds per single-source action)."""
    import multiprocessing as mp
    procs = procs or min(os.cpu_count() or 1, 32)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_worker, [(workload, i, reps) for i in range(procs)])
    t1 = max(times)
    # a solve applies the full operator (all sources) twice per iteration
    solves_per_s = procs / (t1 * nsources * 2 * iterations)
    return solves_per_s, procs, t1


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_available
    if not ref_available():
        emit({"impl": "reference", "unavailable": "reference CPU build oracle/_ref not built"})
        return
    nsrc = 16
    for _ in range(a.warmup):
        pass  # the warm-up of the CPU arm is the first (untimed) sample below
    cpu_reference_sample(a.workload, nsrc, procs=2)            # warm-up: page in, build plans
    vals, t_all = [], time.perf_counter()
    for _ in range(a.steps):
        v, cores, t1 = cpu_reference_sample(a.workload, nsrc)
        vals.append(v)
    elapsed = time.perf_counter() - t_all
    value = sum(vals) / len(vals)
    sample = ("reference action_t<double,2,1>::multiply (oracle/_ref CPU build) of the %s cell with one source "
              "cube per process, %d processes, %.2f s per action; solve = 16 sources x 2 x %d FP64 tfQMR "
              "iterations (extrapolated)" % (a.workload, cores, t1, FP64_ITERATIONS))
    emit({
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * elapsed / max(a.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": a.workload, "tolerance": TOLERANCE, "sources": nsrc, "E": [ENERGY.real, ENERGY.imag]},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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
        dist.init_process_group("nccl", init_method="env://", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    hbm, bf16, peak_kind = peaks()
    w = workloads.make(a.workload)
    # every rank solves its own energy point of the contour (weak scaling)
    E = complex(ENERGY.real - 0.01*rank, ENERGY.imag)
    plan = gf.construct_Green_function(w.geometry)
    gf.update_potential(plan, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(plan, E, w.dVol)
    plan.upload()
    stream = torch.cuda.Stream()
    # schedule of the FP32 action chosen by timing, outside the timed region
    tune_report = green_action.autotune(plan, "float32", stream)
    # convergence read back after every iteration: a check costs one host round trip (tens of us)
    # against about 23 ms per FP32 iteration, and ends each sweep on the iteration it converges
    # inner tolerance 1e-4 (the library default): sweeps then end near the FP32 floor (about 1e-3
    # of their right-hand side) by convergence or by the short stall rule; a tighter one leaves
    # columns above the stall level, where they wait four times as long (measured: 430-450
    # iterations at 1e-4, 480-630 at 1e-5)
    opts = dict(tolerance=TOLERANCE, max_iterations=3000, precision="float32", inner_tolerance=1e-4,
                max_refinements=8, check_every=1)
    rho_all = torch.zeros((plan.nCols, 64, 2), dtype=torch.float64, device="cuda")

    def step():
        stats, rho = green_action.solve(plan, stream=stream, **opts)
        if world > 1:
            rho_all.copy_(torch.from_numpy(np.stack([rho.real, rho.imag], axis=-1)))
            dist.all_reduce(rho_all)
        return stats

    for _ in range(a.warmup):
        st = step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.lib().a43g_kernel_launches()
    stats = []
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            stats.append(step())
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        wall = time.perf_counter() - t0
    launches = _lib.lib().a43g_kernel_launches() - launches0
    # device-side time of the steps: the solver records its own events per solve
    dev = sum(s["seconds"] for s in stats)
    t = torch.tensor([max(dev, 1e-9)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tmax = float(t.item())
    value = world*a.steps/tmax
    converged = all(s["converged"] for s in stats)
    iters = [s["iterations"] for s in stats]
    refs = [s["refinements"] for s in stats]
    res = max(s["residual_max"] for s in stats)

    # end to end through the public API: host potential, matrices and energy in, density out
    Vpin = torch.from_numpy(w.Vcell).pin_memory().numpy()
    Mpin = torch.from_numpy(w.mats).pin_memory().numpy()
    ke2e = 0 if a.no_e2e else max(1, a.steps//2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke2e):
        gf.update_potential(plan, Vpin, Mpin, w.offsets, layout="cells")
        gf.update_energy_parameter(plan, E, w.dVol)
        s_e2e, rho = green_action.solve(plan, stream=stream, **opts)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0)/max(ke2e, 1)
    h2d = w.Vcell.nbytes + w.mats.nbytes
    d2h = plan.nCols*64*16

    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": 1e3*tmax/a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32+3xtf32 (fp64 refinement)", "data": "synthetic (seeded)",
               "config": {"workload": a.workload, "cell_cubes": list(np.array(w.geometry.ng)//4),
                          "sources": plan.nCols, "rhs_columns": plan.nCols*64, "atoms": w.natoms, "numax": 5,
                          "nnzb": plan.nnzb, "tolerance": TOLERANCE, "E": [E.real, E.imag],
                          "parallelism": "dp%d (energy points)" % world,
                          "l2": "inputs larger than L2 (%.1f GB per FP32 vector)" % (plan.nnzb*32768/1e9)},
               "solve": {"iterations": iters, "refinements": refs, "residual_max": res, "converged": converged,
                         "wall_s_per_step": wall/a.steps},
               "e2e": None if 0 == ke2e else {"value": 1.0/e2e_s*world, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h)},
               "gpu_launches": int(launches), "clocks": clocks.summary(),
               "autotune": [l for l in tune_report.splitlines() if l.startswith("chosen")]}
    return plan, w, E, stream, opts, out, hbm, bf16, peak_kind, world, rank


def measure_kernels(a, plan, w, stream, out, hbm, bf16, peak_kind):
    """Rooflines of the fused local kernel (HBM) and of the tensor-core projector (TF32)."""
    import torch
    from angstromcube_b200 import _lib
    nnzb = plan.nnzb
    x = torch.randn((nnzb, 2, 64, 64), device="cuda", dtype=torch.float32)
    y = torch.empty_like(x)
    t_local = time_part(_lib, plan, 0, _lib.A43G_F32, x, y, 20, stream)
    bytes_local = 2*nnzb*8192*4 + plan.sizes["ncells"]*64*4 + nnzb*(7*4) + plan.sizes["lists_nnz2"]*4
    ach = bytes_local/t_local/1e9
    kname, tkey = local_kernel_of(out.get("autotune", []))
    traffic = read_traffic(tkey) if tkey else None
    out["roofline"] = {"kernel": kname,
                       "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach/hbm,
                       "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_local,
                       "ms_per_launch": t_local*1e3,
                       "traffic": traffic*nnzb if traffic is not None else None}
    t_dyadic = time_part(_lib, plan, 1, _lib.A43G_F32, x, y, 10, stream)
    nsho = 56
    flops = 4.0*nsho*64*128*plan.sizes["SHOadd_nnz"]
    tf32_peak = bf16/2
    tc = os.environ.get("A43G_PROJECTOR", "") == "tc"
    out["roofline_projector"] = {"kernel": ("sho_project_tc + sho_add_tc (tcgen05 kind::tf32, 3xTF32)" if tc else
                                            "sho_project_kernel + sho_add_kernel (SIMT FP32, sum-factorized)")
                                 + " + atom matrices",
                                 "bound": "tensor", "achieved": flops/t_dyadic/1e12, "peak": tf32_peak,
                                 "unit": "TFLOP/s", "frac": flops/t_dyadic/1e12/tf32_peak,
                                 "peak_kind": "dense TF32 = half of the %s bf16 peak" % peak_kind,
                                 "algorithmic_flops_per_launch": flops, "ms_per_launch": t_dyadic*1e3,
                                 "note": "flops of the dense contraction P (64 x 64 per block and image) x X (64 x 128)"}
    x64 = torch.randn((nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    y64 = torch.empty_like(x64)
    del x, y
    out["action_ms"] = {"fp32_local": t_local*1e3, "fp32_projector": t_dyadic*1e3,
                        "fp64_local": time_part(_lib, plan, 0, _lib.A43G_F64, x64, y64, 10, stream)*1e3,
                        "fp64_projector": time_part(_lib, plan, 1, _lib.A43G_F64, x64, y64, 3, stream)*1e3}
    del x64, y64
    torch.cuda.empty_cache()


def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
        return
    plan, w, E, stream, opts, out, hbm, bf16, peak_kind, world, rank = our_arm(a)
    if rank == 0:
        measure_kernels(a, plan, w, stream, out, hbm, bf16, peak_kind)
        if not a.no_fp64:
            from angstromcube_b200 import green_action
            o64 = dict(opts); o64["precision"] = "float64"
            s64, _ = green_action.solve(plan, stream=stream, want_rho=False, **o64)
            out["fp64_plain"] = {"solves_per_s": 1.0/s64["seconds"], "iterations": s64["iterations"],
                                 "residual_max": s64["residual_max"], "converged": s64["converged"],
                                 "speedup_mixed_vs_fp64": out["value"]/world*s64["seconds"]}
        if world == 1 and not a.no_cpu:
            from oracle import ref_available
            if ref_available():
                nit = out.get("fp64_plain", {}).get("iterations", FP64_ITERATIONS)
                v, cores, t1 = cpu_reference_sample(a.workload, plan.nCols, iterations=nit)
                out["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                                       "sample": "reference CPU action (oracle/_ref) of the cell with one source cube "
                                                 "per process, %d processes, %.2f s per action; solve = %d sources x 2 x "
                                                 "%d FP64 tfQMR iterations (extrapolated)"
                                                 % (cores, t1, plan.nCols, nit)}
        emit(out)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
