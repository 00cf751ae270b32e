"""Benchmark of the B200 pressure-correction CG.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (N=1): the 60x120x84 production mesh (604,800 cells, 24 scrap
spheres, density contrast 7800:0.3) driven through SIMPLE-like warm-started
re-solves: re-solve s perturbs abar_P by a fresh per-cell U[0.9, 1.1], draws
a fresh zero-mean RHS and starts from the previous solution; plain FP64 CG
to relative residual 1e-8. One step = one re-solve. Each rank runs its own
furnace (seed = rank) with no data-path collective: weak scaling.

value : cell-iterations/s with every system already resident in HBM
        (device-pointer C-ABI call: pack + solve + unpack), device time from
        CUDA events on the solver's stream, L2 flushed between steps.
e2e   : the same chain through the host-pointer C-ABI call (the Fortran
        drop-in), pinned host buffers, uploads and the phi download inside
        each timed step.
The reference arm (--impl reference) times the oracle port of the
reference CG (no Fortran toolchain exists to build the reference itself) on
all host cores over a bounded sample of the same workload.

Further lines (--workload; one JSON line each, not the headline):
  fine      120x240x168 FP64 cold solves to 1e-10 and the mixed form
  batch     96 uneven systems in one persistent launch vs one by one
  serve     Poisson streams of furnace runs through the serving loop
  tdma      line-by-line TDMA sweeps of a transport system
  pcorr     the post-CG corrections of the pressure step
  assemble  the assembly of the pressure-correction equation
  pstep     one whole pressure step: assembly, CG, corrections
  fixed     a fixed amount of work for profiling and per-iteration timing:
            --repeat solves of exactly --iters CG iterations on --mesh
            (tol 0; --launch, --cluster and --kernel pick the form), or
            --batch-size systems of the batch mix, or --tdma-sweeps sweeps
            with --fixed-tdma
--cg-form selects the FP64 CG's recurrences (reference: two all-reduces per
iteration, the default; one-reduction: the Chronopoulos-Gear form).
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "hornofusion-full3d_b200"

METRIC = ("pressure-CG cell-iters/s + HBM GB/s (60x120x84); "
          "serve p99 latency @1e-8 resid")
MESH = (60, 120, 84, 24)
TOL = 1e-8
MAX_ITER = 200000
BYTES_PER_CELL_ITER = 120          # algorithmic FP64 bytes per cell-iteration
L2_FLUSH_BYTES = 256 << 20
DATA = ("synthetic: seeded eafgen systems (uniform cylindrical mesh, steel "
        "bath + gas + scrap spheres, log-uniform abar_P), no dataset")


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def solver_kernel_name(solver, plan):
    """Name of the persistent kernel the last solve of `solver` ran."""
    if len(plan) > 2:
        return "cg_dsm_kernel" if plan[0] == plan[2] else "cg_cluster_kernel"
    return {solver.KERNEL_LOADS: "cg_f64_kernel", solver.KERNEL_STREAM: "cg_stream_kernel",
            solver.KERNEL_SLOTS: "cg_cluster_kernel",
            solver.KERNEL_KEEP: "cg_keep_kernel"}[solver.last_kernel()]


def traffic_profile(kernel):
    return os.path.join("profiles", f"{kernel}_60x120x84.txt")


def ncu_traffic_per_launch(kernel):
    """DRAM bytes of one solver launch of this workload (a warm-started
    re-solve), from the committed ncu summary of that kernel, or None when
    no capture has been summarised yet. The working set stays in L2 for the
    whole solve, so a launch's traffic is its first read of the system plus
    the final write and does not grow with its iterations; it is reported
    as captured."""
    path = os.path.join(ROOT, traffic_profile(kernel))
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch"):
            try:
                return float(line.split("=")[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_sequence(g, n_steps, seed):
    nr, nth, nz, nsph = MESH
    mesh = g.make_mesh(nr, nth, nz, nsph, seed)
    return [g.make_system(nr, nth, nz, nsph, seed, resolve=s, mesh=mesh)
            for s in range(n_steps)]


def cpu_baseline_sample(g, seed, budget_s=12.0):
    """Oracle (port of the reference CG) on all host cores, bounded sample."""
    import oracle
    nr, nth, nz, nsph = MESH
    s = g.make_system(nr, nth, nz, nsph, seed, resolve=0)
    threads = max(1, oracle.max_threads())
    phi = g.zeros_phi(nr, nth, nz)
    # calibrate on 50 iterations, then size the sample to ~budget_s
    t0 = time.perf_counter()
    oracle.cg(s, phi, 50, 0.0, nthreads=threads)
    dt = time.perf_counter() - t0
    iters = int(max(50, min(20000, 50 * budget_s / max(dt, 1e-6))))
    phi = g.zeros_phi(nr, nth, nz)
    t0 = time.perf_counter()
    _, nit = oracle.cg(s, phi, iters, 0.0, nthreads=threads)
    dt = time.perf_counter() - t0
    return {"value": nr * nth * nz * nit / dt, "unit": "cell-iters/s",
            "cores": threads, "kind": "port",
            "sample": (f"oracle port of cg_3d_mpi, {nr}x{nth}x{nz} re-solve 0, "
                       f"{nit} iterations (tol 0) on {threads} OpenMP threads, "
                       f"{dt:.1f} s"),
            "seconds": dt}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz, nsph = MESH
    n = nr * nth * nz
    threads = max(1, oracle.max_threads())
    steps = make_sequence(g, min(args.warmup + args.steps, 4), seed=0)
    cap = args.ref_iters
    phi = g.zeros_phi(nr, nth, nz)
    for w in range(args.warmup):
        oracle.cg(steps[w % len(steps)], phi, min(cap, 50), TOL, nthreads=threads)
    total_ci, total_s = 0, 0.0
    for k in range(args.steps):
        s = steps[k % len(steps)]
        t0 = time.perf_counter()
        _, nit = oracle.cg(s, phi, cap, TOL, nthreads=threads)
        total_s += time.perf_counter() - t0
        total_ci += n * nit
    value = total_ci / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "cell-iters/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": DATA,
        "config": {"workload": "pressure-CG 60x120x84 FP64 warm-started re-solves",
                   "mesh": [nr, nth, nz], "cells": n, "tol": TOL,
                   "iteration_cap_per_step": cap},
        "cpu_baseline": {"value": value, "unit": "cell-iters/s", "cores": threads,
                         "kind": "port",
                         "sample": (f"each step: one warm-started re-solve capped at "
                                    f"{cap} iterations, oracle port of cg_3d_mpi on "
                                    f"{threads} OpenMP threads (the Fortran reference "
                                    "has no compiler here)")},
        "e2e": {"value": value, "unit": "cell-iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = local_rank
    torch.cuda.set_device(dev)
    nr, nth, nz, nsph = MESH
    n = nr * nth * nz
    n_total = args.warmup + args.steps
    seq = make_sequence(g, n_total, seed=rank)
    # device-resident copies of every re-solve's inputs (value leg)
    dev_sys = [[torch.from_numpy(a).to(f"cuda:{dev}") for a in s.arrays()]
               for s in seq]
    phi_d = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64,
                        device=f"cuda:{dev}")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{dev}")
    torch.cuda.synchronize()
    solver = eaf.CGSolver(nr, nth, nz, device=dev)
    solver.set_form(CG_FORMS[args.cg_form])
    if args.cluster is not None:
        solver.set_cluster(args.cluster)

    def one(k, resident=True, host_arrays=None, phi_h=None):
        if resident:
            res, nit, st = solver.solve(dev_sys[k], phi_d, MAX_ITER, TOL,
                                        device_ptrs=True)
        else:
            res, nit, st = solver.solve(host_arrays, phi_h, MAX_ITER, TOL)
        if st != 0 or not res < TOL:
            raise RuntimeError(f"solve {k} did not converge: status {st} res {res}")
        return nit, solver.last_timing()

    for w in range(args.warmup):
        one(w)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    solve_ms = kern_ms = 0.0
    iters = []
    for k in range(args.warmup, n_total):
        flush.zero_()
        torch.cuda.synchronize()
        nit, t = one(k)
        iters.append(nit)
        solve_ms += t["solve_ms"]
        kern_ms += t["kernel_ms"]
    torch.cuda.synchronize()
    clk = clocks.stop()
    plan = solver.last_launch()
    kernel = solver_kernel_name(solver, plan)
    if dist is not None:
        dist.barrier()

    # e2e leg: host arrays (pinned), uploads + download inside each step
    host_sys = []
    for s in seq:
        hs = []
        for a in s.arrays():
            h = eaf.host_empty(a.shape)
            h[...] = a
            hs.append(h)
        host_sys.append(hs)
    phi_h = eaf.host_empty(g.halo_shape(nr, nth, nz))
    phi_h[...] = 0.0
    for w in range(args.warmup):
        one(w, False, host_sys[w], phi_h)
    e2e_ms = 0.0
    e2e_ci = 0
    for k in range(args.warmup, n_total):
        flush.zero_()
        torch.cuda.synchronize()
        nit, t = one(k, False, host_sys[k], phi_h)
        e2e_ms += t["e2e_ms"]
        e2e_ci += n * nit
    halo_bytes = 8 * (nr + 4) * (nth + 4) * (nz + 4)

    cell_iters = n * sum(iters)
    stats = torch.tensor([solve_ms, kern_ms, e2e_ms, float(cell_iters),
                          float(e2e_ci)], dtype=torch.float64, device=f"cuda:{dev}")
    if dist is not None:
        mx = stats.clone()
        sm = stats.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        solve_ms, kern_ms, e2e_ms = (float(v) for v in mx[:3])
        cell_iters, e2e_ci = float(sm[3]), float(sm[4])
    if rank != 0:
        solver.close()
        return 0

    value = cell_iters / (solve_ms / 1e3)
    per_rank_ci = n * sum(iters)
    achieved = BYTES_PER_CELL_ITER * per_rank_ci / (kern_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic_per_launch(kernel)
    cpu = cpu_baseline_sample(g, seed=0) if world == 1 else None
    line = {
        "metric": METRIC, "value": value, "unit": "cell-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": solve_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": {"workload": "pressure-CG 60x120x84 FP64 warm-started re-solves",
                   "mesh": [nr, nth, nz], "cells": n, "spheres": nsph, "tol": TOL,
                   "iterations_per_solve": iters,
                   "launch": {"grid": plan[0], "block": plan[1],
                              "cluster": plan[2] if len(plan) > 2 else 1},
                   "cg_form": args.cg_form,
                   "l2": "flushed between steps (256 MiB memset); within a solve "
                         "the ~39 MB symmetric working set is L2-resident",
                   "parallelism": f"replicas x{world} (one furnace per GPU)"},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read+write of one bench "
                                       f"launch ({traffic_profile(kernel)})",
                     "kernel": kernel + " (persistent, one launch per solve)",
                     "algorithmic_bytes_per_cell_iter": BYTES_PER_CELL_ITER},
        "cpu_baseline": ({k: v for k, v in cpu.items() if k != "seconds"}
                         if cpu else None),
        "e2e": {"value": e2e_ci / (e2e_ms / 1e3), "unit": "cell-iters/s",
                "h2d_bytes_per_step": 9 * halo_bytes,
                "d2h_bytes_per_step": halo_bytes + 40},
        # pack, solver, unpack; the flat kernels' launcher also fills the
        # p.q slot sets with the empty-slot marker (one small kernel)
        "gpu_launches": (4 if kernel in ("cg_keep_kernel", "cg_f64_kernel")
                         and 1 < plan[0] <= 160 else 3) * args.steps,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    solver.close()
    return 0


# ---------------------------------------------------------------------------
# Further named workloads (one JSON line each; not the driver's headline)
# ---------------------------------------------------------------------------
def _base_line(metric, value, unit, steps, warmup, ms_per_step, workload, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1,
            "steps": steps, "warmup": warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": DATA, "config": {"workload": workload}}
    line["config"].update(extra)
    return line


def run_fine(args):
    """120x240x168, 64 spheres: FP64 plain solves (HBM-bound roofline case)
    and the mixed FP32/FP64 form on the same system, with its error against
    the FP64 solution."""
    import numpy as np
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz, nsph = g.FINE
    n = nr * nth * nz
    s = g.make_system(nr, nth, nz, nsph, seed=0)
    dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
    phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
    with eaf.CGSolver(nr, nth, nz) as cg:
        cg.set_form(CG_FORMS[args.cg_form])
        for _ in range(args.warmup):           # warm-ups capped at 300 iterations
            phi.zero_()
            cg.solve(dev, phi, 300, 0.0, device_ptrs=True)
        ms, kms, its = 0.0, 0.0, []
        for _ in range(args.steps):
            phi.zero_()
            torch.cuda.synchronize()
            res, nit, st = cg.solve(dev, phi, MAX_ITER, 1e-10, device_ptrs=True)
            t = cg.last_timing()
            ms += t["solve_ms"]
            kms += t["kernel_ms"]
            its.append(nit)
        x64 = phi.cpu().numpy()
        launch = cg.last_launch()
        phim = torch.zeros_like(phi)
        rm, nm, no, stm = cg.solve_mixed(dev, phim, tol=1e-10, inner_tol=0.1,
                                         max_outer=args.mixed_outer,
                                         max_inner=args.mixed_inner, device_ptrs=True)
        tm = cg.last_timing()
        trace = cg.mixed_trace(args.mixed_outer)
        xm = phim.cpu().numpy()
    I = g.interior
    err = float(np.linalg.norm(I(xm) - I(x64)) / np.linalg.norm(I(x64)))
    ci = n * sum(its)
    value = ci / (ms / 1e3)
    achieved = BYTES_PER_CELL_ITER * ci / (kms / 1e3) / 1e9
    peak, kind = measured_peaks()
    line = _base_line("pressure-CG cell-iters/s (120x240x168, FP64, tol 1e-10)", value,
                      "cell-iters/s", args.steps, args.warmup, ms / args.steps,
                      "pressure-CG 120x240x168 FP64 cold solves",
                      {"mesh": [nr, nth, nz], "cells": n, "tol": 1e-10,
                       "iterations_per_solve": its, "cg_form": args.cg_form,
                       "launch": {"grid": launch[0], "block": launch[1]}})
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                        "kernel": "cg_f64_kernel"}
    line["mixed"] = {"residual": rm, "status": stm, "inner_iterations": nm,
                     "outer_steps": no, "kernel_ms": tm["kernel_ms"],
                     "caps": {"max_outer": args.mixed_outer, "max_inner": args.mixed_inner},
                     "rel_l2_error_vs_fp64": err,
                     "fp64_kernel_ms_per_solve": kms / args.steps,
                     "trace": trace}
    print(json.dumps(line), flush=True)
    return 0


def run_tdma(args):
    """Line-by-line TDMA (tdma_3d_mpi) on a 60x120x84 transport system:
    args.tdma_sweeps sweeps per step from phi = 0, device-resident inputs
    (value) and through the host-pointer entry (e2e: 9 uploads + 1 download
    per step), with the single-thread CPU restatement as baseline (the
    reference's serial sweeps are one sequential loop nest)."""
    import numpy as np
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz = MESH[:3]
    n = nr * nth * nz
    ns = args.tdma_sweeps
    s = g.make_transport_system(nr, nth, nz, seed=0)
    dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
    phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    host = [eaf.host_empty(g.halo_shape(nr, nth, nz)) for _ in range(9)]
    for h, a in zip(host, s.arrays()):
        h[...] = a
    with eaf.CGSolver(nr, nth, nz) as cg:
        for _ in range(args.warmup):
            phi.zero_()
            cg.tdma(dev, phi, ns, device_ptrs=True)
        ms = kms = 0.0
        for _ in range(args.steps):
            phi.zero_()
            flush.fill_(1)
            torch.cuda.synchronize()
            cg.tdma(dev, phi, ns, device_ptrs=True)
            t = cg.last_timing()
            ms += t["solve_ms"]
            kms += t["kernel_ms"]
        e2e = 0.0
        for _ in range(args.steps):
            host[8][...] = 0.0
            cg.tdma(host[:8], host[8], ns)
            e2e += cg.last_timing()["e2e_ms"]
        x_gpu = host[8].copy()
        launch = cg.last_launch()
    # CPU baseline: the oracle's serial sweeps on one thread, same system.
    import oracle
    x_cpu = g.zeros_phi(nr, nth, nz)
    t0 = time.perf_counter()
    oracle.tdma_3d(s, x_cpu, ns)
    cpu_s = time.perf_counter() - t0
    crit = sum((A + B - 1) * L for A, B, L in ((nth, nz, nr), (nr, nz, nth), (nth, nr, nz)))
    value = n * ns * args.steps / (ms / 1e3)
    line = _base_line("line-TDMA cell-sweeps/s (60x120x84 transport system)", value,
                      "cell-sweeps/s", args.steps, args.warmup, ms / args.steps,
                      f"tdma_3d_mpi, {ns} sweeps from phi = 0",
                      {"mesh": [nr, nth, nz], "cells": n, "sweeps_per_step": ns,
                       "launch": {"grid": launch[0], "block": launch[1]},
                       "l2": "flushed between steps (256 MiB memset)"})
    line["e2e"] = {"value": n * ns * args.steps / (e2e / 1e3), "unit": "cell-sweeps/s",
                   "h2d_bytes_per_step": 9 * host[0].nbytes,
                   "d2h_bytes_per_step": host[0].nbytes}
    line["bitwise_equal_to_cpu"] = bool(np.array_equal(x_gpu, x_cpu))
    line["cpu_baseline"] = {"value": n * ns / cpu_s, "unit": "cell-sweeps/s", "cores": 1,
                            "kind": "port",
                            "sample": f"oracle port of tdma_3d_mpi, {ns} sweeps, one "
                                      f"thread, {cpu_s:.2f} s"}
    line["critical_path"] = {
        "elements_per_sweep": crit,
        "ns_per_element": 1e6 * (kms / args.steps) / ns / crit,
        "note": "lines of one direction run as a wavefront: (A+B-1) dependent line "
                "solves of L elements each, one sequential Thomas step per element"}
    line["gpu_launches"] = 2 * args.steps
    print(json.dumps(line), flush=True)
    return 0


def _pinned_fields(eaf, f):
    """A copy of an eafgen fields object whose arrays live in pinned host
    memory (the e2e legs upload from page-locked buffers, as a caller that
    registers its workspace does)."""
    import numpy as np
    c = f.copy()
    for k, v in list(c.__dict__.items()):
        if isinstance(v, np.ndarray):
            h = eaf.host_empty(v.shape, v.dtype)
            h[...] = v
            setattr(c, k, h)
    return c


def _refill(dst, src) -> None:
    import numpy as np
    for k, v in src.__dict__.items():
        if isinstance(v, np.ndarray):
            getattr(dst, k)[...] = v


# eaf_cg_set_form values
CG_FORMS = {"reference": 0, "one-reduction": 1}
DEFAULT_CG_FORM = "reference"

PCORR_BYTES_PER_CELL = 300  # reads 23 doubles + 6 ints, writes 10 doubles (update + sealed pass)


def run_pcorr(args):
    """Post-CG corrections of the pressure step (solve_pressure_correction
    after the CG) on the 60x120x84 mesh, liquid and gas phases, with the
    fields resident on the device (value, HBM roofline) and through the
    host-pointer entry (e2e); the single-thread CPU restatement as baseline."""
    import numpy as np
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz = MESH[:3]
    n = nr * nth * nz
    f0 = g.make_pcorr_fields(nr, nth, nz, seed=0)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def to_dev(f):
        d = f.copy()
        for k, v in list(d.__dict__.items()):
            if isinstance(v, np.ndarray):
                setattr(d, k, torch.from_numpy(v).cuda())
        return d

    with eaf.CGSolver(nr, nth, nz) as cg:
        d = to_dev(f0)
        for _ in range(args.warmup):
            cg.pressure_correct(d, device_ptrs=True)
        kms = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            cg.pressure_correct(d, device_ptrs=True)
            kms += cg.last_timing()["kernel_ms"]
        host = f0.copy()
        e2e = 0.0
        h = _pinned_fields(eaf, f0)
        for _ in range(args.steps):
            _refill(h, f0)
            cg.pressure_correct(h)
            e2e += cg.last_timing()["e2e_ms"]
        cg.pressure_correct(host)
    import oracle
    ref = f0.copy()
    t0 = time.perf_counter()
    oracle.pressure_correct(ref)
    cpu_s = time.perf_counter() - t0
    same = all(np.array_equal(a, ref.outputs()[k]) for k, a in host.outputs().items())
    value = n * args.steps / (kms / 1e3)
    achieved = PCORR_BYTES_PER_CELL * n * args.steps / (kms / 1e3) / 1e9
    peak, kind = measured_peaks()
    nh = (nr + 4) * (nth + 4) * (nz + 4)
    line = _base_line("post-CG pressure corrections, cells/s (60x120x84, two phases)", value,
                      "cells/s", args.steps, args.warmup, kms / args.steps,
                      "flux export + velocity/pressure corrections + sealed cells",
                      {"mesh": [nr, nth, nz], "cells": n, "phases": 2,
                       "l2": "flushed between steps (256 MiB memset)"})
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                        "algorithmic_bytes_per_cell": PCORR_BYTES_PER_CELL,
                        "kernel": "pcorr_update_kernel + pcorr_sealed_kernel + pcorr_wrap_kernel"}
    line["e2e"] = {"value": n * args.steps / (e2e / 1e3), "unit": "cells/s",
                   "h2d_bytes_per_step": 26 * 8 * nh + 6 * 4 * nh,
                   "d2h_bytes_per_step": 10 * 8 * nh + 3 * 4 * nh}
    line["bitwise_equal_to_cpu"] = bool(same)
    line["cpu_baseline"] = {"value": n / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
                            "sample": f"oracle port, one call, one thread, {cpu_s:.3f} s"}
    line["gpu_launches"] = 3 * args.steps
    print(json.dumps(line), flush=True)
    return 0


# flags 7 (liquid room, gas in the equation, gas compressibility): reads 24
# doubles (vol, Ar, Ath, Az, p, liq_room, 8 + 8 phase arrays, liq_T, gas
# T_old) and 4 ints (cell type, outlet, activity masks), writes 18 doubles
# (coefficients, Su, pp, Fs/ac/Fc) and 3 ints (link flags), each once per
# halo-layout element.
ASSEMBLY_BYTES_PER_ELEM = 24 * 8 + 4 * 4 + 18 * 8 + 3 * 4


def run_assemble(args):
    """Assembly of the pressure-correction equation (solve_pressure_correction
    up to the CG) on the 60x120x84 mesh with both phases and every switch on,
    fields resident on the device (value, HBM roofline) and through the
    host-pointer entry (e2e); the single-thread CPU restatement as baseline."""
    import numpy as np
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz = MESH[:3]
    n = nr * nth * nz
    nh = (nr + 4) * (nth + 4) * (nz + 4)
    f0 = g.make_assembly_fields(nr, nth, nz, seed=0, flags=7)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def to_dev(f):
        d = f.copy()
        for k, v in list(d.__dict__.items()):
            if isinstance(v, np.ndarray):
                setattr(d, k, torch.from_numpy(v).cuda())
        return d

    with eaf.CGSolver(nr, nth, nz) as cg:
        d = to_dev(f0)
        for _ in range(args.warmup):
            cg.pressure_assemble(d, device_ptrs=True)
        kms = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            cg.pressure_assemble(d, device_ptrs=True)
            kms += cg.last_timing()["kernel_ms"]
        host = f0.copy()
        e2e = 0.0
        h = _pinned_fields(eaf, f0)
        for _ in range(args.steps):
            _refill(h, f0)
            cg.pressure_assemble(h)
            e2e += cg.last_timing()["e2e_ms"]
        res = cg.pressure_assemble(host)
    import oracle
    ref = f0.copy()
    t0 = time.perf_counter()
    res_ref = oracle.pressure_assemble(ref)
    cpu_s = time.perf_counter() - t0
    same = all(np.array_equal(a, ref.outputs()[k]) for k, a in host.outputs().items())
    value = n * args.steps / (kms / 1e3)
    achieved = ASSEMBLY_BYTES_PER_ELEM * nh * args.steps / (kms / 1e3) / 1e9
    peak, kind = measured_peaks()
    line = _base_line("pressure-equation assembly, cells/s (60x120x84, two phases)", value,
                      "cells/s", args.steps, args.warmup, kms / args.steps,
                      "gradients + liquid/gas Rhie-Chow faces + compressibility + "
                      "diagonal + boundary folding + continuity residual",
                      {"mesh": [nr, nth, nz], "cells": n, "phases": 2, "flags": 7,
                       "l2": "flushed between steps (256 MiB memset)"})
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                        "algorithmic_bytes_per_halo_element": ASSEMBLY_BYTES_PER_ELEM,
                        "kernel": "asm_gradient_kernel + asm_face_kernel + "
                                  "asm_cell_kernel + asm_residual_kernel"}
    line["e2e"] = {"value": n * args.steps / (e2e / 1e3), "unit": "cells/s",
                   "h2d_bytes_per_step": 24 * 8 * nh + 4 * 4 * nh
                   + 8 * (nr + nth + nz + 12),
                   "d2h_bytes_per_step": 18 * 8 * nh + 3 * 4 * nh + 8}
    line["bitwise_equal_to_cpu"] = bool(same)
    line["residual_rel_diff"] = abs(res - res_ref) / abs(res_ref)
    line["cpu_baseline"] = {"value": n / cpu_s, "unit": "cells/s", "cores": 1, "kind": "port",
                            "sample": f"oracle port, one call, one thread, {cpu_s:.3f} s"}
    line["gpu_launches"] = 4 * args.steps
    print(json.dumps(line), flush=True)
    return 0


def run_pstep(args):
    """One whole pressure step (solve_pressure_correction's numerics: the
    assembly, the CG to 1e-8, the post-CG corrections) on a consistent
    60x120x84 furnace state (eafgen.make_pressure_state, both phases, every
    switch on), fields resident on the device (value) and through the
    host-pointer entry (e2e); each step restarts from the same state (the
    restore is outside the timed region), so every step is the same work.
    CPU baseline: the oracle's assembly and corrections on one thread, its CG
    on all host threads."""
    import numpy as np
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz = MESH[:3]
    n = nr * nth * nz
    nh = (nr + 4) * (nth + 4) * (nz + 4)
    f0 = g.make_pressure_state(nr, nth, nz, seed=0, flags=7)
    alpha_p, max_iter, tol = 0.7, 20000, 1e-8
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    pristine = {k: torch.from_numpy(v).cuda() for k, v in f0.__dict__.items()
                if isinstance(v, np.ndarray)}
    d = f0.copy()
    for k, v in pristine.items():
        setattr(d, k, v.clone())

    def restore():
        for k, v in pristine.items():
            getattr(d, k).copy_(v)

    with eaf.CGSolver(nr, nth, nz) as cg:
        cg.set_form(CG_FORMS[args.cg_form])
        for _ in range(args.warmup):
            restore()
            cg.pressure_step(d, alpha_p, max_iter, tol, device_ptrs=True)
        kms, iters = 0.0, []
        for _ in range(args.steps):
            restore()
            flush.fill_(1)
            torch.cuda.synchronize()
            _, cres, nit, _ = cg.pressure_step(d, alpha_p, max_iter, tol, device_ptrs=True)
            kms += cg.last_timing()["kernel_ms"]
            iters.append(nit)
        cg_kernel = solver_kernel_name(cg, cg.last_launch())
        e2e = 0.0
        h = _pinned_fields(eaf, f0)
        for _ in range(args.steps):
            _refill(h, f0)
            cg.pressure_step(h, alpha_p, max_iter, tol)
            e2e += cg.last_timing()["e2e_ms"]
        host = f0.copy()
        res, cres, nit, _ = cg.pressure_step(host, alpha_p, max_iter, tol)
    import oracle
    ref = f0.copy()
    t0 = time.perf_counter()
    cont = oracle.pressure_assemble(ref)
    s = g.System(nr=nr, nth=nth, nz=nz, **{k: getattr(ref, k) for k in g.COEF_NAMES})
    cores = os.cpu_count() or 1
    cres_o, nit_o = oracle.cg(s, ref.pp, max_iter, tol, nthreads=cores)
    oracle.pressure_correct(g.pcorr_view(ref, alpha_p))
    cpu_s = time.perf_counter() - t0
    ms = kms / args.steps
    line = _base_line("pressure steps/s (assembly + CG to 1e-8 + corrections, 60x120x84)",
                      1e3 / ms, "steps/s", args.steps, args.warmup, ms,
                      "solve_pressure_correction numerics on the device: assembly, CG, "
                      "post-CG corrections",
                      {"mesh": [nr, nth, nz], "cells": n, "phases": 2, "flags": 7,
                       "cg_tol": tol, "cg_iterations": int(np.median(iters)),
                       "cg_form": args.cg_form,
                       "l2": "flushed between steps (256 MiB memset)"})
    cg_bytes = 120 * n * float(np.median(iters))
    step_bytes = cg_bytes + ASSEMBLY_BYTES_PER_ELEM * nh + PCORR_BYTES_PER_CELL * n
    achieved = step_bytes / (ms / 1e3) / 1e9
    peak, kind = measured_peaks()
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                        "algorithmic_bytes": "120 B per cell-iteration (CG) + 364 B per halo "
                                             "element (assembly) + 300 B per cell "
                                             "(corrections)",
                        "kernel": f"asm_* + {cg_kernel} + pcorr_*"}
    line["e2e"] = {"value": 1e3 / (e2e / args.steps), "unit": "steps/s",
                   "h2d_bytes_per_step": 24 * 8 * nh + 4 * 4 * nh + 8 * (nr + nth + nz + 12),
                   "d2h_bytes_per_step": 18 * 8 * nh + 3 * 4 * nh + 7 * 8 * nh}
    line["cg"] = {"residual": cres, "iterations": nit, "cpu_iterations": nit_o}
    line["continuity_residual"] = res
    line["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "steps/s", "cores": cores,
                            "kind": "port",
                            "sample": f"oracle port: assembly and corrections on one thread, "
                                      f"CG on {cores} threads, one step, {cpu_s:.2f} s"}
    # assembly 4; pack, solver, unpack (+ the p.q slot fill of a flat grid); corrections 3
    cg_launches = 4 if cg_kernel in ("cg_keep_kernel", "cg_f64_kernel") else 3
    line["gpu_launches"] = (4 + cg_launches + 3) * args.steps
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """96 uneven systems (40 at 12x24x16, 30 at 18x36x24, 20 at 35x70x50,
    6 at 60x120x84; seed = system id) in one persistent launch replayed from
    a CUDA graph, against the same systems solved one by one.

    Under torchrun (N ranks, one GPU each) the systems are partitioned
    across the ranks by estimated work within each GPU's HBM budget
    (multigpu.partition), every rank solves its share in one batched launch
    of its own, and the line reports the whole job: all systems over the
    slowest rank's device time (strong scaling: the mix is fixed)."""
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    mg = importlib.import_module(PKG + ".multigpu")
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    specs = []
    for (dims, count) in g.BATCH_MIX:
        for _ in range(count):
            specs.append(dims)
    items = [mg.Item(k, d[0] * d[1] * d[2], mg.device_footprint(*d[:3]),
                     mg.estimated_work(*d[:3])) for k, d in enumerate(specs)]
    plans = {}

    def share(form):
        mixed = form == "mixed"

        def solve_share(mine):
            keys = [it.key for it in mine]
            if not keys:
                return 0.0, {}
            systems = [g.make_system(*specs[k], seed=k) for k in keys]
            dims = [(s.nr, s.nth, s.nz) for s in systems]
            dev = [[torch.from_numpy(a).cuda() for a in s.arrays()] for s in systems]
            phis = [torch.zeros(g.halo_shape(*d), dtype=torch.float64, device="cuda")
                    for d in dims]
            kw = dict(mixed=mixed, max_iter=args.mixed_inner if mixed else MAX_ITER,
                      tol=TOL, max_outer=args.mixed_outer, inner_tol=0.1)
            with eaf.Batch(dims) as b:
                for i in range(len(systems)):
                    b.set_system(i, dev[i][:8], phis[i], device_ptrs=True)
                plans[form] = b.plan()
                plans["widths"] = sorted({(d, b.lane_width(i)) for i, d in enumerate(dims)})
                for _ in range(args.warmup if not mixed else 1):
                    for p in phis:
                        p.zero_()
                    b.solve(**kw)
                ms = 0.0
                steps = args.steps if not mixed else 1
                for _ in range(steps):
                    for p in phis:
                        p.zero_()
                    torch.cuda.synchronize()
                    b.solve(**kw)
                    ms += b.last_ms
                res = {}
                for i, k in enumerate(keys):
                    r, nit, no, st = b.result(i)
                    res[k] = (r, nit, st)
            return ms / steps / 1e3, res
        return solve_share

    out = {}
    for form in ("fp64", "mixed"):
        t, res, parts = mg.solve_sharded(items, share(form))
        ci = sum(specs[k][0] * specs[k][1] * specs[k][2] * res[k][1] for k in res)
        out[form] = {"ms_per_batch": t * 1e3, "cell_iters_per_s": ci / t,
                     "solves_per_s": len(specs) / t,
                     "max_residual": max(r for r, _, _ in res.values()),
                     "systems_per_rank": [len(p) for p in parts]}
    seq = None
    if world == 1:
        # the same systems one by one through the single-system FP64 solver
        seq_ms = 0.0
        for k, d in enumerate(specs):
            s = g.make_system(*d, seed=k)
            dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
            phi = torch.zeros(g.halo_shape(*d[:3]), dtype=torch.float64, device="cuda")
            with eaf.CGSolver(*d[:3]) as cg:
                cg.solve(dev[:8], phi, MAX_ITER, TOL, device_ptrs=True)
                phi.zero_()
                torch.cuda.synchronize()
                cg.solve(dev[:8], phi, MAX_ITER, TOL, device_ptrs=True)
                seq_ms += cg.last_timing()["solve_ms"]
        seq = {"ms_per_96": seq_ms, "solves_per_s": len(specs) / (seq_ms / 1e3)}
    if rank != 0:
        return 0
    total_cells = sum(d[0] * d[1] * d[2] for d in specs)
    grid, block, nlanes = plans.get("fp64", (0, 0, 0))
    line = _base_line("batched pressure-CG solves/s (96-system mix, one launch)",
                      out["fp64"]["solves_per_s"], "solves/s", args.steps, args.warmup,
                      out["fp64"]["ms_per_batch"], "96 uneven systems, one persistent launch",
                      {"systems": len(specs), "cells": total_cells,
                       "mix": [[list(d[:3]), c] for d, c in g.BATCH_MIX],
                       "plan_rank0": {"grid": grid, "block": block, "lanes": nlanes},
                       "lane_widths": [[list(d), w] for d, w in plans.get("widths", [])],
                       "graph": "pack + persistent batch kernel + unpack captured once, replayed",
                       "parallelism": f"systems sharded over {world} GPU(s), one batch each"})
    line["n_gpus"] = world
    line["scaling"] = "strong"
    line["forms"] = out
    if seq is not None:
        line["sequential_fp64"] = seq
        line["speedup_vs_sequential_fp64"] = out["fp64"]["solves_per_s"] / seq["solves_per_s"]
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Poisson arrivals of simulated furnace runs (serving mix), 50 warm-
    started solves per run, continuous batching; p50/p99 per rate.

    Under torchrun (N ranks, one GPU each) every rank serves its own stream
    of rate lambda/N on its own GPU (runs never span GPUs); the line reports
    all solves over the slowest rank's wall time and p50/p99 over every
    rank's client-observed latencies."""
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    sc = importlib.import_module(PKG + ".serve_client")
    mg = importlib.import_module(PKG + ".multigpu")
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    mix = g.SERVE_MIX
    pool = sc.build_pool(g, eaf, mix, 4, 0)
    rates = [float(r) for r in args.rates.split(",")]
    points = []
    for mixed in ([False, True] if args.serve_mixed else [False]):
        with eaf.Server(budget_bytes=150e9, mixed=mixed,
                        max_iter=args.mixed_inner if mixed else MAX_ITER, tol=TOL,
                        max_outer=args.mixed_outer, inner_tol=0.1) as srv:
            for rate in (rates if not mixed else rates[:1]):
                def stream():
                    return sc.run_stream(srv, g, eaf, pool, mix, rate / world,
                                         duration=args.serve_runs / rate,
                                         solves=args.solves_per_run,
                                         seed=int(rate * 100) + 7919 * rank, max_wall=900.0)
                per_rank = mg.gather_outcomes(stream)
                st = {k: v for k, v in per_rank[0].items() if k != "client_latency_ms"}
                if world > 1:
                    st = sc.merge_streams(per_rank)
                    st["p50_ms"], st["p99_ms"] = st["client_p50_ms"], st["client_p99_ms"]
                    st["mean_ms"] = float(np.mean(np.concatenate(
                        [r["client_latency_ms"] for r in per_rank])))
                st.update({"rate_runs_per_s": rate, "mixed": mixed, "gpus": world})
                points.append(st)
    # plain FP64 per-solve path on the same pool, one solve at a time
    per = {}
    for (dims, share) in mix:
        nr, nth, nz, _ = dims
        with eaf.CGSolver(nr, nth, nz) as cg:
            phi = eaf.host_empty(g.halo_shape(nr, nth, nz))
            phi[...] = 0.0
            times = []
            for k, arrs in enumerate(pool[dims]):
                cg.solve(arrs, phi, MAX_ITER, TOL)
                times.append(cg.last_timing()["e2e_ms"])
            per[str([nr, nth, nz])] = float(np.mean(times[1:] if len(times) > 1 else times))
    if rank != 0:
        return 0
    mean_ms = sum(share * per[str(list(d[:3]))] for d, share in mix)
    first = [p for p in points if not p["mixed"]]
    best = max(first, key=lambda p: p["solves_per_s"])
    line = _base_line("serve p99 latency @1e-8 resid (Poisson furnace runs)",
                      best["p99_ms"], "ms", len(points), 0, best["mean_ms"],
                      "serving stream, continuous batching",
                      {"mix": [[list(d[:3]), sh] for d, sh in mix],
                       "solves_per_run": args.solves_per_run,
                       "runs_per_rate": args.serve_runs,
                       "rates_runs_per_s": rates, "budget_gb": 150,
                       "parallelism": f"one stream of rate/{world} per GPU"})
    line["n_gpus"] = world
    line["higher_is_better"] = False
    line["points"] = points
    line["per_solve_fp64"] = {"mean_ms_by_mesh": per, "mix_mean_ms": mean_ms,
                              "solves_per_s": 1e3 / mean_ms}
    print(json.dumps(line), flush=True)
    return 0


def run_fixed(args):
    """A fixed amount of work per launch, for ncu captures and per-iteration
    timing: the seeded system of --mesh uploaded once, then --repeat solves
    of exactly --iters iterations (tol 0) through the device-pointer entry;
    or --batch-size systems of the batch mix (round robin) at --iters
    iterations each; or --tdma-sweeps sweeps of a transport system
    (--fixed-tdma)."""
    import torch
    eaf = importlib.import_module(PKG)
    g = importlib.import_module(PKG + ".eafgen")
    nr, nth, nz = args.mesh
    runs = []
    if args.batch_size:
        meshes = [d for d, _ in g.BATCH_MIX]
        systems = [g.make_system(*meshes[k % len(meshes)], seed=k)
                   for k in range(args.batch_size)]
        dims = [(s.nr, s.nth, s.nz) for s in systems]
        dev = [[torch.from_numpy(a).cuda() for a in s.arrays()] for s in systems]
        phis = [torch.zeros(g.halo_shape(*d), dtype=torch.float64, device="cuda")
                for d in dims]
        cells = sum(d[0] * d[1] * d[2] for d in dims)
        with eaf.Batch(dims) as b:
            for i in range(len(systems)):
                b.set_system(i, dev[i], phis[i], device_ptrs=True)
            for _ in range(args.repeat):
                for p in phis:
                    p.zero_()
                torch.cuda.synchronize()
                b.solve(max_iter=args.iters, tol=0.0)
                runs.append({"batch_ms": b.last_ms,
                             "cell_iters_per_s": cells * args.iters / (b.last_ms / 1e3)})
            launch = list(b.plan())
        case = {"batch": dims}
    elif args.fixed_tdma:
        s = g.make_transport_system(nr, nth, nz, seed=0)
        dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
        phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
        with eaf.CGSolver(nr, nth, nz) as cg:
            for _ in range(args.repeat):
                phi.zero_()
                torch.cuda.synchronize()
                cg.tdma(dev, phi, args.tdma_sweeps, device_ptrs=True)
                t = cg.last_timing()
                runs.append({"sweeps": args.tdma_sweeps, "kernel_ms": t["kernel_ms"],
                             "ms_per_sweep": t["kernel_ms"] / args.tdma_sweeps})
            launch = list(cg.last_launch())
        case = {"mesh": [nr, nth, nz], "tdma": True}
    else:
        s = g.make_system(nr, nth, nz, args.spheres, seed=0)
        dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
        phi = torch.zeros(g.halo_shape(nr, nth, nz), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        with eaf.CGSolver(nr, nth, nz) as cg:
            cg.set_form(CG_FORMS[args.cg_form])
            if args.launch:
                cg.set_launch(*args.launch)
            if args.cluster is not None:
                cg.set_cluster(args.cluster)
            if args.kernel is not None:
                cg.set_kernel({"loads": cg.KERNEL_LOADS, "stream": cg.KERNEL_STREAM,
                               "slots": cg.KERNEL_SLOTS, "keep": cg.KERNEL_KEEP}[args.kernel])
            for _ in range(args.repeat):
                phi.zero_()
                torch.cuda.synchronize()
                if args.mixed:
                    res, nit, nout, st = cg.solve_mixed(
                        dev, phi, tol=0.0, inner_tol=1e-30, max_outer=1,
                        max_inner=args.iters, device_ptrs=True)
                else:
                    res, nit, st = cg.solve(dev, phi, args.iters, 0.0, device_ptrs=True)
                t = cg.last_timing()
                runs.append({"iters": nit, "residual": res, "status": st,
                             "kernel_ms": t["kernel_ms"], "solve_ms": t["solve_ms"],
                             "us_per_iter": 1e3 * t["kernel_ms"] / max(nit, 1)})
            launch = list(cg.last_launch())
            kernel = cg.last_kernel()
        case = {"mesh": [nr, nth, nz], "iters": args.iters, "mixed": args.mixed,
                "cg_form": args.cg_form, "flat_kernel": kernel}
    print(json.dumps({"workload": "fixed", "case": case, "launch": launch, "runs": runs}),
          flush=True)
    return 0


def run_sharded_workload(fn, args):
    """A workload whose independent systems are sharded over the ranks of a
    torchrun launch (one GPU each, NCCL for the host-side result gather)."""
    import datetime

    import torch
    import torch.distributed as dist
    local_rank = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device(f"cuda:{local_rank}"))
    try:
        return fn(args)
    finally:
        dist.destroy_process_group()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-iters", type=int, default=1500,
                    help="iteration cap per reference-arm step (bounded sample)")
    ap.add_argument("--tdma-sweeps", type=int, default=3)
    ap.add_argument("--workload", choices=["production", "fine", "batch", "serve", "tdma",
                                           "pcorr", "assemble", "pstep", "fixed"],
                    default="production")
    ap.add_argument("--cg-form", choices=sorted(CG_FORMS), default=DEFAULT_CG_FORM,
                    help="FP64 CG recurrences: the reference's (two all-reduces per "
                         "iteration) or the single-reduction rearrangement")
    ap.add_argument("--cluster", type=int, default=None,
                    help="blocks per thread-block cluster of the FP64 CG (1 = none, "
                         "0 = the tuned choice; default: the tuned choice)")
    ap.add_argument("--mixed-outer", type=int, default=30)
    ap.add_argument("--mixed-inner", type=int, default=3000)
    ap.add_argument("--rates", default="5,20,50,200")
    ap.add_argument("--serve-runs", type=int, default=25)
    ap.add_argument("--solves-per-run", type=int, default=50)
    ap.add_argument("--serve-mixed", action="store_true")
    # --workload fixed
    ap.add_argument("--mesh", type=int, nargs=3, default=list(MESH[:3]))
    ap.add_argument("--spheres", type=int, default=MESH[3])
    ap.add_argument("--iters", type=int, default=400)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--launch", type=int, nargs=2, default=None, metavar=("BLOCK", "GRID"))
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--batch-size", type=int, default=0)
    ap.add_argument("--kernel", choices=["loads", "stream", "slots", "keep"], default=None,
                    help="FP64 kernel on a flat grid (default: the tuned choice)")
    ap.add_argument("--fixed-tdma", action="store_true")
    args = ap.parse_args(argv)
    if (args.workload in ("batch", "serve") and args.impl == "ours"
            and _env_int("WORLD_SIZE", 1) > 1):
        return run_sharded_workload(run_batch if args.workload == "batch" else run_serve, args)
    if args.workload != "production" and args.impl == "ours":
        return {"fine": run_fine, "batch": run_batch, "serve": run_serve,
                "tdma": run_tdma, "pcorr": run_pcorr,
                "assemble": run_assemble, "pstep": run_pstep,
                "fixed": run_fixed}[args.workload](args)
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local_rank}"))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
