"""Benchmark of the per-Newton-step HDG hot path on B200.

Workload: 2D p-n diode, 256 x 256 quads, HDG degree 2 (65 536 cells), GaAs
material, SRH recombination, FP64.  A step is one pass of the hot path over
all cells: the per-cell assembly + static condensation onto the trace
(ddhdg_assemble_condense) and the cell reconstruction from a trace update
(ddhdg_reconstruct).  The metric is HDG cells condensed per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the diode
(the hot path is per cell and per device; no data-path collective) and the
time is the maximum over ranks.  --impl reference times the reference's
algorithm on the host cores (the CPU oracle restating it; the reference
itself needs deal.II and cannot be built here).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(dim=2, m=256, k=2)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_flops_per_cell(dim, k):
    """Condensation flops of one cell in LU form on the full local system
    (cell dofs Nc = 3(d+1)(k+1)^d, trace dofs Nt = 6d(k+1)^(d-1)):
    2/3 Nc^3 (factorisation of cc) + 2 Nc^2 (Nt+1) (solve for [ct | rhs])
    + 2 Nt Nc (Nt+1) (Schur product and rhs update)."""
    Nc = 3 * (dim + 1) * (k + 1) ** dim
    Nt = 6 * dim * (k + 1) ** (dim - 1)
    return 2 * Nc ** 3 / 3 + 2 * Nc ** 2 * (Nt + 1) + 2 * Nt * Nc * (Nt + 1)


def flops_per_cell(dim, k, ncomp=3):
    """FP64 flops the condense kernel executes per cell (2 per FMA), after
    the flux unknowns are eliminated through the constant mass matrix: S and
    R assembly from the quadrature contractions, the inverse of S,
    Y = S^-1 [residual | trace columns], the reduced trace operator T and
    tt = T Y_t + tc_W Q_t."""
    nb = (k + 1) ** dim
    nf = (k + 1) ** (dim - 1)
    F = 2 * dim
    nqc, nqf = nb, nf
    Fq, Ft = F * nqf, F * nf
    Nt = F * ncomp * nf
    Ns = ncomp * nb
    fma = (Ns * Ns * (nqc * (1 + dim) + 2 * Fq)            # S
           + Ns * ncomp * Ft * (nqc * dim + Fq)            # R, trace columns
           + Ns * (nqc * (1 + dim) + Fq)                   # R, residual column
           + Ns ** 3                                       # S^-1
           + Ns * Ns * (1 + Nt)                            # Y
           + Nt * Ns * 2 * nqf                             # T
           + Nt * Nt * Ns + Nt * Nt * nqf)                 # tt
    return 2 * fma


def fp64_peak_tflops(dev):
    """cuBLAS DGEMM 8192^3 throughput on this GPU (the FP64 ceiling)."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        c = a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        c = a @ b
    e1.record()
    torch.cuda.synchronize()
    del a, b, c
    torch.cuda.empty_cache()
    return 3 * 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12


# DRAM bytes (read + write) per cell of one launch of the FP64 condense
# kernel, measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on
# the 128 x 128 mesh of the same diode and scaled to a launch by the cells it
# processes.  The figure belongs to one version of the kernel source: it is
# reported only while the sha256 of hdg_condense3.cuh matches, else null.
# Capture: 14 794 752 bytes read + 258 160 128 written for 16 384 cells.
TRAFFIC = {"bytes_per_cell": 16660, "kernel_source": "ddhdg_b200/csrc/hdg_condense3.cuh",
           "kernel_sha256": "1cfe923fd485f5579e11ee1313a621295d4d6072db3a2e1641a45f1aea850a50"}


def traffic_bytes_per_cell():
    import hashlib

    if not TRAFFIC["kernel_sha256"]:
        return None
    try:
        with open(os.path.join(ROOT, TRAFFIC["kernel_source"]), "rb") as f:
            sha = hashlib.sha256(f.read()).hexdigest()
    except OSError:
        return None
    return TRAFFIC["bytes_per_cell"] if sha == TRAFFIC["kernel_sha256"] else None


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def bytes_per_cell(dim, k, ncomp=3):
    nb = (k + 1) ** dim
    nf = (k + 1) ** (dim - 1)
    F = 2 * dim
    Nc_all = 3 * (dim + 1) * nb
    Nt = F * ncomp * nf
    Ns = ncomp * nb
    condense = 8 * (Nc_all + F * 3 * nf + nb) + 8 * (Nt * Nt + 2 * Nt) + 4 * Nt + 8 * Ns * (1 + Nt)
    reconstruct = 8 * (Ns * (1 + Nt) + Nc_all + 2 * F * 3 * nf) + 8 * Nc_all
    return condense, reconstruct


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(k_sample_cells=4096, steps=1, nthreads=None):
    """The oracle (the reference's per-cell algorithm restated in C++,
    OpenMP over cells) on a slab of the same diode (same cell size, degree
    and physics; 64 x 64 cells by default): assembly + condensation +
    reconstruction."""
    from oracle.oracle import OracleSolver
    from ddhdg_b200 import workloads as cases

    m_side = int(round(k_sample_cells ** 0.5))
    length = m_side / WORKLOAD["m"]
    pb, prm, adim = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"], length=length)
    cores = nthreads or os.cpu_count() or 1
    o = OracleSolver(pb, prm, adim, nthreads=cores)
    o.compute_local_charge_neutrality()
    o.project_quasi_fermi(1)
    o.project_quasi_fermi(2)
    upd = 1e-6 * np.ones((o.nfaces, 3, o.nf))
    best = None
    for _ in range(steps):
        t0 = time.perf_counter()
        o.assemble_condense()
        o.reconstruct(upd)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return {"value": o.ncells / best, "unit": "cells/s", "cores": cores,
            "kind": "port", "cells": o.ncells, "ms_per_sample": best * 1e3, "cpu_model": cpu_model(),
            "sample": f"{m_side}x{m_side} cells of the 256x256 k=2 diode (same cell size), "
                      f"assembly+condensation+reconstruction, {o.ncells} cells per step"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = []
    info = None
    for _ in range(args.warmup):
        cpu_baseline(steps=1)
    for _ in range(args.steps):
        info = cpu_baseline(steps=1)
        steps.append(info["value"])
    v = float(np.median(steps))
    single = cpu_baseline(k_sample_cells=256, steps=1, nthreads=1)
    line = {
        "impl": "reference", "metric": "HDG cells condensed/s (assemble+condense+reconstruct)",
        "value": v, "unit": "cells/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        # what one timed step processed: the bounded 64 x 64 sample
        "ms_per_step": info["cells"] / v * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "2D p-n diode, HDG degree 2, FP64, cell size 1/256 um: a 64x64-cell sample "
                               "of the 256x256 mesh per step (cells are independent, so cells/s carries over)",
                   "cells": info["cells"], "full_mesh_cells": 65536},
        "ms_per_cell": 1e3 / v,
        "full_mesh_ms_estimate": 65536 / v * 1e3,
        "cpu_model": info["cpu_model"],
        "single_thread": {"value": single["value"], "unit": "cells/s", "cells": single["cells"]},
        "cpu_baseline": dict(info, value=v),
        "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_serve(args):
    """The serving configuration: Poisson arrivals (seeded) of 2D (32^2..256^2)
    and 3D (8^3..16^3, degree 1) diode solves, degrees 1-2, biases uniform in
    0..0.8 V; continuous batching on one GPU (ddhdg_b200.serving)."""
    import torch

    from ddhdg_b200 import serving

    torch.cuda.init()
    # warm the library and the kernels once (not part of the stream)
    serving.solve_one(serving.Request(-1, 2, 32, 1, 0.1, 0.0), mixed=args.serve_precision == "mixed")
    reqs = serving.poisson_requests(args.serve_requests, args.serve_rate, seed=2024,
                                    sizes_3d=(args.serve_3d_min, args.serve_3d_max))
    mixed = args.serve_precision == "mixed"
    server = serving.DiodeServer(max_inflight=16, mixed=mixed)
    t0 = time.perf_counter()
    res = server.run(reqs)
    wall = time.perf_counter() - t0
    st = serving.latency_stats(res, wall)
    line = {"metric": "serve p50/p99 latency (diode solves, continuous batching)",
            "value": st["p99_s"], "unit": "s", "higher_is_better": False, "n_gpus": 1, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"Poisson stream of 2D 32^2..256^2 (k 1-2) and 3D {args.serve_3d_min}^3.."
                                   f"{args.serve_3d_max}^3 (k 1) diode solves, bias U[0, 0.8] V, equilibrium + "
                                   "warm-started Newton; kernel-level continuous batching (one condensation "
                                   "launch per server step over the requests in flight)",
                       "requests": len(reqs), "rate_per_s": args.serve_rate, "seed": 2024,
                       "max_inflight": server.max_inflight,
                       "precision": ("mixed: FP32 Jacobian, FP64 residuals and trace solve (FP64 for 2D "
                                     "degree 3 and 3D degree 2, which have no mixed kernel)") if mixed else "fp64"},
            "server_steps": server.steps, "peak_batch": server.peak_batch,
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "mean_s": st["mean_s"],
            "solves_per_s": st["solves_per_s"], "cells_per_s": st["cells_per_s"],
            "converged": st["converged"], "peak_inflight": server.peak_inflight, "wall_s": wall,
            "per_request": [{"dim": q.dim, "m": q.m, "k": q.k, "bias": round(q.bias, 3),
                             "arrival_s": round(r.arrival, 3), "wait_s": round(r.start - r.arrival, 3),
                             "latency_s": round(r.latency, 3), "iterations": r.iterations}
                            for q, r in zip(reqs, res)]}
    print(json.dumps(line))


def serve_quick(n=10, rate=4.0, seed=7):
    """A short seeded Poisson stream of small diode solves through the
    serving layer (2D 32^2..96^2 at degree 1-2, 3D 8^3..12^3 at degree 1,
    mixed-precision condensation): p50 / p99 latency and solves/s, for the
    default bench line."""
    from ddhdg_b200 import serving

    serving.solve_one(serving.Request(-1, 2, 32, 1, 0.1, 0.0), mixed=True)  # warm the kernels
    reqs = serving.poisson_requests(n, rate, seed=seed, sizes_2d=(32, 96), sizes_3d=(8, 12))
    server = serving.DiodeServer(max_inflight=16, mixed=True)
    t0 = time.perf_counter()
    res = server.run(reqs)
    wall = time.perf_counter() - t0
    st = serving.latency_stats(res, wall)
    return {"p50_s": st["p50_s"], "p99_s": st["p99_s"], "solves_per_s": st["solves_per_s"],
            "converged": st["converged"], "requests": n, "rate_per_s": rate, "seed": seed,
            "peak_inflight": server.peak_inflight, "peak_batch": server.peak_batch,
            "server_steps": server.steps, "wall_s": wall,
            "workload": "Poisson stream of 2D 32^2..96^2 (k 1-2) and 3D 8^3..12^3 (k 1) diode solves, "
                        "bias U[0, 0.8] V, mixed-precision condensation (full-size stream: bench.py --serve)"}


def batch_quick(n=64, steps=5):
    """The first n diodes of the batched configuration (seed 2025: mesh
    cells per side U[16, 128], degree U{1, 2, 3}) condensed in one launch and
    reconstructed in one more per step, tile shapes autotuned: cells/s for
    the default bench line (the full 512-diode batch: bench.py --batch)."""
    import torch

    from ddhdg_b200 import _lib
    from ddhdg_b200 import workloads as cases
    from ddhdg_b200.batch import CondenseBatch
    from ddhdg_b200.solver import NPSolver

    specs = cases.batch_diodes(512, seed=2025)[:n]
    solvers = []
    for pb, prm, adim, _ in specs:
        g = NPSolver(pb, prm, adim)
        g.compute_local_charge_neutrality()
        for c in (1, 2):
            _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                                 g.trace_state.data_ptr(), g._sp()), "project_density")
        solvers.append(g)
    batch = CondenseBatch(solvers)
    for i in range(n):
        batch.update_trace[i].fill_(1e-6)
    batch.autotune(reps=1)
    stream = batch.stream
    for _ in range(3):
        batch.condense()
        batch.reconstruct()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for _ in range(steps):
        batch.condense()
    ev[1].record(stream)
    for _ in range(steps):
        batch.reconstruct()
    ev[2].record(stream)
    torch.cuda.synchronize()
    cm, rm = ev[0].elapsed_time(ev[1]) / steps, ev[1].elapsed_time(ev[2]) / steps
    out = {"devices": n, "cells": batch.cells, "condense_ms": cm, "reconstruct_ms": rm,
           "cells_per_s": batch.cells / ((cm + rm) * 1e-3), "launches_per_step": 2, "shape": batch.shape(),
           "workload": "the first 64 diodes of the 512-diode batch (seed 2025; 2D, cells per side U[16,128], "
                       "degree U{1,2,3}), FP64 (full batch: bench.py --batch)"}
    batch.close()
    del solvers
    torch.cuda.empty_cache()
    return out


def run_bias_sweep(args):
    """The second diode configuration end to end: equilibrium, then a forward
    bias sweep 0.0..0.8 V in 0.05 V steps, each point warm-started, every
    Newton step on the device (assembly + condensation, nested-dissection
    trace solve, reconstruction).  Consistent Jacobian (the reference's
    diverges on this diode)."""
    import torch

    from ddhdg_b200 import workloads as cases
    from ddhdg_b200.solver import NPSolver

    m_side = args.cells_per_side
    pb, prm, adim = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"], length=m_side / WORKLOAD["m"])
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    g = NPSolver(pb, prm, adim)
    t0 = time.perf_counter()
    req = g.compute_thermodynamic_equilibrium()
    torch.cuda.synchronize()
    t_eq = time.perf_counter() - t0
    biases = [0.05 * i for i in range(17)]
    steps, points = 0, []
    t0 = time.perf_counter()

    def keep(v, s, r):
        points.append({"bias": round(v, 3), "iterations": r.iterations, "converged": bool(r.converged)})

    if not args.mixed:
        cases.bias_sweep(g, pb, biases, 1e-10, 1e-10, 50, callback=keep)
        torch.cuda.synchronize()
        t_sweep = time.perf_counter() - t0
    else:
        # the same sweep with the mixed-precision condensation, in lockstep
        # from the same equilibrium state: every point's final V, n, p against
        # the FP64 sweep's (largest difference per component block, relative
        # to the block's largest magnitude)
        pbm, prmm, adimm = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"],
                                       length=m_side / WORKLOAD["m"], precision=1)
        prmm.consistent_drift_jacobian = True
        prmm.consistent_recombination_jacobian = True
        gm = NPSolver(pbm, prmm, adimm)
        gm.set_state(g.get_cell_state(), g.get_trace_state())
        d, nb = WORKLOAD["dim"], (WORKLOAD["k"] + 1) ** WORKLOAD["dim"]
        t_sweep = t_mixed = 0.0
        for v in biases:
            tp = time.perf_counter()
            cases.set_bias(pb, v)
            g.update_boundary_tables()
            r = g.run(1e-10, 1e-10, 50)
            torch.cuda.synchronize()
            t_sweep += time.perf_counter() - tp
            tp = time.perf_counter()
            cases.set_bias(pbm, v)
            gm.update_boundary_tables()
            rm = gm.run(1e-10, 1e-10, 50)
            torch.cuda.synchronize()
            t_mixed += time.perf_counter() - tp
            c64, t64, c32, t32 = g.get_cell_state(), g.get_trace_state(), gm.get_cell_state(), gm.get_trace_state()
            err = 0.0
            for c in range(3):
                ia = slice(c * (d + 1) * nb, (c + 1) * (d + 1) * nb)
                for x, y in ((c32[:, ia], c64[:, ia]), (t32[:, c], t64[:, c])):
                    err = max(err, float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)))
            points.append({"bias": round(v, 3), "iterations": r.iterations, "converged": bool(r.converged),
                           "mixed_iterations": rm.iterations, "mixed_converged": bool(rm.converged),
                           "mixed_vs_fp64_rel_diff": err})
    steps = sum(p["iterations"] for p in points)
    line = {"metric": "bias sweep wall time (17 points, warm-started Newton)", "value": t_sweep, "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2D p-n diode {m_side}x{m_side} quads, HDG degree 2, FP64, 0..0.8 V",
                       "trace_dofs": int(g.sizes().n_trace_dofs), "cells": g.ncells},
            "equilibrium_s": t_eq, "equilibrium_iterations": req.iterations,
            "newton_steps": steps, "ms_per_newton_step": 1e3 * t_sweep / max(steps, 1), "points": points}
    if args.mixed:
        msteps = sum(p["mixed_iterations"] for p in points)
        line["mixed"] = {"sweep_s": t_mixed, "newton_steps": msteps,
                         "ms_per_newton_step": 1e3 * t_mixed / max(msteps, 1),
                         "max_rel_diff_vs_fp64": max(p["mixed_vs_fp64_rel_diff"] for p in points)}
    print(json.dumps(line))


def run_batch(args):
    """The batched configuration: a seeded batch of 2D diodes (mesh cells per
    side uniform in 16..128, degree uniform in {1, 2, 3}, doping log-uniform
    in 1e21..1e24 m^-3, junction uniform in 0.3..0.7), condensed in ONE
    persistent launch per Newton step and reconstructed in one more
    (ddhdg_batch_*, tile shapes from the autotuner, replayed from CUDA
    graphs), FP64.  Timed with CUDA events over `steps` batch steps; next to
    it the same work as one launch per device (a batch of one per device) on
    the first `compare` devices, and the batch of those devices alone."""
    import torch

    from ddhdg_b200 import _lib
    from ddhdg_b200 import workloads as cases
    from ddhdg_b200.batch import CondenseBatch
    from ddhdg_b200.solver import NPSolver

    t0 = time.perf_counter()
    specs = cases.batch_diodes(args.batch_devices, seed=2025)
    solvers = []
    for pb, prm, adim, _ in specs:
        g = NPSolver(pb, prm, adim)
        g.compute_local_charge_neutrality()
        for c in (1, 2):
            _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                                 g.trace_state.data_ptr(), g._sp()), "project_density")
        solvers.append(g)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    batch = CondenseBatch(solvers)
    for i, g in enumerate(solvers):
        batch.update_trace[i].fill_(1e-6)
    t0 = time.perf_counter()
    tuned_ms = batch.autotune(reps=2)
    t_tune = time.perf_counter() - t0
    stream = batch.stream

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    steps = max(3, min(args.steps, 20))
    sampler = ClockSampler(0)
    sampler.start()
    cond_ms = timed(batch.condense, steps)
    rec_ms = timed(batch.reconstruct, steps)
    clocks = sampler.stop()
    cells = batch.cells
    # the same devices' work as one launch per device, on a subset
    nsub = min(args.batch_compare, len(solvers))
    sub = solvers[:nsub]
    sub_batch = CondenseBatch(sub)
    sub_batch.autotune(reps=2)
    singles = [CondenseBatch([g]) for g in sub]
    for b in singles:
        b.autotune(reps=1)
    sub_ms = timed(sub_batch.condense, steps)

    def each():
        for b in singles:
            b.condense()

    each_ms = timed(each, steps)
    sub_cells = sum(g.ncells for g in sub)
    # algorithmic FP64 flops of the condensation (LU form on the full cell
    # system) summed over the devices, against the DGEMM rate of this GPU
    flops = sum(algorithmic_flops_per_cell(2, s[3]["k"]) * (s[3]["m"] ** 2) for s in specs)
    peak = fp64_peak_tflops(torch.device("cuda:0"))
    by_k = {}
    for s in specs:
        by_k.setdefault(s[3]["k"], [0, 0])
        by_k[s[3]["k"]][0] += 1
        by_k[s[3]["k"]][1] += s[3]["m"] ** 2
    line = {"metric": "HDG cells condensed/s, batched heterogeneous diodes (one launch per Newton step)",
            "value": cells / ((cond_ms + rec_ms) * 1e-3), "unit": "cells/s", "higher_is_better": True,
            "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3), "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{len(specs)} 2D p-n diodes, cells per side U[16,128], degree U{{1,2,3}}, "
                                   "doping log-U[1e21,1e24] m^-3, junction U[0.3,0.7], seed 2025",
                       "cells": cells, "devices_per_degree": {str(k): v[0] for k, v in sorted(by_k.items())},
                       "cells_per_degree": {str(k): v[1] for k, v in sorted(by_k.items())}},
            "ms_per_step": cond_ms + rec_ms,
            "stages_ms": {"condense": cond_ms, "reconstruct": rec_ms},
            "launches_per_step": 2,
            "autotune": dict(batch.shape(), best_ms=tuned_ms, seconds=t_tune),
            "roofline": {"bound": "fp64", "achieved": flops / (cond_ms * 1e-3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": flops / (cond_ms * 1e-3) / 1e12 / peak,
                         "peak_source": "cuBLAS DGEMM 8192^3 timed in this run",
                         "algorithmic_flops": flops},
            "per_device_launches": {"devices": nsub, "cells": sub_cells, "batched_condense_ms": sub_ms,
                                    "one_launch_per_device_ms": each_ms, "speedup": each_ms / sub_ms},
            "setup_s": t_setup, "clocks": clocks}
    print(json.dumps(line))


def run_trace_solve(args):
    """The global FP64 trace solve alone (ddhdg_solve_condensed: nested-
    dissection multifrontal LU on the device) on the condensed system of the
    256 x 256 degree-2 diode, timed with CUDA events on the solver's stream.
    The first call builds the elimination tree, the second captures the
    numeric sequence in a CUDA graph; both are warm-up."""
    import torch

    from ddhdg_b200 import _lib
    from ddhdg_b200 import workloads as cases
    from ddhdg_b200.solver import NPSolver

    m_side = args.cells_per_side
    pb, prm, adim = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"], length=m_side / WORKLOAD["m"])
    g = NPSolver(pb, prm, adim)
    g.compute_local_charge_neutrality()
    for c in (1, 2):
        _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                             g.trace_state.data_ptr(), g._sp()), "project_density")
    tt, rhs, fl, dv = g.assemble_condense()
    n = g.sizes().n_trace_dofs
    x = torch.zeros(n, dtype=torch.float64, device=g.device)

    def solve():
        _lib.check(g.L.ddhdg_solve_condensed(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(), dv.data_ptr(),
                                             x.data_ptr(), 0, g._sp()), "solve_condensed")

    for _ in range(max(args.warmup, 2)):
        solve()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(g.stream)
    for i in range(args.steps):
        solve()
        ev[i + 1].record(g.stream)
    torch.cuda.synchronize()
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    line = {"metric": "global trace solve ms (nested-dissection multifrontal LU, FP64)",
            "value": float(np.mean(per)), "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "steps": args.steps, "warmup": max(args.warmup, 2), "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2D p-n diode {m_side}x{m_side} quads, HDG degree 2, condensed trace system",
                       "trace_dofs": int(n)},
            "min_ms": float(np.min(per)), "max_ms": float(np.max(per))}
    print(json.dumps(line))


def run_condense_3d(args):
    """The condensation of the 3D diode configuration: 64^3 hexahedra (262 144
    cells), degree 1, step doping along x, ohmic x contacts, SRH, 0.6 V.  The
    FP64 kernel and the mixed one (FP32 Jacobian, FP64 residuals) on the same
    state, each timed with CUDA events; the mixed result's largest deviation
    from the FP64 one is reported relative to the largest FP64 magnitude of
    each output.  (The full Newton solve of this size is out of reach of the
    dense nested-dissection fronts: the top separators hold 49 152 dofs.)"""
    import torch

    from ddhdg_b200 import _lib
    from ddhdg_b200 import workloads as cases
    from ddhdg_b200.solver import NPSolver

    m_side = args.cells_per_side if args.cells_per_side != WORKLOAD["m"] else 64
    out, timing = {}, {}
    state = None
    for prec in (0, 1):
        pb, prm, adim = cases.diode(dim=3, m=m_side, k=1, bias=0.6, precision=prec)
        g = NPSolver(pb, prm, adim)
        if state is None:
            g.compute_local_charge_neutrality()
            for c in (1, 2):
                _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                                     g.trace_state.data_ptr(), g._sp()), "project_density")
            state = (g.get_cell_state(), g.get_trace_state())
        else:
            g.set_state(*state)
        Nt = g.sizes().Nt
        tt = torch.empty(g.ncells * Nt * Nt, dtype=torch.float64, device=g.device)
        rhs = torch.empty(g.ncells * Nt, dtype=torch.float64, device=g.device)
        fl = torch.empty(g.ncells * Nt, dtype=torch.int32, device=g.device)
        dv = torch.empty(g.ncells * Nt, dtype=torch.float64, device=g.device)
        torch.cuda.synchronize()

        def condense():
            _lib.check(g.L.ddhdg_assemble_condense(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(), 0,
                                                   tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(), dv.data_ptr(),
                                                   g._sp()), "condense")

        for _ in range(max(args.warmup, 3)):
            condense()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        steps = min(args.steps, 20)
        e0.record(g.stream)
        for _ in range(steps):
            condense()
        e1.record(g.stream)
        torch.cuda.synchronize()
        timing[prec] = e0.elapsed_time(e1) / steps
        out[prec] = (tt, rhs)
        ncells = g.ncells
        del g, fl, dv
        torch.cuda.empty_cache()
    (t64, r64), (t32, r32) = out[0], out[1]
    e_tt = float((t32 - t64).abs().max() / t64.abs().max())
    e_rhs = float((r32 - r64).abs().max() / r64.abs().max())
    line = {"metric": "HDG cells condensed/s, 3D diode (FP64 and mixed precision)",
            "value": ncells / (timing[1] * 1e-3), "unit": "cells/s", "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32 Jacobian / f64 residual", "data": "synthetic",
            "config": {"workload": f"3D p-n diode {m_side}^3 hexahedra, HDG degree 1, 0.6 V, SRH",
                       "cells": ncells},
            "condense_ms": {"fp64": timing[0], "mixed": timing[1]},
            "cells_per_s": {"fp64": ncells / (timing[0] * 1e-3), "mixed": ncells / (timing[1] * 1e-3)},
            "mixed_vs_fp64_rel_diff": {"tt": e_tt, "rhs": e_rhs}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the short serving stream and the 64-diode batch of the default line")
    ap.add_argument("--serve", action="store_true",
                    help="serve a seeded Poisson stream of diode solves and report p50/p99 latency")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=4.0, help="arrivals per second")
    ap.add_argument("--serve-precision", choices=("mixed", "fp64"), default="mixed",
                    help="condensation precision of the served solves")
    ap.add_argument("--serve-3d-min", type=int, default=16)
    ap.add_argument("--serve-3d-max", type=int, default=32,
                    help="largest 3D mesh of the stream (the nested-dissection fronts grow as m^4.1 in 3D)")
    ap.add_argument("--bias-sweep", action="store_true",
                    help="time the warm-started 0..0.8 V sweep (17 points) instead of the step")
    ap.add_argument("--mixed", action="store_true",
                    help="with --bias-sweep: the same sweep with the mixed-precision condensation, compared point by point")
    ap.add_argument("--trace-solve", action="store_true",
                    help="time the global trace solve alone (nested dissection) on the diode's condensed system")
    ap.add_argument("--condense-3d", action="store_true",
                    help="condensation of the 3D 64^3 degree-1 diode at 0.6 V, FP64 and mixed")
    ap.add_argument("--batch", action="store_true",
                    help="batched heterogeneous diodes: one persistent condensation launch per Newton step")
    ap.add_argument("--batch-devices", type=int, default=512)
    ap.add_argument("--batch-compare", type=int, default=64,
                    help="devices of the one-launch-per-device comparison")
    ap.add_argument("--cells-per-side", type=int, default=WORKLOAD["m"],
                    help="smaller meshes of the same diode for profiling runs")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.bias_sweep:
        return run_bias_sweep(args)
    if args.serve:
        return run_serve(args)
    if args.trace_solve:
        return run_trace_solve(args)
    if args.condense_3d:
        return run_condense_3d(args)
    if args.batch:
        return run_batch(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)

    from ddhdg_b200 import build as _b

    _b.build()
    from ddhdg_b200.solver import NPSolver
    from ddhdg_b200 import _lib
    from ddhdg_b200 import replicas
    from ddhdg_b200 import workloads as cases

    m_side = args.cells_per_side
    pb, prm, adim = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"],
                                length=m_side / WORKLOAD["m"])
    g = NPSolver(pb, prm, adim, device=str(dev))
    g.compute_local_charge_neutrality()
    for c in (1, 2):
        _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                             g.trace_state.data_ptr(), g._sp()), "project_density")
    torch.cuda.synchronize()
    s = g.sizes()
    nc, Nt = g.ncells, s.Nt
    stream = g.stream
    tt = torch.empty(nc * Nt * Nt, dtype=torch.float64, device=dev)
    rhs = torch.empty(nc * Nt, dtype=torch.float64, device=dev)
    dflag = torch.empty(nc * Nt, dtype=torch.int32, device=dev)
    dval = torch.empty(nc * Nt, dtype=torch.float64, device=dev)
    dtrace = (1e-6 * torch.ones(g.nfaces * 3 * g.nf, dtype=torch.float64, device=dev))
    dcell = torch.empty(nc * g.Nc_all, dtype=torch.float64, device=dev)
    L = g.L
    sp = g._sp()

    def condense():
        _lib.check(L.ddhdg_assemble_condense(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(), 0,
                                             tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(), dval.data_ptr(),
                                             sp), "condense")

    def reconstruct():
        _lib.check(L.ddhdg_reconstruct(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(),
                                       dtrace.data_ptr(), dcell.data_ptr(), 0, sp), "reconstruct")

    for _ in range(max(args.warmup, 3)):
        condense()
        reconstruct()
    torch.cuda.synchronize()

    # ---- device-resident timing (inputs in HBM; per-step traffic > L2)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps + 2)]
    sampler = ClockSampler(local)
    replicas.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    ev[0].record(stream)
    for i in range(args.steps):
        ev[1 + 3 * i].record(stream)
        condense()
        ev[2 + 3 * i].record(stream)
        reconstruct()
        ev[3 + 3 * i].record(stream)
    ev[-1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = ev[0].elapsed_time(ev[-1])
    cond_ms = [ev[1 + 3 * i].elapsed_time(ev[2 + 3 * i]) for i in range(args.steps)]
    rec_ms = [ev[2 + 3 * i].elapsed_time(ev[3 + 3 * i]) for i in range(args.steps)]
    total_ms = replicas.max_over_ranks(total_ms, dev)
    ms_per_step = total_ms / args.steps
    value = replicas.job_throughput(nc, ms_per_step)

    # ---- end to end through the C ABI with host buffers
    pin_cell = torch.empty(nc * g.Nc_all, dtype=torch.float64).pin_memory()
    pin_trace = torch.empty(g.nfaces * 3 * g.nf, dtype=torch.float64).pin_memory()
    pin_dtrace = torch.empty(g.nfaces * 3 * g.nf, dtype=torch.float64).pin_memory()
    pin_out = torch.empty(nc * g.Nc_all, dtype=torch.float64).pin_memory()
    pin_cell.copy_(g.cell_state.cpu())
    pin_trace.copy_(g.trace_state.cpu())
    pin_dtrace.copy_(dtrace.cpu())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h2d = (pin_cell.numel() + pin_trace.numel() + pin_dtrace.numel()) * 8
    d2h = pin_out.numel() * 8

    def e2e_step():
        # the host-buffer entry points: the state is read from and the cell
        # update written to pinned host memory by the calls themselves, the
        # copies overlapping the kernels chunk by chunk
        _lib.check(L.ddhdg_assemble_condense_host(g._ctx, pin_cell.data_ptr(), pin_trace.data_ptr(), 0,
                                                  tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(),
                                                  dval.data_ptr(), sp), "condense (host buffers)")
        _lib.check(L.ddhdg_reconstruct_host(g._ctx, pin_dtrace.data_ptr(), 0, pin_out.data_ptr(), sp),
                   "reconstruct (host buffers)")

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    replicas.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1), dev) / args.steps
    e2e_value = replicas.job_throughput(nc, e2e_ms)

    # ---- the mixed-precision condensation (FP32 Jacobian, FP64 residuals)
    # on the same diode and state, timed the same way
    mixed = None
    if 3 * (WORKLOAD["k"] + 1) ** WORKLOAD["dim"] <= 32:
        pbm, prmm, adimm = cases.diode(dim=WORKLOAD["dim"], m=m_side, k=WORKLOAD["k"],
                                       length=m_side / WORKLOAD["m"], precision=1)
        gm = NPSolver(pbm, prmm, adimm, device=str(dev))
        gm.set_state(g.get_cell_state(), g.get_trace_state())
        spm = gm._sp()

        def condense_m():
            _lib.check(L.ddhdg_assemble_condense(gm._ctx, gm.cell_state.data_ptr(), gm.trace_state.data_ptr(),
                                                 0, tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(),
                                                 dval.data_ptr(), spm), "condense (mixed)")

        def reconstruct_m():
            _lib.check(L.ddhdg_reconstruct(gm._ctx, gm.cell_state.data_ptr(), gm.trace_state.data_ptr(),
                                           dtrace.data_ptr(), dcell.data_ptr(), 0, spm), "reconstruct (mixed)")

        for _ in range(max(args.warmup, 3)):
            condense_m()
            reconstruct_m()
        torch.cuda.synchronize()
        evm = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
        replicas.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            evm[3 * i].record(gm.stream)
            condense_m()
            evm[3 * i + 1].record(gm.stream)
            reconstruct_m()
            evm[3 * i + 2].record(gm.stream)
        torch.cuda.synchronize()
        cm = float(np.mean([evm[3 * i].elapsed_time(evm[3 * i + 1]) for i in range(args.steps)]))
        rm = float(np.mean([evm[3 * i + 1].elapsed_time(evm[3 * i + 2]) for i in range(args.steps)]))
        cm = replicas.max_over_ranks(cm, dev)
        mixed = {"condense_ms": cm, "reconstruct_ms": rm,
                 "cells_per_s": replicas.job_throughput(nc, cm + rm),
                 "condense_speedup_vs_fp64": float(np.mean(cond_ms)) / cm,
                 "kernel": "condense3_kernel<2,2,float>",
                 "precision": "FP32 Jacobian (local operators, Gauss-Jordan, Y, Schur operands; "
                              "FP64 accumulation of the products), FP64 residuals, FP64 outputs"}

        # the same mixed-precision device through the batched launch (one
        # persistent launch per stage, graph replay, tiles autotuned)
        from ddhdg_b200.batch import CondenseBatch

        bm = CondenseBatch([gm])
        bm.update_trace[0].copy_(dtrace)
        bm.autotune(reps=2)
        for _ in range(max(args.warmup, 3)):
            bm.condense()
            bm.reconstruct()
        torch.cuda.synchronize()
        evb = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
        replicas.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            evb[3 * i].record(bm.stream)
            bm.condense()
            evb[3 * i + 1].record(bm.stream)
            bm.reconstruct()
            evb[3 * i + 2].record(bm.stream)
        torch.cuda.synchronize()
        cb = float(np.mean([evb[3 * i].elapsed_time(evb[3 * i + 1]) for i in range(args.steps)]))
        rb = float(np.mean([evb[3 * i + 1].elapsed_time(evb[3 * i + 2]) for i in range(args.steps)]))
        cb = replicas.max_over_ranks(cb, dev)
        mixed["batched"] = {"condense_ms": cb, "reconstruct_ms": rb, "cells_per_s": replicas.job_throughput(nc, cb + rb),
                            "shape": bm.shape(), "kernel": "batch_condense_kernel<2> (mixed job)"}
        bm.close()
        del bm, gm
        torch.cuda.empty_cache()

    # ---- the plain FP64 GPU path (the reference's per-cell algorithm as
    # written: full local system, LU of cc per cell, Schur complement; the
    # reconstruction assembles the cell systems again and solves them) on
    # the same state
    psteps = max(3, min(args.steps, 20))

    def condense_p():
        _lib.check(L.ddhdg_assemble_condense_plain(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(), 0,
                                                   tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(),
                                                   dval.data_ptr(), sp), "condense (plain)")

    def reconstruct_p():
        _lib.check(L.ddhdg_reconstruct_plain(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(),
                                             dtrace.data_ptr(), dcell.data_ptr(), 0, sp), "reconstruct (plain)")

    for _ in range(max(args.warmup, 3)):
        condense_p()
        reconstruct_p()
    torch.cuda.synchronize()
    evp = [torch.cuda.Event(enable_timing=True) for _ in range(3 * psteps)]
    replicas.barrier()
    torch.cuda.synchronize()
    for i in range(psteps):
        evp[3 * i].record(stream)
        condense_p()
        evp[3 * i + 1].record(stream)
        reconstruct_p()
        evp[3 * i + 2].record(stream)
    torch.cuda.synchronize()
    pc = replicas.max_over_ranks(float(np.mean([evp[3 * i].elapsed_time(evp[3 * i + 1]) for i in range(psteps)])), dev)
    pr = replicas.max_over_ranks(float(np.mean([evp[3 * i + 1].elapsed_time(evp[3 * i + 2]) for i in range(psteps)])), dev)
    plain = {"condense_ms": pc, "reconstruct_ms": pr, "steps": psteps,
             "cells_per_s": replicas.job_throughput(nc, pc + pr),
             "kernel": "plain_kernel<2,2> (81x81 cell system assembled term by term, row-equilibrated LU "
                       "with partial pivoting, Schur complement; reconstruction: second assembly + solve)"}

    # ---- one whole Newton step (BASELINE's second metric): assembly +
    # condensation, nested-dissection trace solve, reconstruction, norms and
    # update, state on the device.  The consistent Jacobian keeps the
    # iterates finite from this start; the kernels' cost is the same.
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    gn = NPSolver(pb, prm, adim, device=str(dev))
    gn.set_state(g.get_cell_state(), g.get_trace_state())
    gn.private_run(0.0, 0.0, 2)  # builds the elimination tree, then captures the solve graph
    torch.cuda.synchronize()
    newton_steps = 3
    gn.set_state(g.get_cell_state(), g.get_trace_state())
    replicas.barrier()
    en0, en1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    en0.record(gn.stream)
    gn.private_run(0.0, 0.0, newton_steps)
    en1.record(gn.stream)
    torch.cuda.synchronize()
    nt = gn.last_timings()
    newton = {"ms": replicas.max_over_ranks(en0.elapsed_time(en1), dev) / newton_steps,
              "steps": newton_steps,
              "stages_ms": {"assemble_condense": nt["condense_ms"] / nt["steps"],
                            "trace_solve": nt["solve_ms"] / nt["steps"],
                            "reconstruct": nt["reconstruct_ms"] / nt["steps"]},
              "trace_dofs": int(gn.sizes().n_trace_dofs),
              "solver": "nested-dissection multifrontal LU on the device (FP64)"}
    del gn
    torch.cuda.empty_cache()

    # ---- the target comparison: condensation per Newton step of the
    # mixed-precision and FP64 block-eliminated paths against the plain FP64
    # GPU path, and the whole Newton step (the trace solve is the same in all)
    fp64_c = float(np.mean(cond_ms))
    fp64_r = float(np.mean(rec_ms))
    solve_ms = newton["stages_ms"]["trace_solve"]
    target = {"condense_ms": {"plain_fp64": pc, "fp64": fp64_c},
              "condense_speedup_vs_plain": {"fp64": pc / fp64_c},
              "newton_step_ms": {"plain_fp64": pc + solve_ms + pr, "fp64": fp64_c + solve_ms + fp64_r},
              "note": "Newton-step figures add the measured trace solve (same solver in every path) to each "
                      "path's measured condense and reconstruct times"}
    if mixed is not None:
        target["condense_ms"]["mixed"] = mixed["condense_ms"]
        target["condense_speedup_vs_plain"]["mixed"] = pc / mixed["condense_ms"]
        target["newton_step_ms"]["mixed"] = mixed["condense_ms"] + solve_ms + mixed["reconstruct_ms"]
        mb = mixed["batched"]
        target["condense_ms"]["batched_mixed"] = mb["condense_ms"]
        target["condense_speedup_vs_plain"]["batched_mixed"] = pc / mb["condense_ms"]
        target["newton_step_ms"]["batched_mixed"] = mb["condense_ms"] + solve_ms + mb["reconstruct_ms"]
    base = target["newton_step_ms"]["plain_fp64"]
    target["newton_step_speedup_vs_plain"] = {k: base / v for k, v in target["newton_step_ms"].items()
                                              if k != "plain_fp64"}

    # ---- a short seeded serving stream (continuous batching of diode
    # solves): p50 / p99 latency and solves/s
    serve = None
    if world == 1 and not args.no_serve:
        serve = serve_quick()
    batchq = batch_quick() if world == 1 and not args.no_serve else None

    fp64_peak = fp64_peak_tflops(dev)
    if rank == 0:
        hbm_peak, peak_kind = peaks()
        bc, br = bytes_per_cell(WORKLOAD["dim"], WORKLOAD["k"])
        fa = algorithmic_flops_per_cell(WORKLOAD["dim"], WORKLOAD["k"])
        fc = flops_per_cell(WORKLOAD["dim"], WORKLOAD["k"])
        cond_avg = float(np.mean(cond_ms))
        achieved = fa * nc / (cond_avg * 1e-3) / 1e12
        executed = fc * nc / (cond_avg * 1e-3) / 1e12
        hbm_achieved = bc * nc / (cond_avg * 1e-3) / 1e9
        line = {
            "metric": "HDG cells condensed/s (assemble+condense+reconstruct)",
            "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2D p-n diode {m_side}x{m_side} quads (cell size 1/256 um), HDG degree 2, FP64, "
                                   "block-eliminated condensation (the plain FP64 path is the `plain` key)",
                       "cells": nc, "trace_dofs_per_cell": Nt,
                       "parallelism": f"replicas x{world}",
                       "l2": "per-step traffic (>1.2 GB) exceeds the 126 MB L2"},
            "stages_ms": {"condense": cond_avg, "reconstruct": float(np.mean(rec_ms))},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp64_peak,
                         "traffic": (tbc * nc) if (tbc := traffic_bytes_per_cell()) else None,
                         "kernel": "condense3_kernel<2,2>",
                         "peak_source": "cuBLAS DGEMM 8192^3 timed in this run",
                         "algorithmic_flops_per_cell": fa,
                         "executed": {"flops_per_cell": fc, "tflops": executed,
                                      "frac": executed / fp64_peak},
                         "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                                 "frac": hbm_achieved / hbm_peak, "peak_source": peak_kind,
                                 "algorithmic_bytes_per_cell": bc}},
            "e2e": {"value": e2e_value, "unit": "cells/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "newton_step": newton,
            "mixed": mixed,
            "plain": plain,
            "target": target,
            "serve": serve,
            "batch": batchq,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
