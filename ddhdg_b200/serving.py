"""Serving: a request loop for diode solves of different sizes.

Requests (a diode's dimension, mesh, degree and bias) arrive over time.  The
server admits a request as soon as an in-flight slot and enough free device
memory are available, and keeps its Newton state on the device for the whole
solve.  ``DiodeServer`` batches at kernel level, step by step: every request
in flight advances one Newton step per server step, the assembly and
condensation of all requests in the same phase run as ONE batched launch
(``ddhdg_batch_newton_step``), their trace solves overlap on side streams,
and the reconstruction is one more launch; requests join at the next step
after they arrive and leave when they converge (continuous batching).
``ThreadedDiodeServer`` is the simpler form: one host thread, context and
stream per request, overlapping only on the device.  Results do not depend on
what else runs: every kernel is deterministic (no atomics with more than two
contributions, no order-dependent reductions) and a device's results in a
batched launch are bitwise those of its own launch, so a request's fields
are the same alone and in the mix.

A solve is: thermodynamic equilibrium (charge-neutral first guess, V-only
Newton, density projection), then, for a nonzero bias, the contact
conditions for that bias and the Newton solve warm-started from equilibrium.
The consistent Jacobian is used (the reference's diverges on these diodes).
"""

from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    dim: int
    m: int          # cells per side
    k: int          # degree
    bias: float     # volts on the p contact
    arrival: float  # seconds after the start of the run


@dataclass
class Result:
    rid: int
    arrival: float
    start: float
    finish: float
    iterations: int
    converged: bool
    cells: int
    state: tuple = field(default=None, repr=False)  # (cell, trace) on the host, if kept

    @property
    def latency(self):
        return self.finish - self.arrival


def trace_solver_bytes(dim: int, m: int, k: int, ncomp: int) -> int:
    """Device bytes of the nested-dissection trace solver of an m^dim mesh
    at degree k with `ncomp` enabled components, from the solver's own plan
    (``ddhdg_trace_solver_bytes``: host only; the plan is cached and reused
    by the solver that the request builds)."""
    import ctypes

    from . import _lib

    L = _lib.load()
    n = (ctypes.c_int * 3)(m, m, m)
    out = ctypes.c_int64()
    _lib.check(L.ddhdg_trace_solver_bytes(int(dim), n, int(k), int(ncomp), ctypes.byref(out)),
               "trace_solver_bytes")
    return int(out.value)


# Device bytes of one request beyond its arrays and its trace solver (whose
# library handles trace_solver_bytes counts): CUDA graphs, the context's and
# the batch's streams and events
REQUEST_OVERHEAD = 256 << 20


def memory_estimate(dim: int, m: int, k: int) -> int:
    """Device bytes of one solve: the larger of the two phases' trace
    solvers (the V-only equilibrium system's is released before the biased
    system's is built) from their plans, the global trace sparsity,
    the per-cell states, condensed blocks and Y cache of both phases, and the
    per-request overhead; the array terms 10 % over."""
    nb = (k + 1) ** dim
    nf = (k + 1) ** (dim - 1)
    cells = m ** dim
    Nt = 2 * dim * 3 * nf
    Ns = 3 * nb
    nd = 3 * nf
    per_cell = 8 * (3 * (dim + 1) * nb * 3 + Nt * Nt + 3 * Nt + Ns * (1 + Nt))
    # the batched launch keeps its own Y cache of the request's cells
    batch_y = 8 * Ns * (1 + Nt)
    fronts = max(trace_solver_bytes(dim, m, k, 3), trace_solver_bytes(dim, m, k, 1))
    # the global trace sparsity of both modes (values, column indices and
    # the permutation maps: about 20 bytes per nonzero; a face couples to
    # the 4 dim - 1 faces of its two cells)
    faces = dim * (m + 1) * m ** (dim - 1)
    csr = 20 * faces * nd * nd * (4 * dim - 1) * (1.0 + 1.0 / 9.0)
    return int(1.1 * ((2 * per_cell + batch_y) * cells + fronts + csr)) + REQUEST_OVERHEAD


def poisson_requests(n: int, rate: float, seed: int, sizes_2d=(32, 256), sizes_3d=(8, 16),
                     degrees=(1, 2), frac_3d=0.25, bias=(0.0, 0.8)) -> list:
    """n requests with exponential inter-arrival times (rate per second),
    2D meshes uniform in sizes_2d, 3D meshes uniform in sizes_3d (degree 1),
    degrees uniform in `degrees`, biases uniform in `bias`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if rng.random() < frac_3d:
            dim, k = 3, 1
            m = int(rng.integers(sizes_3d[0], sizes_3d[1] + 1))
        else:
            dim = 2
            m = int(rng.integers(sizes_2d[0], sizes_2d[1] + 1))
            k = int(rng.choice(degrees))
        out.append(Request(i, dim, m, k, float(rng.uniform(*bias)), t))
    return out


def request_precision(req: Request, mixed: bool) -> int:
    """The context precision of a request: 1 (FP32 Jacobian, FP64 residuals)
    when `mixed` and its degree has a mixed-precision kernel
    (3 (k+1)^dim <= 32), else 0 (FP64)."""
    return 1 if mixed and 3 * (req.k + 1) ** req.dim <= 32 else 0


def solve_one(req: Request, device="cuda:0", keep_state=False, tol=1e-10, max_it=50, mixed=False):
    """One request's solve on the calling thread's current CUDA stream."""
    from . import _lib, workloads
    from .solver import NPSolver

    pb, prm, adim = workloads.diode(dim=req.dim, m=req.m, k=req.k, precision=request_precision(req, mixed))
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    g = NPSolver(pb, prm, adim, device=device)
    res = g.compute_thermodynamic_equilibrium()
    it = res.iterations
    # the equilibrium system's trace solver is not used again
    _lib.check(g.L.ddhdg_release_solver(g._ctx, 1), "release_solver")
    if req.bias != 0.0:
        workloads.set_bias(pb, req.bias)
        g.update_boundary_tables()
        res = g.run(tol, tol, max_it)
        it += res.iterations
    state = (g.get_cell_state().copy(), g.get_trace_state().copy()) if keep_state else None
    return res.converged, it, g.ncells, state


class ThreadedDiodeServer:
    """Concurrent diode solves on one GPU, one host thread per request.

    max_inflight: requests on the device at once (slots).
    hbm_reserve: bytes of device memory left free for everything else.
    hbm_limit: treat the device as having at most this many bytes (tests).
    mem_info: callable returning (free, total) device bytes; defaults to
    cudaMemGetInfo of `device`.
    mixed: condense with the FP32 Jacobian and FP64 residuals where the
    request's degree has that kernel (the Newton loop converges to the FP64
    solution)."""

    def __init__(self, max_inflight=8, hbm_reserve=4 << 30, hbm_limit=None, device="cuda:0",
                 keep_states=False, mem_info=None, mixed=False):
        self.mixed = mixed
        self.max_inflight = max_inflight
        self.hbm_reserve = hbm_reserve
        self.hbm_limit = hbm_limit
        self.device = device
        self.keep_states = keep_states
        self.mem_info = mem_info
        self.peak_inflight = 0
        self.peak_committed = 0  # largest sum of the in-flight requests' memory estimates
        self._used_at_start = 0

    def _mem_info(self):
        if self.mem_info is not None:
            return self.mem_info()
        import torch

        return torch.cuda.mem_get_info(self.device)

    def _start_accounting(self):
        """Device bytes in use before any request runs (other users of the
        device, this process's own caches)."""
        free, total = self._mem_info()
        self._used_at_start = total - free

    def _free_bytes(self, committed):
        """Bytes a new request may take.  A request that has been admitted
        may not have allocated its buffers yet, so the live free figure alone
        would let a burst of arrivals pass the check against the same memory:
        the estimates of all requests in flight are subtracted from what was
        free when the run started, and the live figure only lowers that."""
        free, total = self._mem_info()
        cap = total - self._used_at_start
        if self.hbm_limit is not None:
            cap = min(cap, self.hbm_limit)
        return min(free, cap - committed) - self.hbm_reserve

    def admissible(self, est, committed):
        """Whether a request of `est` bytes fits next to `committed` bytes of
        requests in flight."""
        return est <= self._free_bytes(committed)

    def run(self, requests):
        """Serve the requests (sorted by arrival time); returns their
        results in request order.  Arrival times are honoured in wall-clock
        time from the start of the call."""
        import torch

        reqs = sorted(requests, key=lambda r: r.arrival)
        results = {}
        lock = threading.Lock()
        done = threading.Condition(lock)
        inflight = {}      # rid -> estimated bytes
        committed = [0]
        errors = []
        self._start_accounting()
        t0 = time.perf_counter()

        def worker(req, est, start):
            try:
                stream = torch.cuda.Stream(device=self.device)
                with torch.cuda.stream(stream):
                    conv, it, cells, state = solve_one(req, self.device, self.keep_states, mixed=self.mixed)
                    stream.synchronize()
                finish = time.perf_counter() - t0
                res = Result(req.rid, req.arrival, start, finish, it, conv, cells, state)
            except Exception as e:  # reported after the run
                res = None
                errors.append((req.rid, repr(e)))
            with lock:
                if res is not None:
                    results[req.rid] = res
                committed[0] -= est
                del inflight[req.rid]
                done.notify_all()

        threads = []
        i = 0
        while i < len(reqs):
            req = reqs[i]
            now = time.perf_counter() - t0
            if now < req.arrival:
                time.sleep(min(req.arrival - now, 0.05))
                continue
            est = memory_estimate(req.dim, req.m, req.k)
            with lock:
                while inflight and (len(inflight) >= self.max_inflight or
                                    not self.admissible(est, committed[0])):
                    done.wait(timeout=0.05)
                if not inflight and not self.admissible(est, committed[0]):
                    errors.append((req.rid, "does not fit in device memory"))
                    i += 1
                    continue
                inflight[req.rid] = est
                committed[0] += est
                self.peak_inflight = max(self.peak_inflight, len(inflight))
                self.peak_committed = max(self.peak_committed, committed[0])
            start = time.perf_counter() - t0
            th = threading.Thread(target=worker, args=(req, est, start), daemon=True)
            th.start()
            threads.append(th)
            i += 1
        for th in threads:
            th.join()
        if errors:
            raise RuntimeError(f"requests failed: {errors}")
        return [results[r.rid] for r in requests]


def latency_stats(results, wall):
    lat = np.array([r.latency for r in results])
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "solves_per_s": len(results) / wall,
            "cells_per_s": sum(r.cells for r in results) / wall,
            "converged": int(sum(r.converged for r in results)), "requests": len(results)}


class _Active:
    """A request in flight: its solver, phase and per-phase batch buffers."""

    def __init__(self, req, est, start):
        self.req, self.est, self.start = req, est, start
        self.solver = None
        self.phase = "eq"  # thermodynamic equilibrium, then the biased solve
        self.it = 0        # iterations of the current phase
        self.total_it = 0
        self.buffers = {}


class DiodeServer(ThreadedDiodeServer):
    """Continuous batching of diode solves on one GPU, at kernel level.

    Every server step advances each request in flight by one Newton step:
    one batched condensation launch over all requests of a phase, their trace
    solves overlapped on side streams, one batched reconstruction launch and
    the damped updates (``CondenseBatch.newton_step``).  The loop is
    ``private_run`` (src/np_solver.cpp:1452-1561) per request: the stopping
    rule on the update and state norms and the damping are the solver's.
    Arrivals join at the next step once a slot and their device memory are
    free; converged requests leave.  Memory admission as in
    ``ThreadedDiodeServer``."""

    def __init__(self, max_inflight=16, hbm_reserve=4 << 30, hbm_limit=None, device="cuda:0",
                 keep_states=False, mem_info=None, tol=1e-10, max_it=50, mixed=False):
        super().__init__(max_inflight, hbm_reserve, hbm_limit, device, keep_states, mem_info, mixed)
        self.tol = tol
        self.max_it = max_it
        self.steps = 0
        self.peak_batch = 0

    def _start_request(self, a):
        from . import workloads
        from .solver import NPSolver

        req = a.req
        pb, prm, adim = workloads.diode(dim=req.dim, m=req.m, k=req.k,
                                        precision=request_precision(req, self.mixed))
        prm.consistent_drift_jacobian = True
        prm.consistent_recombination_jacobian = True
        g = NPSolver(pb, prm, adim, device=self.device)
        g.compute_local_charge_neutrality()
        a.solver, a.problem = g, pb
        nl = prm.nonlinear_parameters
        a.eq_tol = (nl.absolute_tolerance, nl.relative_tolerance, nl.max_number_of_iterations)
        a.alpha = nl.alpha

    def _finish_phase(self, a):
        """Equilibrium done: densities from the equilibrium potential, then
        the contact conditions of the bias (or the end of the solve)."""
        from . import _lib, workloads

        g = a.solver
        a.total_it += a.it
        a.it = 0
        if a.phase == "eq":
            for c in (1, 2):
                _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                                     g.trace_state.data_ptr(), g._sp()), "project_density")
            # the equilibrium system's trace solver is not used again: its
            # fronts go back before the biased system's solver is built
            _lib.check(g.L.ddhdg_release_solver(g._ctx, 1), "release_solver")
            if a.req.bias != 0.0:
                workloads.set_bias(a.problem, a.req.bias)
                g.update_boundary_tables()
                a.phase = "bias"
                return False
        return True

    def run(self, requests):
        import torch

        from .batch import CondenseBatch

        reqs = sorted(requests, key=lambda r: r.arrival)
        results, errors = {}, []
        active = []
        committed = 0
        batches = {}  # (phase, dim) -> (member ids, CondenseBatch)
        self._start_accounting()
        t0 = time.perf_counter()
        i = 0
        while i < len(reqs) or active:
            now = time.perf_counter() - t0
            # admission at the step boundary
            while i < len(reqs) and reqs[i].arrival <= now and len(active) < self.max_inflight:
                req = reqs[i]
                est = memory_estimate(req.dim, req.m, req.k)
                if not self.admissible(est, committed):
                    if not active:
                        errors.append((req.rid, "does not fit in device memory"))
                        i += 1
                        continue
                    break
                a = _Active(req, est, time.perf_counter() - t0)
                self._start_request(a)
                active.append(a)
                committed += est
                i += 1
                self.peak_inflight = max(self.peak_inflight, len(active))
                self.peak_committed = max(self.peak_committed, committed)
            if not active:
                if i < len(reqs):
                    time.sleep(max(0.0, min(reqs[i].arrival - (time.perf_counter() - t0), 0.05)))
                continue
            self.steps += 1
            done = []
            # one batch per (phase, dimension): a batched launch holds
            # devices of one dimension and one mode
            groups = {}
            for a in active:
                groups.setdefault((a.phase, a.req.dim), []).append(a)
            for bk in sorted(groups):
                phase, group = bk[0], groups[bk]
                key = tuple(id(a) for a in group)
                if bk not in batches or batches[bk][0] != key:
                    if bk in batches:
                        batches[bk][1].close()
                    bufs = []
                    for a in group:
                        if phase not in a.buffers:
                            a.buffers[phase] = CondenseBatch.buffers_for(a.solver, thermo=(phase == "eq"))
                        bufs.append(a.buffers[phase])
                    batches[bk] = (key, CondenseBatch([a.solver for a in group], thermo=(phase == "eq"),
                                                      buffers=bufs))
                self.peak_batch = max(self.peak_batch, len(group))
                norms, status = batches[bk][1].newton_step([a.alpha for a in group])
                for a, nrm, st in zip(group, norms, status):
                    a.it += 1
                    upd, cur = max(nrm[0], nrm[1]), max(nrm[2], nrm[3])
                    abs_tol, rel_tol, max_it = a.eq_tol if phase == "eq" else (self.tol, self.tol, self.max_it)
                    if st or not math.isfinite(upd):
                        errors.append((a.req.rid, f"Newton failed in phase {phase} (status {st})"))
                        done.append((a, False))
                    elif upd < abs_tol or upd < rel_tol * cur:
                        if self._finish_phase(a):
                            done.append((a, True))
                    elif a.it >= max_it:
                        a.total_it += a.it
                        done.append((a, False))
            for a, conv in done:
                active.remove(a)
                committed -= a.est
                g = a.solver
                torch.cuda.synchronize(self.device)
                finish = time.perf_counter() - t0
                state = (g.get_cell_state().copy(), g.get_trace_state().copy()) if self.keep_states else None
                results[a.req.rid] = Result(a.req.rid, a.req.arrival, a.start, finish, a.total_it, conv,
                                            g.ncells, state)
                a.solver = None
                a.buffers = {}
            if done:
                # the batches held the finished requests' buffers; hand the
                # memory back to the device (the trace solver allocates
                # outside torch's cache)
                for bk in [bk for bk, (key, _) in batches.items() if any(id(a) in key for a, _ in done)]:
                    batches.pop(bk)[1].close()
                torch.cuda.empty_cache()
        for _, b in batches.values():
            b.close()
        if errors:
            raise RuntimeError(f"requests failed: {errors}")
        return [results[r.rid] for r in requests]
