"""Serving: a request loop for diode solves of different sizes.

Requests (a diode's dimension, mesh, degree and bias) arrive over time.  The
server admits a request as soon as an in-flight slot and enough free device
memory are available, and keeps its Newton state on the device for the whole
solve.  ``DiodeServer`` batches at kernel level: the requests in flight form
groups by (phase, dimension, size class), and a group advances all its
requests by one Newton step at a time, their assembly and condensation as
ONE batched launch (``ddhdg_batch_newton_step_begin``), their trace solves
overlapped on side streams, and the reconstruction as one more launch.
Groups step independently on their own streams, so small requests are not
held back by large ones; requests join their group at its next step after
they arrive and leave when they converge (continuous batching).
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
    """Device bytes of one solve: the trace solvers of both phases (the
    V-only equilibrium system's is released only when no step is in flight,
    so it may still be held while the biased system's is built) from their
    plans, the global trace sparsity, the per-cell states, condensed blocks
    and Y caches of both phases, and the per-request overhead; the array
    terms 10 % over."""
    nb = (k + 1) ** dim
    nf = (k + 1) ** (dim - 1)
    cells = m ** dim
    Nt = 2 * dim * 3 * nf
    Ns = 3 * nb
    nd = 3 * nf
    per_cell = 8 * (3 * (dim + 1) * nb * 3 + Nt * Nt + 3 * Nt + Ns * (1 + Nt))
    # the batched launch keeps its own Y cache of the request's cells
    batch_y = 8 * Ns * (1 + Nt)
    fronts = trace_solver_bytes(dim, m, k, 3) + trace_solver_bytes(dim, m, k, 1)
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
    from . import workloads
    from .solver import NPSolver

    pb, prm, adim = workloads.diode(dim=req.dim, m=req.m, k=req.k, precision=request_precision(req, mixed))
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    g = NPSolver(pb, prm, adim, device=device)
    res = g.compute_thermodynamic_equilibrium()
    it = res.iterations
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


class _Deferred:
    """Device memory handed back when no step is in flight: a cudaFree
    waits for the whole device, so the server does not free while other
    requests' steps run (unless an arrival needs the memory)."""

    def __init__(self, fn):
        self.fn = fn

    def close(self):
        fn, self.fn = self.fn, None
        if fn is not None:
            fn()


class DiodeServer(ThreadedDiodeServer):
    """Continuous batching of diode solves on one GPU, at kernel level.

    The requests in flight form groups by (phase, dimension, size class);
    each group advances by one Newton step at a time: one batched
    condensation launch over its requests, their trace solves overlapped on
    side streams, one batched reconstruction launch and the damped updates
    (``CondenseBatch.newton_step_begin`` / ``newton_step_end``).  Groups step
    independently, each on its own stream: the host loop begins the step of
    every idle group, then collects the steps that have ended, so a group of
    small requests is not held back by the long trace solves of a group of
    large ones.  The loop is ``private_run`` (src/np_solver.cpp:1452-1561)
    per request: the stopping rule on the update and state norms and the
    damping are the solver's.  Arrivals join their group at its next step
    once a slot and their device memory are free; converged requests leave.
    Memory admission as in ``ThreadedDiodeServer``; memory of finished
    requests and replaced batches goes back when no step is in flight or
    when an arrival needs it.

    big_bytes: requests whose memory estimate exceeds it form their own
    groups (the large class)."""

    def __init__(self, max_inflight=16, hbm_reserve=4 << 30, hbm_limit=None, device="cuda:0",
                 keep_states=False, mem_info=None, tol=1e-10, max_it=50, mixed=False, big_bytes=8 << 30):
        super().__init__(max_inflight, hbm_reserve, hbm_limit, device, keep_states, mem_info, mixed)
        self.tol = tol
        self.max_it = max_it
        self.big_bytes = big_bytes
        self.steps = 0  # group steps
        self.peak_batch = 0
        self._deferred = []

    def _group_key(self, a):
        return (a.phase, a.req.dim, 1 if a.est > self.big_bytes else 0)

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
            # memory goes back with the next deferred release
            self._deferred.append(_Deferred(lambda g=g: _lib.check(g.L.ddhdg_release_solver(g._ctx, 1),
                                                                  "release_solver")))
            if a.req.bias != 0.0:
                workloads.set_bias(a.problem, a.req.bias)
                g.update_boundary_tables()
                a.phase = "bias"
                return False
        return True

    def _release_deferred(self):
        import torch

        while self._deferred:
            self._deferred.pop(0).close()
        torch.cuda.empty_cache()

    def run(self, requests):
        from .batch import CondenseBatch

        reqs = sorted(requests, key=lambda r: r.arrival)
        results, errors = {}, []
        active = []
        committed = 0
        groups = {}  # group key -> {"ids", "batch", "members" of the step in flight or None}
        self._deferred = []
        self._start_accounting()
        t0 = time.perf_counter()
        i = 0
        while i < len(reqs) or active:
            now = time.perf_counter() - t0
            # ---- admission
            while i < len(reqs) and reqs[i].arrival <= now and len(active) < self.max_inflight:
                req = reqs[i]
                est = memory_estimate(req.dim, req.m, req.k)
                if not self.admissible(est, committed) and self._deferred:
                    self._release_deferred()
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
                if self._deferred:
                    self._release_deferred()
                if i < len(reqs):
                    time.sleep(max(0.0, min(reqs[i].arrival - (time.perf_counter() - t0), 0.05)))
                continue
            # ---- begin a step in every idle group (rebuilt when its members changed)
            members_of = {}
            for a in active:
                members_of.setdefault(self._group_key(a), []).append(a)
            for gk, members in members_of.items():
                gs = groups.get(gk)
                if gs is not None and gs["members"] is not None:
                    continue  # its step is running
                ids = tuple(id(a) for a in members)
                thermo = gk[0] == "eq"
                if gs is None or gs["ids"] != ids:
                    if gs is not None:
                        self._deferred.append(gs["batch"])
                    bufs = []
                    for a in members:
                        if gk[0] not in a.buffers:
                            a.buffers[gk[0]] = CondenseBatch.buffers_for(a.solver, thermo=thermo)
                        bufs.append(a.buffers[gk[0]])
                    gs = groups[gk] = {"ids": ids, "members": None,
                                       "batch": CondenseBatch([a.solver for a in members], thermo=thermo,
                                                              buffers=bufs)}
                gs["batch"].newton_step_begin([a.alpha for a in members])
                gs["members"] = members
                self.steps += 1
                self.peak_batch = max(self.peak_batch, len(members))
            for gk in [gk for gk, gs in groups.items() if gs["members"] is None and gk not in members_of]:
                self._deferred.append(groups.pop(gk)["batch"])
            # ---- collect the steps that have ended
            done, progressed = [], False
            for gk, gs in groups.items():
                if gs["members"] is None:
                    continue
                res = gs["batch"].newton_step_end(wait=False)
                if res is None:
                    continue
                progressed = True
                members, gs["members"] = gs["members"], None
                phase = gk[0]
                norms, status = res
                for a, nrm, st in zip(members, norms, status):
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
                finish = time.perf_counter() - t0
                state = (g.get_cell_state().copy(), g.get_trace_state().copy()) if self.keep_states else None
                results[a.req.rid] = Result(a.req.rid, a.req.arrival, a.start, finish, a.total_it, conv,
                                            g.ncells, state)

                def drop(a=a):
                    a.solver = None
                    a.buffers = {}

                self._deferred.append(_Deferred(drop))
            if not progressed:
                if not any(gs["members"] is not None for gs in groups.values()) and self._deferred:
                    self._release_deferred()
                time.sleep(0.0005)
        for gs in groups.values():
            if gs["members"] is not None:
                gs["batch"].newton_step_end(wait=True)
            gs["batch"].close()
        self._release_deferred()
        if errors:
            raise RuntimeError(f"requests failed: {errors}")
        return [results[r.rid] for r in requests]
