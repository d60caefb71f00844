"""Serving admission by device memory, on the host with a fake memory query:
requests admitted but not yet allocated still count against the free memory,
with or without an explicit device-memory cap."""

from ddhdg_b200 import serving

GB = 1 << 30


def test_admission_counts_reservations_that_have_not_allocated_yet():
    # the live query never moves (the admitted requests have not allocated)
    server = serving.DiodeServer(hbm_reserve=0, mem_info=lambda: (10 * GB, 12 * GB))
    server._start_accounting()  # 2 GB in use before the run
    assert server.admissible(6 * GB, 0)
    assert not server.admissible(6 * GB, 6 * GB)  # a burst must not pass twice
    assert server.admissible(4 * GB, 6 * GB)
    assert not server.admissible(5 * GB, 6 * GB)


def test_admission_follows_the_live_figure_when_it_is_lower():
    state = {"free": 10 * GB}
    server = serving.DiodeServer(hbm_reserve=1 * GB, mem_info=lambda: (state["free"], 10 * GB))
    server._start_accounting()
    assert server.admissible(9 * GB, 0)
    state["free"] = 3 * GB  # someone else took memory meanwhile
    assert not server.admissible(3 * GB, 0)
    assert server.admissible(2 * GB, 0)


def test_admission_with_an_explicit_cap():
    server = serving.DiodeServer(hbm_reserve=0, hbm_limit=5 * GB, mem_info=lambda: (80 * GB, 80 * GB))
    server._start_accounting()
    assert server.admissible(5 * GB, 0)
    assert not server.admissible(3 * GB, 3 * GB)
    assert server.admissible(2 * GB, 3 * GB)


def test_estimates_grow_with_the_problem():
    e = serving.memory_estimate
    assert e(2, 64, 2) > e(2, 32, 2) > e(2, 32, 1)
    assert e(3, 16, 1) > e(3, 8, 1)


def test_trace_solver_bytes_come_from_the_plan():
    b3 = serving.trace_solver_bytes(2, 32, 2, 3)
    b1 = serving.trace_solver_bytes(2, 32, 2, 1)
    assert b3 > b1 > 0
    assert serving.trace_solver_bytes(2, 64, 2, 3) > b3
    assert serving.trace_solver_bytes(3, 8, 1, 3) > serving.trace_solver_bytes(3, 6, 1, 3)
    # the estimate holds both modes' solvers
    assert serving.memory_estimate(2, 32, 2) > b3 + b1


def test_groups_step_independently_with_fake_batches(monkeypatch):
    """The batched server's event loop on the host, with fake batches: a
    group of large requests whose steps take longer does not hold back a
    group of small ones, no batch mixes the size classes or the phases, a
    batch never has two steps in flight, every request runs its equilibrium
    then its biased phase, and the deferred releases all happen."""
    import numpy as np

    from ddhdg_b200 import batch as batch_mod

    log, released = [], []

    class FakeSolver:
        def __init__(self, req):
            self.req, self.ncells, self.steps = req, req.m ** req.dim, 0

    class FakeBatch:
        def __init__(self, solvers, thermo=False, buffers=None):
            self.solvers, self.thermo, self.inflight, self.polls = solvers, thermo, False, 0
            log.append((thermo, tuple(s.req.rid for s in solvers)))

        @staticmethod
        def buffers_for(g, thermo=False):
            return {}

        def newton_step_begin(self, alphas):
            assert not self.inflight
            self.inflight, self.polls = True, 0

        def newton_step_end(self, wait=True):
            assert self.inflight
            self.polls += 1
            need = 4 if any(s.req.m > 100 for s in self.solvers) else 1
            if not wait and self.polls < need:
                return None
            self.inflight = False
            norms = []
            for s in self.solvers:
                s.steps += 1
                upd = 10.0 ** (-3 * s.steps)  # below 1e-10 at the fourth step
                norms.append([upd, upd, 1.0, 1.0])
            return np.array(norms), [0] * len(self.solvers)

        def close(self):
            assert not self.inflight

    class FakeServer(serving.DiodeServer):
        def _start_request(self, a):
            a.solver = FakeSolver(a.req)
            a.eq_tol, a.alpha = (1e-10, 1e-10, 50), 1.0

        def _finish_phase(self, a):
            a.total_it += a.it
            a.it = 0
            if a.phase == "eq" and a.req.bias != 0.0:
                a.phase = "bias"
                a.solver.steps = 0
                self._deferred.append(serving._Deferred(lambda rid=a.req.rid: released.append(rid)))
                return False
            return True

    monkeypatch.setattr(batch_mod, "CondenseBatch", FakeBatch)
    monkeypatch.setattr(serving, "memory_estimate", lambda dim, m, k: (10 if m > 100 else 1) * GB)
    reqs = [serving.Request(0, 2, 200, 2, 0.3, 0.0), serving.Request(1, 2, 20, 1, 0.2, 0.0),
            serving.Request(2, 2, 24, 2, 0.0, 0.0), serving.Request(3, 2, 180, 1, 0.5, 0.0)]
    server = FakeServer(max_inflight=8, hbm_reserve=0, mem_info=lambda: (100 * GB, 100 * GB))
    res = server.run(reqs)
    assert all(r.converged for r in res)
    assert [r.iterations for r in res] == [8, 8, 4, 8]
    # the small requests finish first although they arrived together
    assert max(res[1].finish, res[2].finish) < min(res[0].finish, res[3].finish)
    big = {0, 3}
    for thermo, ids in log:
        assert set(ids) <= big or not (set(ids) & big)
    assert sorted(released) == [0, 1, 3]
    assert server.peak_inflight == 4
