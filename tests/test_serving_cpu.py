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
