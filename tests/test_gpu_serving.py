"""Serving (continuous batching of diode solves on one GPU): every request's
fields are the same alone and in the mix, requests really overlap (the
batched server condenses all of them in one launch per step), the batched
and the thread-per-request servers give the same bits, and the memory
admission holds requests back when the device is full."""

import numpy as np
import pytest

from ddhdg_b200 import serving

pytestmark = pytest.mark.gpu


def _requests():
    # sizes that the reference's (undamped) Newton solves at these biases:
    # degree 2 needs cells of 1/32 um or less across the junction
    spec = [(2, 16, 1, 0.3), (2, 20, 1, 0.5), (2, 32, 2, 0.8), (1, 64, 2, 0.6), (3, 4, 1, 0.1), (2, 32, 1, 0.2)]
    return [serving.Request(i, d, m, k, b, 0.0) for i, (d, m, k, b) in enumerate(spec)]


def test_results_are_the_same_alone_and_in_the_mix():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    reqs = _requests()
    alone = serving.ThreadedDiodeServer(max_inflight=1, keep_states=True).run(reqs)
    mixed_server = serving.ThreadedDiodeServer(max_inflight=4, keep_states=True)
    mixed = mixed_server.run(reqs)
    assert mixed_server.peak_inflight > 1
    for a, b in zip(alone, mixed):
        assert a.converged and b.converged
        assert a.iterations == b.iterations
        for x, y in zip(a.state, b.state):
            assert np.array_equal(x, y), a.rid


def test_memory_admission_limits_the_requests_in_flight():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    reqs = _requests()
    biggest = max(serving.memory_estimate(r.dim, r.m, r.k) for r in reqs)
    limit = 2 * biggest
    server = serving.ThreadedDiodeServer(max_inflight=8, hbm_reserve=0, hbm_limit=limit)
    res = server.run(reqs)
    assert all(r.converged for r in res)
    assert server.peak_committed <= limit
    total = sum(serving.memory_estimate(r.dim, r.m, r.k) for r in reqs)
    assert server.peak_committed < total  # some requests had to wait
    stats = serving.latency_stats(res, max(r.finish for r in res))
    assert stats["p99_s"] >= stats["p50_s"] > 0


def test_batched_server_same_alone_in_the_mix_and_as_the_threaded_server():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    reqs = _requests()
    alone = serving.DiodeServer(max_inflight=1, keep_states=True).run(reqs)
    server = serving.DiodeServer(max_inflight=8, keep_states=True)
    mixed = server.run(reqs)
    assert server.peak_batch > 1  # several requests in one batched launch
    threaded = serving.ThreadedDiodeServer(max_inflight=1, keep_states=True).run(reqs)
    for a, b, c in zip(alone, mixed, threaded):
        assert a.converged and b.converged and c.converged
        assert a.iterations == b.iterations == c.iterations, (a.rid, a.iterations, b.iterations, c.iterations)
        for x, y, z in zip(a.state, b.state, c.state):
            assert np.array_equal(x, y), a.rid
            assert np.array_equal(x, z), a.rid


def test_batched_server_memory_admission():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    reqs = _requests()
    biggest = max(serving.memory_estimate(r.dim, r.m, r.k) for r in reqs)
    limit = 2 * biggest
    server = serving.DiodeServer(max_inflight=8, hbm_reserve=0, hbm_limit=limit)
    res = server.run(reqs)
    assert all(r.converged for r in res)
    assert server.peak_committed <= limit
    total = sum(serving.memory_estimate(r.dim, r.m, r.k) for r in reqs)
    assert server.peak_committed < total


@pytest.mark.parametrize("dim,m,k", [(2, 64, 2), (3, 8, 1)])
def test_memory_estimate_bounds_a_request(dim, m, k):
    """The device memory a request takes at its peak (sampled from another
    thread through the whole solve) stays below its admission estimate."""
    import gc
    import threading
    import time

    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    serving.solve_one(serving.Request(-1, 2, 16, 1, 0.1, 0.0))  # library state outside the request
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0, _ = torch.cuda.mem_get_info()
    peak, stop = [0], [False]

    def poll():
        while not stop[0]:
            free, _ = torch.cuda.mem_get_info()
            peak[0] = max(peak[0], free0 - free)
            time.sleep(0.005)

    th = threading.Thread(target=poll, daemon=True)
    th.start()
    try:
        res = serving.DiodeServer(max_inflight=2).run([serving.Request(0, dim, m, k, 0.3, 0.0)])
        torch.cuda.synchronize()
    finally:
        stop[0] = True
        th.join()
    assert res[0].converged
    assert 0 < peak[0] <= serving.memory_estimate(dim, m, k)


def test_mixed_precision_server():
    """Mixed-precision condensation in the batched server: each result is
    the same alone and in the mix (bitwise), and the final fields agree with
    the FP64 server's to 1e-8 relative."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    reqs = _requests()
    alone = serving.DiodeServer(max_inflight=1, keep_states=True, mixed=True).run(reqs)
    server = serving.DiodeServer(max_inflight=8, keep_states=True, mixed=True)
    mix = server.run(reqs)
    assert server.peak_batch > 1
    fp64 = serving.DiodeServer(max_inflight=8, keep_states=True).run(reqs)
    for r, a, b, c in zip(reqs, alone, mix, fp64):
        assert a.converged and b.converged and c.converged
        assert a.iterations == b.iterations
        for x, y in zip(a.state, b.state):
            assert np.array_equal(x, y), a.rid
        # per component block: cells [cell][V, n, p][flux axes, value][node],
        # trace [face][V, n, p][node]
        cell_x = a.state[0].reshape(r.m ** r.dim, 3, r.dim + 1, -1)
        cell_z = c.state[0].reshape(cell_x.shape)
        trace_x = a.state[1].reshape(-1, 3, (r.k + 1) ** (r.dim - 1))
        trace_z = c.state[1].reshape(trace_x.shape)
        # the relative error of each field: the scalar V, n, p against their
        # own largest magnitude, the flux vectors E, Wn, Wp against their
        # largest component (the transverse components of these diodes are
        # near zero), the trace values per component
        for b_ in range(3):
            for sl in (slice(r.dim, r.dim + 1), slice(0, r.dim)):
                z = cell_z[:, b_, sl]
                err = np.max(np.abs(cell_x[:, b_, sl] - z))
                assert err <= 1e-8 * np.max(np.abs(z)), (a.rid, b_, sl)
            z = trace_z[:, b_]
            assert np.max(np.abs(trace_x[:, b_] - z)) <= 1e-8 * np.max(np.abs(z)), (a.rid, b_)
