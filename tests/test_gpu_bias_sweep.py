"""Warm-started forward bias sweep on the GPU (contact conditions replaced on
the device between points, src/np_solver.cpp:2160-2233) against the oracle
doing the same sweep."""

import numpy as np
import pytest

from oracle import oracle as O
from ddhdg_b200 import workloads
from tests import cases

pytestmark = pytest.mark.gpu


def test_bias_sweep_matches_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = cases.diode(dim=2, m=16, k=1)
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    o = O.OracleSolver(pb, prm, adim)
    o.compute_local_charge_neutrality()
    o.private_run(1e-10, 1e-10, 50, thermo=True)
    o.project_quasi_fermi(1)
    o.project_quasi_fermi(2)
    g = NPSolver(pb, prm, adim)
    g.set_state(o.cell_state, o.trace_state)
    biases = [0.0, 0.1, 0.2, 0.3]
    states = {}

    def keep(v, s, r):
        states[v] = (s.get_cell_state().copy(), s.get_trace_state().copy(), r)

    workloads.bias_sweep(g, pb, biases, 1e-10, 1e-10, 50, callback=keep)
    for v in biases:
        workloads.set_bias(pb, v)
        ro = o.run(1e-10, 1e-10, 50)
        gc, gt, rg = states[v]
        assert rg.converged and ro.converged, v
        assert rg.iterations == ro.iterations, (v, rg.iterations, ro.iterations)
        d, nb = o.dim, o.nb
        for c in range(3):
            ia = slice(c * (d + 1) * nb, (c + 1) * (d + 1) * nb)
            for a, b in ((gc[:, ia], o.cell_state[:, ia]), (gt[:, c], o.trace_state[:, c])):
                assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300), (v, c)
