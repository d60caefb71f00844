"""Thermodynamic equilibrium on the GPU (src/thermodynamic_equilibrium.cpp:
9-405): local-charge-neutrality first guess projected on the device, the
V-only Newton solve on the device, and the projection of the equilibrium
densities n, p from the potential (src/project_component.cpp:575-654),
against the oracle doing the same."""

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases

pytestmark = pytest.mark.gpu


def _blocks_close(gc, gt, o, comps, tol):
    d, nb = o.dim, o.nb
    for c in comps:
        ia = slice(c * (d + 1) * nb, (c + 1) * (d + 1) * nb)
        for a, b in ((gc[:, ia], o.cell_state[:, ia]), (gt[:, c], o.trace_state[:, c])):
            err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
            assert err < tol, (c, err)


@pytest.mark.parametrize("dim,m,k", [(1, 16, 2), (2, 16, 1), (2, 8, 2), (3, 4, 1)])
def test_equilibrium_matches_oracle(dim, m, k):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g = NPSolver(pb, prm, adim)
    o = O.OracleSolver(pb, prm, adim)
    g.compute_local_charge_neutrality()
    o.compute_local_charge_neutrality()
    _blocks_close(g.get_cell_state(), g.get_trace_state(), o, [0], 1e-12)
    rg = g.compute_thermodynamic_equilibrium(generate_first_guess=False)
    ro = o.compute_thermodynamic_equilibrium(generate_first_guess=False)
    assert rg.converged and ro.converged
    assert rg.iterations == ro.iterations
    _blocks_close(g.get_cell_state(), g.get_trace_state(), o, [0, 1, 2], 1e-10)
