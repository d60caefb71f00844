"""Residual, Jacobian and linear-system solution export (pyddhdg
NPSolver::get_residual / get_jacobian / get_linear_system_solution_vector,
src/pyddhdg/pyddhdg.cpp:1601-1935) from the device-assembled system, against
the oracle's global system built from its own condensed cell blocks."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from ddhdg_b200.problem import Component
from tests import cases
from tests.gpu_helpers import make_pair

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("dim,m,k", [(1, 8, 2), (2, 6, 2), (2, 6, 1), (3, 3, 1)])
def test_residual_jacobian_and_solution_match_oracle(dim, m, k):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g, o = make_pair(pb, prm, adim, seed=11)
    g.assemble_system()
    J = g.get_jacobian()
    r = g.get_residual()
    # the oracle's condensed blocks (row-equilibrated solve of its term-by-term
    # local systems), assembled the same way: unit Dirichlet rows whose
    # right-hand side is the projected Dirichlet increment
    _, _, flag, val = o.assemble_condense()
    S, gv = o.condense_accurate()
    s_tt, s_rhs = o.condense_term_scale
    A, b, ddofs, dvals = o.global_system(S, gv, flag, val, 3)
    b = b.copy()
    b[ddofs] = dvals
    A = A.tocsr()
    n = A.shape[0]
    idx = np.arange(n).reshape(o.nfaces, 3, o.nf)
    comps = {Component(c): idx[:, c, :].ravel() for c in range(3)}
    assert set(J) == {(c1, c2) for c1 in comps for c2 in comps}
    # each (component, component) block at the scale of the terms summed in
    # that block (a global entry sums at most two cells' contributions)
    b_tt, b_rhs = o.condense_block_scale
    for (c1, c2), blk in J.items():
        ref = A[comps[c1]][:, comps[c2]].toarray()
        err = np.abs(blk.toarray() - ref).max() / max(2 * b_tt[int(c1), int(c2)], 1e-300)
        assert err < TOL, (c1, c2, err)
    for c, v in r.items():
        ref = b[comps[c]]
        # Dirichlet rows carry the projected values (trace scale)
        err = np.abs(v - ref).max() / max(2 * b_rhs[int(c)], np.abs(o.trace_state[:, int(c)]).max())
        assert err < TOL, (c, err)
    # the solution of the assembled system: against a sparse LU of the same
    # (device-assembled) system, and, within its conditioning, the oracle's
    import scipy.sparse as sp

    rowptr, colind = g._csr_structure()
    Ag = sp.csr_matrix((g._system["values"].cpu().numpy(), colind, rowptr), shape=(n, n))
    xg_ref = spla.spsolve(Ag.tocsc(), g._system["rhs"].cpu().numpy())
    x_ref = spla.spsolve(A.tocsc(), b)
    x = g.get_linear_system_solution_vector()
    scale = np.abs(xg_ref).max()
    for c, v in x.items():
        assert np.abs(v - xg_ref[comps[c]]).max() <= 1e-9 * scale, c
        assert np.abs(v - x_ref[comps[c]]).max() <= 1e-6 * scale, c
