"""Failure reporting on the GPU without a device fault: bad numbers come back
as status codes from the kernels' own checks (zero or non-finite pivots),
and the context stays usable afterwards."""

import numpy as np
import pytest

from ddhdg_b200 import _lib
from oracle import oracle as O
from tests import cases

pytestmark = pytest.mark.gpu


def _solver():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = cases.diode(dim=2, m=8, k=1)
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    o = O.OracleSolver(pb, prm, adim)
    o.compute_local_charge_neutrality()
    return torch, NPSolver(pb, prm, adim), o


def test_non_finite_state_is_reported_and_the_context_recovers():
    torch, g, o = _solver()
    bad = o.cell_state.copy()
    bad[3, :] = np.nan
    g.set_state(bad, o.trace_state)
    with pytest.raises(_lib.DDHDGError) as e:
        g.private_run(1e-10, 1e-10, 5, thermo=True)
    # DDHDG_SINGULAR_PIVOT (local system) or DDHDG_SOLVER_ERROR (trace solve)
    assert e.value.code in (3, 8), e.value.code
    # the same context solves the good state
    g.set_state(o.cell_state, o.trace_state)
    res = g.private_run(1e-10, 1e-10, 50, thermo=True)
    assert res.converged


def test_singular_trace_system_is_reported():
    torch, g, o = _solver()
    g.set_state(o.cell_state, o.trace_state)
    tt, rhs, fl, dv = g.assemble_condense()
    n = g.sizes().n_trace_dofs
    x = torch.zeros(n, dtype=torch.float64, device=g.device)
    z = torch.zeros_like(tt)
    zi = torch.zeros_like(fl)
    code = g.L.ddhdg_solve_condensed(g._ctx, z.data_ptr(), torch.zeros_like(rhs).data_ptr(), zi.data_ptr(),
                                     torch.zeros_like(dv).data_ptr(), x.data_ptr(), 0, g._sp())
    assert code == 8, code  # DDHDG_SOLVER_ERROR
    assert "singular" in g.L.ddhdg_last_error().decode()
    # and the next solve of the real system works
    _lib.check(g.L.ddhdg_solve_condensed(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(), dv.data_ptr(),
                                         x.data_ptr(), 0, g._sp()), "solve_condensed")
    assert torch.isfinite(x).all()
