"""Mixed precision: the local condensation with an FP32 Jacobian (the linearised
cell and trace operators, the Gauss-Jordan inverse of the scalar system, Y and
the Schur product operands) and FP64 residuals, against the FP64 path and the
oracle.

The Newton loop is then a defect correction: each step solves with an FP32-
accurate Jacobian for an FP64 residual, so it converges (linearly, at a rate of
about the FP32 round-off times the local condition number) to the FP64
solution.  The stated errors: condensed systems within MIXED_TOL of the
oracle's FP64 ones, relative to the summed terms; final V, n, p within 1e-8 of
the FP64 solution."""

import numpy as np
import pytest

from oracle import oracle as O
from ddhdg_b200.problem import Precision
from tests import cases
from tests.gpu_helpers import block_rel_errs, make_pair

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
FINAL_TOL = 1e-8


def _npsolver():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    return NPSolver


def _field_rel_err(a_cell, b_cell, a_trace, b_trace, dim, nb):
    err = 0.0
    for c in range(3):
        ia = slice(c * (dim + 1) * nb, (c + 1) * (dim + 1) * nb)
        for a, b in ((a_cell[:, ia], b_cell[:, ia]), (a_trace[:, c], b_trace[:, c])):
            scale = max(np.abs(b).max(), 1e-300)
            err = max(err, float(np.abs(a - b).max() / scale))
    return err


@pytest.mark.parametrize("dim,k,m", [(2, 1, 6), (2, 2, 6), (3, 1, 3), (1, 2, 8)])
def test_mixed_condense_error_against_oracle(dim, k, m):
    _npsolver()
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k, precision=Precision.mixed)
    g, o = make_pair(pb, prm, adim, seed=dim * 10 + k)
    tt, rhs, flag, val = g.assemble_condense(False)
    oflag = o.assemble_condense(False)[2]
    assert np.array_equal(flag.cpu().numpy(), oflag)
    S, g_ = o.condense_accurate(False)
    e_tt, e_rhs, table = block_rel_errs(tt.cpu().numpy(), rhs.cpu().numpy(), S, g_, o)
    print(f"mixed condense {dim}D k={k}: worst block tt {e_tt:.2e}, rhs {e_rhs:.2e}; {table}")
    assert e_tt < MIXED_TOL, table
    assert e_rhs < MIXED_TOL, table
    # the FP32 kernel ran: its error is far above FP64 round-off
    assert e_tt > 1e-12


def test_mixed_precision_rejected_without_fp32_kernel():
    """2D degree 3 has 48 scalar unknowns per cell: no warp-per-cell kernel, so
    no mixed variant; the context creation fails with a bad-argument error."""
    NPSolver = _npsolver()
    from ddhdg_b200._lib import DDHDGError

    pb, prm, adim = cases.diode(dim=2, m=4, k=3, precision=Precision.mixed)
    with pytest.raises(DDHDGError, match="mixed precision"):
        NPSolver(pb, prm, adim)


def _start(pb, prm, adim):
    o = O.OracleSolver(pb, prm, adim)
    o.compute_local_charge_neutrality()
    o.private_run(1e-10, 1e-10, 50, thermo=True)
    o.project_quasi_fermi(1)
    o.project_quasi_fermi(2)
    return o


@pytest.mark.parametrize("dim,k,m,bias", [(2, 1, 32, 0.0), (2, 2, 32, 0.3), (3, 1, 8, 0.2)])
def test_mixed_newton_matches_fp64(dim, k, m, bias):
    """Newton from the equilibrium state, FP64 and mixed, same start: both
    converge and the final fields agree to 1e-8 relative.  The mixed loop may
    take a few more iterations (linear instead of quadratic end phase)."""
    NPSolver = _npsolver()
    res, states = {}, {}
    for prec in (Precision.fp64, Precision.mixed):
        pb, prm, adim = cases.diode(dim=dim, m=m, k=k, bias=bias, precision=prec)
        prm.consistent_drift_jacobian = True
        prm.consistent_recombination_jacobian = True
        o = _start(pb, prm, adim)
        g = NPSolver(pb, prm, adim)
        g.set_state(o.cell_state, o.trace_state)
        res[prec] = g.private_run(1e-12, 1e-12, 60)
        states[prec] = (g.get_cell_state(), g.get_trace_state())
    r64, r32 = res[Precision.fp64], res[Precision.mixed]
    assert r64.converged and r32.converged
    print(f"{dim}D k={k} m={m} bias={bias}: FP64 {r64.iterations} iterations, mixed {r32.iterations}")
    assert r32.iterations <= r64.iterations + 6
    (c64, t64), (c32, t32) = states[Precision.fp64], states[Precision.mixed]
    e = _field_rel_err(c32, c64, t32, t64, dim, (k + 1) ** dim)
    print(f"  final field error of mixed against FP64: {e:.2e}")
    assert e < FINAL_TOL, e
