"""Parity of the CUDA hot path against the CPU oracle (the reference's
algorithm restated), through the C ABI.

The condensed systems are compared with the oracle's term-by-term local
matrices condensed by a row-equilibrated LU refined in long double.  The
tolerance 1e-10 holds in every (row component, column component) block of tt
and every component block of rhs separately, relative to the magnitude of the
terms summed inside that block: in the junction cells of the diodes the
condensed right-hand side is a difference of two terms up to 5e6 times larger
than itself, so FP64 round-off of any implementation is relative to those
terms, not to the result; and the p-n coupling block is ~1e-4 of the V-n one,
so a global scale would not check it.  The reconstructed cell update is
checked the same way per component and per field (flux, scalar).  The
oracle's own reference-style (unequilibrated Gauss-Jordan) inversion is
pinned against the same target on the global scale only: in 3D Dirichlet
cells its round-off reaches 2e-8 of the V block."""

import numpy as np
import pytest

from ddhdg_b200.problem import (CellFaceTauNPSolverParameters, Component, DDFluxType,
                                LinearRecombinationTerm, NonlinearSolverParameters,
                                FixedTauNPSolverParameters, BoundaryConditionType as BCT)
from tests import cases
from tests.gpu_helpers import block_rel_errs, cell_block_rel_err, make_pair, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


def compare_condense(g, o, thermo=False, tol=TOL):
    tt, rhs, flag, val = g.assemble_condense(thermo)
    ott, orhs, oflag, oval = o.assemble_condense(thermo)
    assert np.array_equal(flag.cpu().numpy(), oflag)
    # Dirichlet increments are differences of O(trace) numbers
    assert rel_err(val.cpu().numpy(), oval, floor=np.abs(o.trace_state).max()) < tol
    # the oracle's terms, condensed with a row-equilibrated solve: the GPU must
    # match it to FP64 round-off
    S, g_ = o.condense_accurate(thermo)
    s_tt, s_rhs = o.condense_term_scale
    e_tt, e_rhs, table = block_rel_errs(tt.cpu().numpy(), rhs.cpu().numpy(), S, g_, o, thermo)
    assert e_tt < tol, table
    assert e_rhs < tol, table
    # the reference's own inversion (LU of the transpose, FullMatrix::
    # gauss_jordan) agrees with it within its round-off
    assert rel_err(ott, S, floor=s_tt) < tol
    assert rel_err(orhs, g_, floor=s_rhs) < tol
    return tt, rhs


def compare_reconstruct(g, o, thermo=False, tol=TOL, seed=5):
    g.assemble_condense(thermo)
    rng = np.random.default_rng(seed)
    comps = [0] if thermo else [c for c in range(3) if o.enabled[c]]
    upd = np.zeros((o.nfaces, 3, o.nf))
    for c in comps:
        upd[:, c] = rng.standard_normal((o.nfaces, o.nf)) * max(np.abs(o.trace_state[:, c]).max(), 1e-3) * 1e-2
    gu = g.reconstruct(upd, thermo).cpu().numpy()
    ou = o.reconstruct(upd, thermo)
    acc = o.reconstruct_accurate(upd, thermo)
    e, table = cell_block_rel_err(gu, acc, o)
    assert e < tol, table
    assert rel_err(ou, acc) < 1e-5


# m keeps every quadrature point off the junction x = 0.5, where the step
# doping is discontinuous (two independently computed Gauss rules may differ
# by an ulp there and sample opposite sides of the step)
@pytest.mark.parametrize("dim,k,m", [(2, 1, 6), (2, 2, 6), (2, 3, 4), (3, 1, 3), (1, 2, 8), (3, 2, 2)])
def test_diode_condense_and_reconstruct(dim, k, m):
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g, o = make_pair(pb, prm, adim, seed=dim * 10 + k)
    compare_condense(g, o)
    compare_reconstruct(g, o)


@pytest.mark.parametrize("flux", [DDFluxType.use_trace, DDFluxType.qiu_shi_stabilization])
def test_fluxes(flux):
    pb, prm, adim = cases.diode(dim=2, m=6, k=2, flux=flux)
    g, o = make_pair(pb, prm, adim, seed=int(flux))
    compare_condense(g, o)
    compare_reconstruct(g, o)


@pytest.mark.parametrize("fix", [1, 2, 3])
def test_jacobian_options(fix):
    pb, prm, adim = cases.diode(dim=2, m=6, k=2)
    prm.consistent_drift_jacobian = bool(fix & 1)
    prm.consistent_recombination_jacobian = bool(fix & 2)
    g, o = make_pair(pb, prm, adim, seed=fix)
    compare_condense(g, o)


def test_thermodynamic_equilibrium_mode():
    pb, prm, adim = cases.diode(dim=2, m=6, k=2)
    g, o = make_pair(pb, prm, adim, seed=11)
    compare_condense(g, o, thermo=True)
    compare_reconstruct(g, o, thermo=True)


def test_phi_linearize():
    pb, prm, adim = cases.diode(dim=2, m=6, k=1)
    prm.phi_linearize = True
    g, o = make_pair(pb, prm, adim, seed=12, perturb=0.0)
    compare_condense(g, o)
    compare_reconstruct(g, o)


@pytest.mark.parametrize("enabled", [(True, False, False), (False, True, False), (False, True, True),
                                     (True, True, False), (True, False, True)])
def test_partial_components(enabled):
    """disabling_components (tests/disabling_components.cpp) mask variants."""
    pb, prm, adim = cases.diode(dim=2, m=6, k=2)
    g, o = make_pair(pb, prm, adim, seed=sum(enabled) * 7 + enabled[0], enabled=enabled)
    compare_condense(g, o)
    compare_reconstruct(g, o)


def test_cell_face_tau_and_linear_recombination():
    prm = CellFaceTauNPSolverParameters(2, 2, 2, NonlinearSolverParameters())
    pb, _, adim = cases.log_potential(2, prm, refinements=2)
    pb.recombination_term = LinearRecombinationTerm("0.3*x", "0.1*y", 0.2)
    rng = np.random.default_rng(4)
    for cell in range(pb.mesh.n_cells):
        for f in range(4):
            prm.set_face(cell, f, *(rng.uniform(0.5, 2.0, 3) * np.array([1.0, 100.0, 10000.0])))
    g, o = make_pair(pb, prm, adim, seed=4, thermo_start=False)
    o.set_component(0, "-2 * log(x)")
    o.set_component(1, "2 / (x^2 * q)")
    o.cell_state *= 1 + 1e-2 * rng.standard_normal(o.cell_state.shape)
    g.set_state(o.cell_state, o.trace_state)
    compare_condense(g, o)
    compare_reconstruct(g, o)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_neumann_faces(dim):
    pb, prm, adim = cases.neumann_linear(dim)
    g, o = make_pair(pb, prm, adim, seed=dim, thermo_start=False)
    compare_condense(g, o)
    compare_reconstruct(g, o)
