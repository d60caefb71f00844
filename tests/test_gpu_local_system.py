"""The per-cell parity probe and the plain FP64 device path, through the C ABI.

* ddhdg_local_cell_system (get_local_cell_system, src/np_solver.cpp:
  2337-2445): the unreduced local system {cc, ct, tc, tt, c, t} of listed
  cells, assembled on the device term by term, against the oracle's
  restatement of the reference's assembly
  (include/assembling_methods.template.h:134-2160, local_condenser.cpp:
  142-160).  Each array is split into blocks by (component, flux or scalar)
  of its rows and columns, and every block is checked at 1e-10 of its own
  largest magnitude: the assembly sums a handful of quadrature terms, so the
  differences are FP64 round-off of those terms (up to a few 1e-12 of the
  block where the terms cancel, e.g. the flux rows of c, V0 div q - E0 . q).
* ddhdg_assemble_condense_plain / ddhdg_reconstruct_plain (the full local
  system, LU of cc, Schur complement, and the second assembly pass of the
  reconstruction) against the oracle's accurate condensation, per block at
  1e-10, like the block-eliminated kernels in test_gpu_parity."""

import numpy as np
import pytest

from ddhdg_b200.problem import (CellFaceTauNPSolverParameters, DDFluxType, LinearRecombinationTerm,
                                NonlinearSolverParameters)
from tests import cases
from tests.gpu_helpers import block_rel_errs, cell_block_rel_err, make_pair

pytestmark = pytest.mark.gpu

TOL_ASSEMBLY = 1e-10
TOL = 1e-10


def _labels(o, thermo):
    """(component, 'flux'|'scalar') of every enabled cell dof, and the
    component of every restricted trace dof."""
    comps = [0] if thermo else [c for c in range(3) if o.enabled[c]]
    d, nb = o.dim, o.nb
    cell = [(comps[i // ((d + 1) * nb)], "flux" if (i // nb) % (d + 1) < d else "scalar")
            for i in range(len(comps) * (d + 1) * nb)]
    Nt = o.F * len(comps) * o.nf
    trace = [(comps[(j // o.nf) % len(comps)], "trace") for j in range(Nt)]
    return cell, trace


def _blocks(rows, cols):
    for r in sorted(set(rows)):
        ri = np.array([x == r for x in rows])
        for c in sorted(set(cols)):
            ci = np.array([x == c for x in cols])
            yield (r, c), ri, ci


def _local_state(o, cell, thermo):
    """The cell's enabled cell dofs and restricted trace dofs [face][comp][node]."""
    comps = [0] if thermo else [c for c in range(3) if o.enabled[c]]
    d, nb = o.dim, o.nb
    u = np.concatenate([o.cell_state[cell, c * (d + 1) * nb:(c + 1) * (d + 1) * nb] for c in comps])
    lam = np.concatenate([o.trace_state[o.cell_faces[cell, f], c] for f in range(o.F) for c in comps])
    return u, lam


def compare_local_systems(g, o, cells, thermo=False):
    """cc, ct, tc, tt per block at TOL_ASSEMBLY of the block's largest
    magnitude; the residual vectors c and t per block at TOL_ASSEMBLY of the
    magnitude of the terms they sum, |c| + |cc| |u0| + |ct| |lambda0| (and
    |t| + |tc| |u0| + |tt| |lambda0|): at a projected equilibrium state the
    flux rows of c cancel to round-off."""
    got = g.get_local_cell_system(cells, thermo)
    cell_l, trace_l = _labels(o, thermo)
    worst = 0.0
    for i, cell in enumerate(cells):
        ref = o.local_cell_system(int(cell), thermo)
        u0, lam0 = _local_state(o, int(cell), thermo)
        term = {"c": np.abs(ref["c"]) + np.abs(ref["cc"]) @ np.abs(u0) + np.abs(ref["ct"]) @ np.abs(lam0),
                "t": np.abs(ref["t"]) + np.abs(ref["tc"]) @ np.abs(u0) + np.abs(ref["tt"]) @ np.abs(lam0)}
        for key, (rl, cl) in dict(cc=(cell_l, cell_l), ct=(cell_l, trace_l), tc=(trace_l, cell_l),
                                  tt=(trace_l, trace_l)).items():
            a, b = got[key][i], ref[key]
            assert a.shape == b.shape, (key, a.shape, b.shape)
            for blk, ri, ci in _blocks(rl, cl):
                rb, gb = b[np.ix_(ri, ci)], a[np.ix_(ri, ci)]
                scale = np.abs(rb).max()
                if scale == 0.0:
                    assert np.all(gb == 0.0), (key, blk, cell)
                    continue
                e = float(np.abs(gb - rb).max() / scale)
                worst = max(worst, e)
                assert e < TOL_ASSEMBLY, (key, blk, int(cell), e)
        for key, lab in (("c", cell_l), ("t", trace_l)):
            a, b = got[key][i], ref[key]
            for r in sorted(set(lab)):
                ri = np.array([x == r for x in lab])
                scale = term[key][ri].max()
                if scale == 0.0:
                    assert np.all(a[ri] == 0.0), (key, r, cell)
                    continue
                e = float(np.abs(a[ri] - b[ri]).max() / scale)
                worst = max(worst, e)
                assert e < TOL_ASSEMBLY, (key, r, int(cell), e)
    return worst


def compare_plain(g, o, thermo=False, tol=TOL, seed=5):
    tt, rhs, flag, val = g.assemble_condense_plain(thermo)
    _, _, oflag, oval = o.assemble_condense(thermo)
    assert np.array_equal(flag.cpu().numpy(), oflag)
    assert np.abs(val.cpu().numpy() - oval).max() <= tol * max(np.abs(oval).max(), np.abs(o.trace_state).max())
    S, g_ = o.condense_accurate(thermo)
    e_tt, e_rhs, table = block_rel_errs(tt.cpu().numpy(), rhs.cpu().numpy(), S, g_, o, thermo)
    assert e_tt < tol, table
    assert e_rhs < tol, table
    rng = np.random.default_rng(seed)
    comps = [0] if thermo else [c for c in range(3) if o.enabled[c]]
    upd = np.zeros((o.nfaces, 3, o.nf))
    for c in comps:
        upd[:, c] = rng.standard_normal((o.nfaces, o.nf)) * max(np.abs(o.trace_state[:, c]).max(), 1e-3) * 1e-2
    du = g.reconstruct_plain(upd, thermo).cpu().numpy()
    acc = o.reconstruct_accurate(upd, thermo)
    e, table = cell_block_rel_err(du, acc, o)
    assert e < tol, table


def _some_cells(o, n=12, seed=3):
    """Both contact columns, the junction and seeded others."""
    rng = np.random.default_rng(seed)
    m = o.ncells
    pick = {0, m - 1, m // 2, m // 2 - 1}
    pick |= set(rng.choice(m, size=min(n, m), replace=False).tolist())
    return np.array(sorted(pick), dtype=np.int64)


@pytest.mark.parametrize("dim,k,m", [(2, 1, 6), (2, 2, 6), (2, 3, 4), (3, 1, 3), (3, 2, 2), (1, 2, 8)])
def test_local_cell_system_matches_oracle(dim, k, m):
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g, o = make_pair(pb, prm, adim, seed=dim * 10 + k)
    compare_local_systems(g, o, _some_cells(o))
    compare_local_systems(g, o, _some_cells(o), thermo=True)


@pytest.mark.parametrize("variant", ["use_trace", "qiu_shi", "jacobian_fix", "phi_linearize", "n_only",
                                     "V_p", "cell_face_tau", "neumann"])
def test_local_cell_system_variants(variant):
    if variant == "cell_face_tau":
        prm = CellFaceTauNPSolverParameters(2, 2, 2, NonlinearSolverParameters())
        pb, _, adim = cases.log_potential(2, prm, refinements=2)
        pb.recombination_term = LinearRecombinationTerm("0.3*x", "0.1*y", 0.2)
        rng = np.random.default_rng(4)
        for cell in range(pb.mesh.n_cells):
            for f in range(4):
                prm.set_face(cell, f, *(rng.uniform(0.5, 2.0, 3) * np.array([1.0, 100.0, 10000.0])))
        g, o = make_pair(pb, prm, adim, seed=4, thermo_start=False)
    elif variant == "neumann":
        pb, prm, adim = cases.neumann_linear(2)
        g, o = make_pair(pb, prm, adim, seed=2, thermo_start=False)
    else:
        flux = {"use_trace": DDFluxType.use_trace, "qiu_shi": DDFluxType.qiu_shi_stabilization}.get(
            variant, DDFluxType.use_cell)
        pb, prm, adim = cases.diode(dim=2, m=6, k=2, flux=flux)
        enabled = {"n_only": (False, True, False), "V_p": (True, False, True)}.get(variant, (True, True, True))
        if variant == "jacobian_fix":
            prm.consistent_drift_jacobian = True
            prm.consistent_recombination_jacobian = True
        if variant == "phi_linearize":
            prm.phi_linearize = True
        g, o = make_pair(pb, prm, adim, seed=7, enabled=enabled,
                         perturb=0.0 if variant == "phi_linearize" else 1e-3)
    compare_local_systems(g, o, np.arange(o.ncells, dtype=np.int64))


@pytest.mark.parametrize("dim,k,m", [(2, 1, 6), (2, 2, 6), (2, 3, 4), (3, 1, 3), (3, 2, 2), (1, 2, 8)])
def test_plain_path_matches_oracle(dim, k, m):
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g, o = make_pair(pb, prm, adim, seed=dim * 10 + k)
    compare_plain(g, o)
    compare_plain(g, o, thermo=True)


@pytest.mark.parametrize("flux", [DDFluxType.use_trace, DDFluxType.qiu_shi_stabilization])
def test_plain_path_fluxes(flux):
    pb, prm, adim = cases.diode(dim=2, m=6, k=2, flux=flux)
    g, o = make_pair(pb, prm, adim, seed=int(flux) + 20)
    compare_plain(g, o)


def test_plain_path_agrees_with_the_block_eliminated_kernel():
    """Two algorithms for the same condensed system: the plain path (full
    81 x 81 cell system, LU) and the block-eliminated kernel agree per block."""
    pb, prm, adim = cases.diode(dim=2, m=16, k=2)
    g, o = make_pair(pb, prm, adim, seed=31)
    a = [t.cpu().numpy() for t in g.assemble_condense()]
    b = [t.cpu().numpy() for t in g.assemble_condense_plain()]
    assert np.array_equal(a[2], b[2])
    S, g_ = o.condense_accurate()
    e_tt, e_rhs, table = block_rel_errs(a[0], a[1], b[0], b[1], o)
    assert max(e_tt, e_rhs) < 2 * TOL, table
