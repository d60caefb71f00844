"""Size-independent checks on the second diode configuration's mesh
(256 x 256 quads, degree 2, 1 184 256 trace dofs):

* the nested-dissection trace solve satisfies the assembled system
  (A x - b from the per-cell blocks, on the device, to FP64 round-off);
* a forward-biased Newton solve (warm start from equilibrium) drives the
  assembled residual down by at least eight orders of magnitude;
* the condensed systems of a seeded sample of 1 280 cells (both junction
  columns, both contacts, the other boundaries and the interior) match the
  oracle's to 1e-10 in every component block: tt at the converged 0.3 V
  state, tt and rhs at that state perturbed by a seeded 1e-3 (at the
  converged state the rhs is the Newton residual itself, round-off of terms
  ~1e14 times larger)."""

import numpy as np
import pytest

from ddhdg_b200 import workloads
from tests.gpu_helpers import block_rel_errs

pytestmark = pytest.mark.gpu


def _sample_cells(m, n_interior=1024, seed=7):
    """Cells of an m x m mesh (x fastest): the two columns at the junction,
    the two contact columns, the bottom and top rows, and seeded interior
    cells."""
    ix = np.arange(m * m) % m
    iy = np.arange(m * m) // m
    special = np.flatnonzero((ix == m // 2 - 1) | (ix == m // 2) | (ix == 0) | (ix == m - 1) |
                             (iy == 0) | (iy == m - 1))
    rng = np.random.default_rng(seed)
    special = rng.choice(special, size=min(256, special.size), replace=False)
    rest = np.setdiff1d(np.arange(m * m), special)
    return np.sort(np.concatenate([special, rng.choice(rest, size=n_interior, replace=False)]))


def _oracle_residuals(o, m, nf, n_pairs=256, seed=11):
    """The oracle's equations at its current state on a sample of an m x m
    mesh: the cell-equation residuals (cc_rhs) of the sampled cells, and the
    trace-equation residuals assembled on faces whose two cells are both in
    the sample (the sum of the two cells' tt_rhs rows of that face).  Both
    vanish at a solution of the discrete problem."""
    rng = np.random.default_rng(seed)
    ix = np.arange(m * m) % m
    iy = np.arange(m * m) // m
    base = rng.choice(np.flatnonzero((ix < m - 1) & (iy < m - 1)), size=n_pairs, replace=False)
    cells = np.unique(np.concatenate([base, base + 1, base + m]))
    pos = {int(c): i for i, c in enumerate(cells)}
    _, _, _, _, c_rhs, t_rhs = o.local_cell_systems(cells=cells)
    rows = lambda f: slice(f * 3 * nf, (f + 1) * 3 * nf)  # trace rows of local face f, [f][component][node]
    faces = []
    for c in base:
        a = t_rhs[pos[int(c)]]
        faces.append(a[rows(1)] + t_rhs[pos[int(c) + 1]][rows(0)])  # x face between c and c + 1
        faces.append(a[rows(3)] + t_rhs[pos[int(c) + m]][rows(2)])  # y face between c and c + m
    return c_rhs, np.array(faces)


def _residual_of(torch, g, x):
    """(A x - b, b) for the assembled system, from the per-cell blocks."""
    sysm = g._system
    tt, rhs, flag, val = sysm["blocks"]
    nc = g.ncells
    Nt = tt.shape[-1]
    nd = Nt // g.F
    faces = torch.as_tensor(g.cell_faces, device=g.device, dtype=torch.int64)        # [ncells, F]
    dof = (faces[:, :, None] * nd + torch.arange(nd, device=g.device)).reshape(nc, Nt)  # [ncells, Nt]
    xc = x[dof]                                                                      # [ncells, Nt]
    flag = flag.reshape(nc, Nt).bool()
    y = torch.bmm(tt.reshape(nc, Nt, Nt), xc.unsqueeze(-1)).squeeze(-1)
    y = torch.where(flag, xc, y)            # Dirichlet rows are identity rows
    Ax = torch.zeros_like(x).index_add_(0, dof.reshape(-1), y.reshape(-1) * (~flag).reshape(-1))
    # identity rows once per Dirichlet dof (each sits on one boundary face)
    Ax.index_put_((dof[flag],), xc[flag])
    return Ax - sysm["rhs"], sysm["rhs"]


def test_full_size_solve_and_newton():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = workloads.diode(dim=2, m=256, k=2)
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    g = NPSolver(pb, prm, adim)
    assert g.ncells == 65536
    assert g.compute_thermodynamic_equilibrium().converged
    workloads.set_bias(pb, 0.3)
    g.update_boundary_tables()
    start = (g.get_cell_state(), g.get_trace_state())
    # 1) the trace solve at full size
    g.assemble_system()
    xs = g.get_linear_system_solution_vector()
    n = g.sizes().n_trace_dofs
    x = torch.empty(n, dtype=torch.float64, device=g.device)
    idx = np.arange(n).reshape(g.nfaces, 3, g.nf)
    for c, v in xs.items():
        x[torch.as_tensor(idx[:, int(c), :].ravel(), device=g.device)] = torch.as_tensor(v, device=g.device)
    r, b = _residual_of(torch, g, x)
    assert torch.isfinite(x).all()
    assert float(r.abs().max()) <= 1e-9 * float(b.abs().max())
    r0 = float(b.abs().max())
    # 2) the Newton solve at full size
    res = g.run(1e-10, 1e-10, 30)
    assert res.converged
    g.assemble_system()
    r1 = float(g._system["rhs"].abs().max())
    assert r1 <= 1e-8 * r0, (r0, r1)
    # 3) the condensed systems at the converged state against the oracle, on
    # a sample of cells
    from oracle.oracle import OracleSolver

    o = OracleSolver(pb, prm, adim)
    sel = _sample_cells(256)
    assert sel.size >= 1024
    # the converged fields solve the oracle's equations: its cell residuals
    # and its assembled face residuals on a sample are 1e8 times below the
    # ones at the start state
    o.cell_state[:], o.trace_state[:] = start
    c_start, f_start = _oracle_residuals(o, 256, g.nf)
    o.cell_state[:] = g.get_cell_state()
    o.trace_state[:] = g.get_trace_state()
    c_conv, f_conv = _oracle_residuals(o, 256, g.nf)
    print(f"oracle residuals on the sample: cells {np.abs(c_start).max():.3e} -> {np.abs(c_conv).max():.3e}, "
          f"faces {np.abs(f_start).max():.3e} -> {np.abs(f_conv).max():.3e}")
    assert np.abs(c_conv).max() <= 1e-8 * np.abs(c_start).max()
    assert np.abs(f_conv).max() <= 1e-8 * np.abs(f_start).max()
    rng = np.random.default_rng(21)
    for perturbed in (False, True):
        cs, ts = g.get_cell_state(), g.get_trace_state()
        if perturbed:
            cs = cs * (1 + 1e-3 * rng.standard_normal(cs.shape))
            ts = ts * (1 + 1e-3 * rng.standard_normal(ts.shape))
            g.set_state(cs, ts)
        tt, rhs, flag, _ = g.assemble_condense()
        o.cell_state[:] = cs
        o.trace_state[:] = ts
        S, gv = o.condense_accurate(cells=sel)
        e_tt, e_rhs, table = block_rel_errs(tt.cpu().numpy()[sel], rhs.cpu().numpy()[sel], S, gv, o)
        print(f"256x256 k=2 sample of {sel.size} cells (perturbed: {perturbed}): worst block tt {e_tt:.2e}, "
              f"rhs {e_rhs:.2e}")
        assert e_tt < 1e-10, table
        if perturbed:
            assert e_rhs < 1e-10, table


def test_full_size_mixed_newton_matches_fp64():
    """The mixed-precision condensation (FP32 Jacobian, FP64 residuals) on the
    256 x 256 degree-2 diode: a 0.3 V Newton solve from the same equilibrium
    state converges, and its final V, n, p agree with the FP64 solve to 1e-8
    relative (per component block, against the block's largest magnitude)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = workloads.diode(dim=2, m=256, k=2)
    prm.consistent_drift_jacobian = True
    prm.consistent_recombination_jacobian = True
    g = NPSolver(pb, prm, adim)
    assert g.compute_thermodynamic_equilibrium().converged
    start = (g.get_cell_state(), g.get_trace_state())
    workloads.set_bias(pb, 0.3)
    g.update_boundary_tables()
    r64 = g.run(1e-10, 1e-10, 30)
    c64, t64 = g.get_cell_state(), g.get_trace_state()
    del g
    pbm, prmm, adimm = workloads.diode(dim=2, m=256, k=2, bias=0.3, precision=1)
    prmm.consistent_drift_jacobian = True
    prmm.consistent_recombination_jacobian = True
    gm = NPSolver(pbm, prmm, adimm)
    gm.set_state(*start)
    rm = gm.run(1e-10, 1e-10, 30)
    assert r64.converged and rm.converged
    c32, t32 = gm.get_cell_state(), gm.get_trace_state()
    nb, d = 9, 2
    err = 0.0
    for c in range(3):
        ia = slice(c * (d + 1) * nb, (c + 1) * (d + 1) * nb)
        for a, b in ((c32[:, ia], c64[:, ia]), (t32[:, c], t64[:, c])):
            err = max(err, float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)))
    print(f"256x256 k=2, 0.3 V: FP64 {r64.iterations} iterations, mixed {rm.iterations}; "
          f"final field difference {err:.2e}")
    assert err < 1e-8, err
    # the mixed result against the oracle's own equations (FP64): its cell
    # and assembled face residuals on a sample are 1e8 times below the start's
    from oracle.oracle import OracleSolver

    o = OracleSolver(pbm, prmm, adimm)
    o.cell_state[:], o.trace_state[:] = start
    c_start, f_start = _oracle_residuals(o, 256, 3)
    o.cell_state[:], o.trace_state[:] = c32, t32
    c_conv, f_conv = _oracle_residuals(o, 256, 3)
    print(f"oracle residuals at the mixed solution: cells {np.abs(c_start).max():.3e} -> "
          f"{np.abs(c_conv).max():.3e}, faces {np.abs(f_start).max():.3e} -> {np.abs(f_conv).max():.3e}")
    assert np.abs(c_conv).max() <= 1e-8 * np.abs(c_start).max()
    assert np.abs(f_conv).max() <= 1e-8 * np.abs(f_start).max()
