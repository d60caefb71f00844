"""Size-independent checks on the second diode configuration's mesh
(256 x 256 quads, degree 2, 1 184 256 trace dofs):

* the nested-dissection trace solve satisfies the assembled system
  (A x - b from the per-cell blocks, on the device, to FP64 round-off);
* a forward-biased Newton solve (warm start from equilibrium) drives the
  assembled residual down by at least eight orders of magnitude."""

import numpy as np
import pytest

from ddhdg_b200 import workloads

pytestmark = pytest.mark.gpu


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
