"""Global trace solve on the GPU (ddhdg_solve_condensed: nested-dissection
multifrontal LU from the per-cell condensed blocks) against a sparse LU
(SuperLU) of the same global system assembled in CSR by ddhdg_scatter
(copy_local_to_global, src/np_solver.cpp:1293-1322; solve_linear_problem,
src/np_solver.cpp:1326-1354)."""

import ctypes

import numpy as np
import pytest

from ddhdg_b200 import _lib
from tests import cases

pytestmark = pytest.mark.gpu


def _setup(dim, m, k):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g = NPSolver(pb, prm, adim)
    g.compute_local_charge_neutrality()
    for c in (1, 2):
        _lib.check(g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(),
                                             g.trace_state.data_ptr(), g._sp()), "project_density")
    return torch, g


def _csr(torch, g, tt, rhs, fl, dv):
    import scipy.sparse as sp

    s = g.sizes(False)
    n, nnz = s.n_trace_dofs, s.nnz
    vals = torch.zeros(nnz, dtype=torch.float64, device=g.device)
    grhs = torch.zeros(n, dtype=torch.float64, device=g.device)
    _lib.check(g.L.ddhdg_scatter(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(), dv.data_ptr(),
                                 vals.data_ptr(), grhs.data_ptr(), 0, g._sp()), "scatter")
    rp, ci = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(g.L.ddhdg_get_csr(g._ctx, 0, ctypes.byref(rp), ctypes.byref(ci)), "get_csr")
    torch.cuda.synchronize()
    # the context owns the CSR structure (device arrays): copy it to the host
    rowptr = np.empty(n + 1, dtype=np.int32)
    colind = np.empty(nnz, dtype=np.int32)
    cudart = ctypes.CDLL("libcudart.so")
    for host, ptr in ((rowptr, rp), (colind, ci)):
        assert cudart.cudaMemcpy(host.ctypes.data_as(ctypes.c_void_p), ptr,
                                 ctypes.c_size_t(host.nbytes), 2) == 0  # device to host
    A = sp.csr_matrix((vals.cpu().numpy(), colind, rowptr), shape=(n, n))
    return A, grhs.cpu().numpy()


# 48 x 48 at degree 2: the root separator has 432 eliminated dofs, so the top
# fronts take the per-front dense LU path; the smaller meshes cover the fused
# small-front kernel, the one-CTA mid-front kernel and batched cuBLAS
@pytest.mark.parametrize("dim,m,k", [(1, 16, 2), (2, 16, 1), (2, 8, 2), (2, 9, 2), (3, 3, 1), (3, 2, 2),
                                     (2, 48, 2)])
def test_nested_dissection_matches_sparse_lu(dim, m, k):
    import scipy.sparse.linalg as spla

    torch, g = _setup(dim, m, k)
    tt, rhs, fl, dv = g.assemble_condense()
    A, b = _csr(torch, g, tt, rhs, fl, dv)
    x_lu = spla.splu(A.tocsc()).solve(b)
    x = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=g.device)
    # the second call reuses the elimination tree and captures the numeric
    # sequence in a CUDA graph, the third replays it
    for _ in range(3):
        _lib.check(g.L.ddhdg_solve_condensed(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(),
                                             dv.data_ptr(), x.data_ptr(), 0, g._sp()), "solve_condensed")
        torch.cuda.synchronize()
        xg = x.cpu().numpy()
        assert np.isfinite(xg).all()
        # the 3D degree-2 system is the worst conditioned of these
        assert np.abs(xg - x_lu).max() <= 1e-9 * np.abs(x_lu).max()
        # residual no worse than the sparse LU's, up to a small factor
        r_nd = np.abs(A @ xg - b).max()
        r_lu = np.abs(A @ x_lu - b).max()
        assert r_nd <= 100 * r_lu + 1e-12 * np.abs(b).max()


def test_solver_graphs_switch_gives_the_same_solution():
    """ddhdg_set_solver_graphs: eager launches and the captured graph run the
    same kernels on the same data, so the solutions are bitwise equal; the
    switch can be flipped between solves (turning it off drops the graph)."""
    torch, g = _setup(2, 16, 2)
    tt, rhs, fl, dv = g.assemble_condense()
    n = g.sizes().n_trace_dofs
    sols = {}
    for graphs in (True, False, True):
        g.set_solver_graphs(graphs)
        for rep in range(3):
            x = torch.full((n,), float("nan"), dtype=torch.float64, device=g.device)
            # fresh output buffers every call, then the same buffer three times
            _lib.check(g.L.ddhdg_solve_condensed(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(),
                                                 dv.data_ptr(), x.data_ptr(), 0, g._sp()), "solve_condensed")
            torch.cuda.synchronize()
            sols.setdefault(graphs, []).append(x.cpu().numpy())
        xs = torch.full((n,), float("nan"), dtype=torch.float64, device=g.device)
        for rep in range(3):
            _lib.check(g.L.ddhdg_solve_condensed(g._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(),
                                                 dv.data_ptr(), xs.data_ptr(), 0, g._sp()), "solve_condensed")
            torch.cuda.synchronize()
            sols[graphs].append(xs.cpu().numpy())
    ref = sols[True][0]
    assert np.isfinite(ref).all()
    for graphs, xs_ in sols.items():
        for x in xs_:
            assert np.array_equal(x, ref), graphs


def test_tensor_path_products_match_the_library_ones(monkeypatch):
    """W = U^-1 L^-1 [F_EK | r_E] and the Schur updates on the FP64 tensor
    path (inverted 32 x 32 diagonal blocks, hdg_ndblas.cuh; the switches
    DDHDG_ND_OWN_TRSM / DDHDG_ND_OWN_GEMM are read when a context builds
    its solver) against the same solve with cuBLAS's triangular solves and
    products:
    the same solution to round-off, on a mesh whose top fronts take the
    per-front LU path."""
    torch, g = _setup(2, 48, 2)
    tt, rhs, fl, dv = g.assemble_condense()
    n = g.sizes().n_trace_dofs
    xs = []
    for own in ("1", "0"):
        monkeypatch.setenv("DDHDG_ND_OWN_TRSM", own)
        monkeypatch.setenv("DDHDG_ND_OWN_GEMM", own)
        _, h = _setup(2, 48, 2)  # a fresh context builds its own solver
        x = torch.full((n,), float("nan"), dtype=torch.float64, device=g.device)
        _lib.check(h.L.ddhdg_solve_condensed(h._ctx, tt.data_ptr(), rhs.data_ptr(), fl.data_ptr(),
                                             dv.data_ptr(), x.data_ptr(), 0, h._sp()), "solve_condensed")
        torch.cuda.synchronize()
        xs.append(x.cpu().numpy())
    assert np.isfinite(xs[0]).all()
    assert np.abs(xs[0] - xs[1]).max() <= 1e-10 * np.abs(xs[1]).max()
