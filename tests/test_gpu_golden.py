"""The CUDA path against the committed golden fixtures (oracle outputs on
seeded diodes, tests/golden): condensed blocks, Dirichlet data and the
reconstructed cell update, through the C ABI.  Every (row component, column
component) block of tt, every component block of rhs and every (component,
flux/scalar) block of the cell update is checked at 1e-10 relative to the
magnitude of the terms summed inside that block (stored in the fixture)."""

import os

import numpy as np
import pytest

from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-10


@pytest.mark.parametrize("name", sorted(mg.CASES))
def test_gpu_matches_fixture(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    ref = np.load(os.path.join(HERE, name + ".npz"))
    dim, m, k, _ = mg.CASES[name]
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g = NPSolver(pb, prm, adim)
    g.set_state(ref["cell"], ref["trace"])
    tt, rhs, flag, val = g.assemble_condense()
    assert np.array_equal(flag.cpu().numpy(), ref["dflag"])
    tt, rhs = tt.cpu().numpy().reshape(ref["tt"].shape), rhs.cpu().numpy().reshape(ref["rhs"].shape)
    b_tt, b_rhs = ref["b_tt"], ref["b_rhs"]
    ncomp = b_tt.shape[0]
    nf = (k + 1) ** (dim - 1)
    comp = (np.arange(ref["tt"].shape[1]) // nf) % ncomp
    for a in range(ncomp):
        ra = comp == a
        e = np.abs(rhs[:, ra] - ref["rhs"][:, ra]).max() / b_rhs[a]
        assert e < TOL, (f"rhs[{a}]", e)
        for b in range(ncomp):
            cb = comp == b
            e = np.abs(tt[:, ra][:, :, cb] - ref["tt"][:, ra][:, :, cb]).max() / b_tt[a, b]
            assert e < TOL, (f"tt[{a},{b}]", e)
    floor = np.abs(ref["trace"]).max()
    assert np.abs(val.cpu().numpy() - ref["dval"]).max() <= TOL * max(np.abs(ref["dval"]).max(), floor)
    du = g.reconstruct(ref["update_trace"]).cpu().numpy()
    nb = (k + 1) ** dim
    a_ = du.reshape(-1, 3, dim + 1, nb)
    b_ = ref["update_cell"].reshape(-1, 3, dim + 1, nb)
    for c in range(3):
        for j, sl in enumerate((slice(0, dim), slice(dim, dim + 1))):
            e = np.abs(a_[:, c, sl] - b_[:, c, sl]).max() / ref["b_du"][c, j]
            assert e < TOL, ("update", c, j, e)
