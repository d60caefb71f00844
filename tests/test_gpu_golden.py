"""The CUDA path against the committed golden fixtures (oracle outputs on
seeded diodes, tests/golden): condensed blocks, Dirichlet data and the
reconstructed cell update, through the C ABI."""

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
    s_tt, s_rhs = float(ref["s_tt"]), float(ref["s_rhs"])
    e_tt = np.abs(tt.cpu().numpy() - ref["tt"]).max() / max(np.abs(ref["tt"]).max(), s_tt)
    e_rhs = np.abs(rhs.cpu().numpy() - ref["rhs"]).max() / max(np.abs(ref["rhs"]).max(), s_rhs)
    assert e_tt < TOL, e_tt
    assert e_rhs < TOL, e_rhs
    floor = np.abs(ref["trace"]).max()
    assert np.abs(val.cpu().numpy() - ref["dval"]).max() <= TOL * max(np.abs(ref["dval"]).max(), floor)
    du = g.reconstruct(ref["update_trace"]).cpu().numpy()
    assert np.abs(du - ref["update_cell"]).max() <= TOL * np.abs(ref["update_cell"]).max()
