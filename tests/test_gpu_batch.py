"""Batched condensation (one persistent launch over many devices of
different mesh sizes and degrees, ddhdg_batch_*): every device's outputs
are bitwise those of its own single-context call (ddhdg_assemble_condense /
ddhdg_reconstruct), whatever the tile shape; and one batch checked directly
against the oracle per block."""

import numpy as np
import pytest

from ddhdg_b200 import workloads
from tests.gpu_helpers import block_rel_errs, make_pair

pytestmark = pytest.mark.gpu


def _solvers(specs, seed=0):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    out = []
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for pb, prm, adim, _ in specs:
        g = NPSolver(pb, prm, adim)
        g.compute_local_charge_neutrality()
        for c in (1, 2):
            g.L.ddhdg_project_density(g._ctx, c, 0.0, g.cell_state.data_ptr(), g.trace_state.data_ptr(), g._sp())
        # a seeded relative perturbation: a state away from equilibrium
        g.cell_state.mul_(1 + 1e-3 * torch.randn(g.cell_state.shape, generator=gen, device="cuda",
                                                  dtype=torch.float64))
        g.trace_state.mul_(1 + 1e-3 * torch.randn(g.trace_state.shape, generator=gen, device="cuda",
                                                  dtype=torch.float64))
        out.append(g)
    return out


def _check_bitwise(batch, solvers, thermo=False, seed=1):
    import torch

    batch.condense()
    torch.cuda.synchronize()
    got = [(batch.tt[i].cpu().numpy(), batch.rhs[i].cpu().numpy(), batch.dflag[i].cpu().numpy(),
            batch.dval[i].cpu().numpy()) for i in range(len(solvers))]
    rng = np.random.default_rng(seed)
    for i, g in enumerate(solvers):
        batch.update_trace[i].copy_(torch.as_tensor(1e-3 * rng.standard_normal(g.nfaces * 3 * g.nf)))
    batch.reconstruct()
    torch.cuda.synchronize()
    for i, g in enumerate(solvers):
        ref = [t.cpu().numpy() for t in g.assemble_condense(thermo)]
        for a, b, name in zip(got[i], ref, ("tt", "rhs", "dflag", "dval")):
            assert np.array_equal(a, b), (i, name, g.k, g.ncells)
        du = g.reconstruct(batch.update_trace[i], thermo).cpu().numpy()
        assert np.array_equal(batch.update_cell[i].cpu().numpy(), du), (i, "update_cell")


def test_heterogeneous_batch_is_bitwise_the_single_context_result():
    from ddhdg_b200.batch import CondenseBatch

    specs = workloads.batch_diodes(9, seed=11, sizes=(6, 20))
    assert {s[3]["k"] for s in specs} == {1, 2, 3}
    solvers = _solvers(specs)
    batch = CondenseBatch(solvers)
    _check_bitwise(batch, solvers)
    # other tile shapes, then the autotuned one: the same bits
    batch.set_shape({1: 4, 2: 8, 3: 1}, 1)
    _check_bitwise(batch, solvers)
    batch.set_shape({1: 256, 2: 128, 3: 32}, 2)
    _check_bitwise(batch, solvers)
    ms = batch.autotune(reps=2)
    assert ms > 0
    sh = batch.shape()
    assert sh["tiles"] > 0 and sh["grid"] > 0
    _check_bitwise(batch, solvers)
    batch.close()


def test_thermodynamic_equilibrium_batch():
    from ddhdg_b200.batch import CondenseBatch

    specs = workloads.batch_diodes(5, seed=12, sizes=(6, 14))
    solvers = _solvers(specs, seed=3)
    batch = CondenseBatch(solvers, thermo=True)
    _check_bitwise(batch, solvers, thermo=True)


@pytest.mark.parametrize("dim,degrees", [(1, (1, 2, 3)), (3, (1, 2))])
def test_batches_in_1d_and_3d(dim, degrees):
    from ddhdg_b200.batch import CondenseBatch

    sizes = (8, 40) if dim == 1 else (2, 4)
    specs = workloads.batch_diodes(6, seed=dim, sizes=sizes, degrees=degrees, dim=dim)
    solvers = _solvers(specs, seed=dim)
    batch = CondenseBatch(solvers)
    _check_bitwise(batch, solvers)


def test_batch_against_the_oracle():
    """Two devices of different size and degree in one launch, against the
    oracle per component block (1e-10, as in test_gpu_parity)."""
    from ddhdg_b200.batch import CondenseBatch
    from ddhdg_b200 import workloads as w

    pairs = [make_pair(*w.diode(dim=2, m=6, k=2, N_D=3e22, N_A=3e22, x_j=0.4), seed=5),
             make_pair(*w.diode(dim=2, m=4, k=3), seed=6),
             make_pair(*w.diode(dim=2, m=8, k=1, N_D=2e21, N_A=2e21, x_j=0.6), seed=7)]
    batch = CondenseBatch([g for g, _ in pairs])
    batch.condense()
    for i, (g, o) in enumerate(pairs):
        S, gv = o.condense_accurate()
        e_tt, e_rhs, table = block_rel_errs(batch.tt[i].cpu().numpy(), batch.rhs[i].cpu().numpy(), S, gv, o)
        assert max(e_tt, e_rhs) < 1e-10, (i, table)
        assert np.array_equal(batch.dflag[i].cpu().numpy(), o.assemble_condense()[2])


def test_batch_rejects_mixed_dimensions():
    from ddhdg_b200._lib import DDHDGError
    from ddhdg_b200.batch import CondenseBatch

    a = _solvers([workloads.diode(dim=2, m=4, k=1) + ({},)])
    b = _solvers([workloads.diode(dim=1, m=8, k=1) + ({},)])
    with pytest.raises(DDHDGError, match="one dimension"):
        CondenseBatch(a + b)


@pytest.mark.parametrize("dim,sizes,degrees", [(2, (6, 20), (1, 2, 3)), (3, (2, 4), (1, 2)), (2, (6, 20), (1, 2))])
def test_mixed_precision_devices_in_a_batch(dim, sizes, degrees):
    """FP64 and mixed-precision devices in one launch (or mixed ones only,
    which take the kernel built for four CTAs per SM): each device's outputs
    are bitwise those of its own context (the mixed ones from the FP32-
    Jacobian kernel), whatever the tile shape."""
    from ddhdg_b200.batch import CondenseBatch

    specs = workloads.batch_diodes(8, seed=20 + dim, sizes=sizes, degrees=degrees, dim=dim, mixed=True)
    precs = {s[3]["precision"] for s in specs}
    assert precs == ({0, 1} if 3 in degrees or dim == 3 else {1})
    solvers = _solvers(specs, seed=4)
    batch = CondenseBatch(solvers)
    _check_bitwise(batch, solvers)
    batch.set_shape({1: 4, 2: 8, 3: 1}, 1)
    _check_bitwise(batch, solvers)
    batch.close()


def test_newton_step_in_two_halves():
    """newton_step_begin / newton_step_end give the bits of newton_step, and
    two batches with steps in flight at the same time do not disturb each
    other (the serving loop drives its groups this way)."""
    from ddhdg_b200.batch import CondenseBatch

    specs = workloads.batch_diodes(4, seed=31, sizes=(8, 16), degrees=(1, 2))
    a_solvers = _solvers(specs, seed=5)
    b_solvers = _solvers(specs, seed=5)
    A = CondenseBatch(a_solvers)
    B = CondenseBatch(b_solvers[:2])
    C = CondenseBatch(b_solvers[2:])
    for _ in range(3):
        nA, sA = A.newton_step([0.5] * 4)
        B.newton_step_begin([0.5] * 2)
        C.newton_step_begin([0.5] * 2)
        rc = None
        while rc is None:
            rc = C.newton_step_end(wait=False)
        nB, sB = B.newton_step_end(wait=True)
        nC, sC = rc
        assert sA == sB + sC == [0, 0, 0, 0]
        assert np.array_equal(nA[:2], nB) and np.array_equal(nA[2:], nC)
    for g, h in zip(a_solvers, b_solvers):
        assert np.array_equal(g.get_cell_state(), h.get_cell_state())
        assert np.array_equal(g.get_trace_state(), h.get_trace_state())
    for b in (A, B, C):
        b.close()
