"""ddhdg_assemble_condense_noalloc (static device scratch, no allocation in
the call) against ddhdg_assemble_condense, through the C ABI.

Collected last, so that it runs both after the other GPU tests and alone."""

import ctypes

import numpy as np
import pytest

from ddhdg_b200 import _lib
from ddhdg_b200.problem import DDFluxType, Precision
from tests import cases
from tests.gpu_helpers import make_pair

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 16 << 20


def _outputs(torch, nc, Nt, device):
    return (torch.empty(nc * Nt * Nt, dtype=torch.float64, device=device),
            torch.empty(nc * Nt, dtype=torch.float64, device=device),
            torch.empty(nc * Nt, dtype=torch.int32, device=device),
            torch.empty(nc * Nt, dtype=torch.float64, device=device))


def _noalloc(g, thermo, outs):
    tt, rhs, dflag, dval = outs
    return g.L.ddhdg_assemble_condense_noalloc(g._ctx, g.cell_state.data_ptr(), g.trace_state.data_ptr(),
                                               int(thermo), tt.data_ptr(), rhs.data_ptr(),
                                               dflag.data_ptr(), dval.data_ptr(), g._sp())


CELL, QS = DDFluxType.use_cell, DDFluxType.qiu_shi_stabilization


FP64, MIXED = Precision.fp64, Precision.mixed


# 3D k = 2 with the drift columns keeps R outside shared memory, so both
# parts of the scratch are exercised; a mixed-precision context must run the
# same FP32-Jacobian kernel as ddhdg_assemble_condense
@pytest.mark.parametrize("dim,m,k,flux,prec", [(2, 8, 2, CELL, FP64), (2, 6, 1, QS, FP64),
                                               (3, 2, 2, QS, FP64), (2, 4, 3, CELL, FP64),
                                               (1, 8, 2, CELL, FP64), (2, 8, 2, CELL, MIXED),
                                               (3, 3, 1, QS, MIXED)])
def test_noalloc_matches_assemble_condense_twice(dim, m, k, flux, prec):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k, flux=flux)
    prm.precision = prec
    g, _ = make_pair(pb, prm, adim)
    for thermo in (False, True):
        ref = [t.reshape(-1).cpu().numpy() for t in g.assemble_condense(thermo)]
        nc, Nt = g.ncells, g.sizes(thermo).Nt
        for call in range(2):
            outs = _outputs(torch, nc, Nt, g.device)
            for t in outs:
                t.fill_(7)  # every output element must be written
            _lib.check(_noalloc(g, thermo, outs), "assemble_condense_noalloc")
            torch.cuda.synchronize()
            got = [t.cpu().numpy() for t in outs]
            scale_tt = max(np.abs(ref[0]).max(), 1e-300)
            scale_rhs = max(np.abs(ref[1]).max(), 1e-300)
            assert np.abs(got[0] - ref[0]).max() <= 1e-12 * scale_tt, (thermo, call)
            assert np.abs(got[1] - ref[1]).max() <= 1e-12 * scale_rhs, (thermo, call)
            assert np.array_equal(got[2], ref[2]), (thermo, call)
            assert np.array_equal(got[3], ref[3]), (thermo, call)


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from ddhdg_b200.solver import NPSolver

    # 2D k = 2, three components: 27 x 37 doubles of Y cache per cell, so
    # 48 x 48 cells need more than 16 MiB
    pb, prm, adim = cases.diode(dim=2, m=48, k=2)
    g = NPSolver(pb, prm, adim)
    nc, Nt = g.ncells, g.sizes(False).Nt
    assert nc * 27 * 37 * 8 > NOALLOC_BYTES
    outs = _outputs(torch, nc, Nt, g.device)
    code = _noalloc(g, False, outs)
    assert code == 1, code  # DDHDG_BAD_ARG
    msg = g.L.ddhdg_last_error().decode()
    assert "bytes of condensation scratch" in msg and str(NOALLOC_BYTES) in msg, msg


def test_noalloc_warm_calls_leave_device_memory_unchanged():
    """The point of the entry point: after a first call (which may load the
    kernel's module), further calls take no device memory at all."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    pb, prm, adim = cases.diode(dim=2, m=8, k=2)
    g, _ = make_pair(pb, prm, adim)
    nc, Nt = g.ncells, g.sizes(False).Nt
    outs = _outputs(torch, nc, Nt, g.device)
    _lib.check(_noalloc(g, False, outs), "assemble_condense_noalloc")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(g.device)
    for _ in range(3):
        _lib.check(_noalloc(g, False, outs), "assemble_condense_noalloc")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(g.device)
    assert free1 == free0, (free0, free1)
