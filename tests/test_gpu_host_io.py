"""The host-buffer calls (ddhdg_assemble_condense_host, ddhdg_reconstruct_host)
against the device-array calls on the same state: the chunked copies and
launches change no per-cell arithmetic, so every output is bitwise equal.
Page-locked and pageable host memory, two states in a row, FP64 and mixed."""

import numpy as np
import pytest

from ddhdg_b200.problem import Precision
from tests import cases
from tests.gpu_helpers import make_pair

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    return torch


def _host(torch, arr, pinned):
    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64).reshape(-1).copy())
    return t.pin_memory() if pinned else t


@pytest.mark.parametrize("dim,k,m,prec,pinned", [
    (2, 2, 12, Precision.fp64, True),
    (2, 2, 12, Precision.fp64, False),
    (3, 1, 4, Precision.fp64, True),
    (2, 1, 10, Precision.mixed, True),
])
def test_host_calls_match_device_calls(dim, k, m, prec, pinned):
    torch = _torch()
    from ddhdg_b200 import _lib

    pb, prm, adim = cases.diode(dim=dim, m=m, k=k, precision=prec)
    g, o = make_pair(pb, prm, adim, seed=7 + dim * 10 + k)
    L = g.L
    rng = np.random.default_rng(11)
    s = g.sizes()
    nc, Nt = g.ncells, s.Nt
    for rep in range(2):
        if rep == 1:
            # a second, different state through the same context
            cell = g.get_cell_state() * (1 + 1e-3 * rng.standard_normal(g.get_cell_state().shape))
            g.set_state(cell, g.get_trace_state())
        tt, rhs, fl, dv = g.assemble_condense()
        upd = 1e-3 * rng.standard_normal((g.nfaces, 3, g.nf))
        dcell = g.reconstruct(upd)
        torch.cuda.synchronize()
        hcell = _host(torch, g.get_cell_state(), pinned)
        htrace = _host(torch, g.get_trace_state(), pinned)
        hupd = _host(torch, upd, pinned)
        hout = torch.full((nc * g.Nc_all,), np.nan, dtype=torch.float64)
        hout = hout.pin_memory() if pinned else hout
        tt2 = torch.empty(nc * Nt * Nt, dtype=torch.float64, device=g.device)
        rhs2 = torch.empty(nc * Nt, dtype=torch.float64, device=g.device)
        fl2 = torch.empty(nc * Nt, dtype=torch.int32, device=g.device)
        dv2 = torch.empty(nc * Nt, dtype=torch.float64, device=g.device)
        _lib.check(L.ddhdg_assemble_condense_host(g._ctx, hcell.data_ptr(), htrace.data_ptr(), 0,
                                                  tt2.data_ptr(), rhs2.data_ptr(), fl2.data_ptr(),
                                                  dv2.data_ptr(), g._sp()), "assemble_condense_host")
        _lib.check(L.ddhdg_reconstruct_host(g._ctx, hupd.data_ptr(), 0, hout.data_ptr(), g._sp()),
                   "reconstruct_host")
        g.stream.synchronize()
        torch.cuda.synchronize()
        assert torch.equal(tt2.view(nc, Nt, Nt), tt)
        assert torch.equal(rhs2.view(nc, Nt), rhs)
        assert torch.equal(fl2.view(nc, Nt), fl)
        assert torch.equal(dv2.view(nc, Nt), dv)
        assert np.array_equal(hout.numpy().reshape(nc, g.Nc_all), dcell.cpu().numpy())


def test_reconstruct_host_needs_a_condensed_state():
    torch = _torch()
    from ddhdg_b200._lib import DDHDGError, check
    from ddhdg_b200.solver import NPSolver

    pb, prm, adim = cases.diode(dim=2, m=4, k=1)
    g = NPSolver(pb, prm, adim)
    upd = torch.zeros(g.nfaces * 3 * g.nf, dtype=torch.float64)
    out = torch.zeros(g.ncells * g.Nc_all, dtype=torch.float64)
    with pytest.raises(DDHDGError, match="preceding ddhdg_assemble_condense_host"):
        check(g.L.ddhdg_reconstruct_host(g._ctx, upd.data_ptr(), 0, out.data_ptr(), g._sp()),
              "reconstruct_host")
