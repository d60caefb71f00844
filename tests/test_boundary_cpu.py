"""CPU-side checks of the C ABI library: it loads without a GPU and exports
every entry point that include/ddhdg_b200.h declares."""

import ctypes
import os
import re

import numpy as np
import pytest

from ddhdg_b200 import _lib
from ddhdg_b200.build import LIB

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ddhdg_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(ddhdg_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first (python __graft_entry__.py or ddhdg_b200/build.py)"
    L = ctypes.CDLL(LIB)
    decl = declared_symbols()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(_lib.EXPORTS) == decl


def test_reference_points_without_gpu():
    L = _lib.load(build_if_missing=False)
    dp = ctypes.POINTER(ctypes.c_double)
    for dim, k in ((1, 1), (2, 2), (3, 1), (2, 3)):
        nq = (k + 1) ** dim
        nqf = (k + 1) ** (dim - 1)
        qc = np.zeros((nq, 3))
        qf = np.zeros((2 * dim, nqf, 3))
        sup = np.zeros(k + 1)
        assert L.ddhdg_reference_points(dim, k, qc.ctypes.data_as(dp), qf.ctypes.data_as(dp),
                                        sup.ctypes.data_as(dp)) == 0
        g, _ = np.polynomial.legendre.leggauss(k + 1)
        assert np.allclose(np.sort(np.unique(np.round(qc[:, 0], 14))), np.sort(0.5 * (g + 1)))
        assert sup[0] == 0.0 and sup[-1] == 1.0
        for f in range(2 * dim):
            assert np.all(qf[f, :, f // 2] == (f % 2))


def test_ctx_create_without_device_fails_cleanly():
    L = _lib.load(build_if_missing=False)
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    D = _lib.ProblemDesc()
    ctx = ctypes.c_void_p()
    assert L.ddhdg_ctx_create(ctypes.byref(D), ctypes.byref(ctx)) != 0
    assert not ctx


def test_argument_checks_before_any_device_work():
    """Null contexts and invalid descriptors are rejected with a bad-argument
    status and a message, before any CUDA call (so also on a machine without
    a GPU): the host-buffer calls, the trace solve and its graph switch; a
    precision other than 0 / 1, mixed precision where no FP32 kernel exists
    (2D degree 3), and meshes of 2^31 cells or more."""
    L = _lib.load(build_if_missing=False)
    vp = ctypes.c_void_p
    null = vp()
    assert L.ddhdg_set_solver_graphs(null, 1) == 1
    assert L.ddhdg_assemble_condense_host(null, null, null, 0, null, null, null, null, null) == 1
    assert L.ddhdg_reconstruct_host(null, null, 0, null, null) == 1
    assert L.ddhdg_solve_condensed(null, null, null, null, null, null, 0, null) == 1

    def create(**kw):
        D = _lib.ProblemDesc()
        D.dim, D.degree = kw.get("dim", 2), kw.get("degree", 1)
        for a in range(3):
            D.n[a] = kw.get("n", 4)
            D.h[a] = 1.0
        D.precision = kw.get("precision", 0)
        ctx = vp()
        rc = L.ddhdg_ctx_create(ctypes.byref(D), ctypes.byref(ctx))
        return rc, L.ddhdg_last_error().decode()

    rc, msg = create(precision=2)
    assert rc == 1 and "precision" in msg
    rc, msg = create(degree=3, precision=1)
    assert rc == 1 and "mixed precision" in msg
    rc, msg = create(n=50000)
    assert rc == 1 and "2^31" in msg
