"""ctypes binding of ``libddhdg_b200.so`` (the C ABI declared in
``include/ddhdg_b200.h``).  The library is built in-tree; loading fails
loudly when it is missing -- there is no CPU fallback."""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libddhdg_b200.so")

c_int, c_double, c_int64, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p
dp = ctypes.POINTER(ctypes.c_double)
ip32 = ctypes.POINTER(ctypes.c_int32)

STATUS = {
    0: "ok", 1: "bad argument", 2: "out of memory", 3: "singular local pivot",
    4: "refinement stalled", 5: "timeout", 6: "CUDA error", 7: "not converged",
    8: "global solver error", 9: "no CUDA device",
}

# every exported entry point of the C ABI
EXPORTS = [
    "ddhdg_ctx_create", "ddhdg_ctx_destroy", "ddhdg_get_sizes", "ddhdg_set_boundary",
    "ddhdg_set_enabled", "ddhdg_assemble_condense", "ddhdg_scatter", "ddhdg_get_csr",
    "ddhdg_solve_trace", "ddhdg_reconstruct", "ddhdg_newton", "ddhdg_last_timings",
    "ddhdg_project_cell", "ddhdg_project_trace", "ddhdg_project_density",
    "ddhdg_reference_points", "ddhdg_last_error", "ddhdg_assemble_condense_noalloc",
    "ddhdg_solve_condensed", "ddhdg_assemble_condense_host", "ddhdg_reconstruct_host",
    "ddhdg_set_solver_graphs", "ddhdg_local_cell_system", "ddhdg_assemble_condense_plain",
    "ddhdg_reconstruct_plain", "ddhdg_sample_points", "ddhdg_batch_create", "ddhdg_batch_destroy",
    "ddhdg_batch_condense", "ddhdg_batch_reconstruct", "ddhdg_batch_set_shape", "ddhdg_batch_get_shape",
    "ddhdg_batch_autotune", "ddhdg_batch_newton_step", "ddhdg_trace_solver_bytes", "ddhdg_release_solver",
    "ddhdg_batch_newton_step_begin", "ddhdg_batch_newton_step_end",
]


class ProblemDesc(ctypes.Structure):
    _fields_ = [
        ("dim", c_int), ("degree", c_int), ("n", c_int * 3),
        ("origin", c_double * 3), ("h", c_double * 3),
        ("enabled", c_int * 3), ("flux", c_int), ("phi_linearize", c_int),
        ("jacobian_fix", c_int), ("precision", c_int),
        ("eps", c_double), ("mu_n", c_double), ("mu_p", c_double),
        ("temperature", c_double), ("thermal_voltage_rescale", c_double),
        ("V_rescale", c_double), ("n_rescale", c_double), ("rec_rescale", c_double),
        ("nc", c_double), ("nv", c_double), ("ec_eV", c_double), ("ev_eV", c_double),
        ("rec_type", c_int), ("srh_ni", c_double), ("srh_tau_n", c_double), ("srh_tau_p", c_double),
        ("rec_a_host", dp), ("rec_b_host", dp), ("rec_c_host", dp),
        ("doping_host", dp), ("tau", c_double * 3), ("tau_host", dp),
        ("face_bc_host", ip32), ("face_bc_val_host", dp),
    ]


class Sizes(ctypes.Structure):
    _fields_ = [
        ("ncells", c_int64), ("nfaces", c_int64), ("Nc_all", c_int), ("Nt", c_int),
        ("ncomp", c_int), ("nqc", c_int), ("nqf", c_int), ("nb", c_int), ("nf", c_int),
        ("n_trace_dofs", c_int64), ("nnz", c_int64),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("ctx", c_void_p), ("cell_state", c_void_p), ("trace_state", c_void_p),
        ("tt", c_void_p), ("rhs", c_void_p), ("dflag", c_void_p), ("dval", c_void_p),
        ("update_trace", c_void_p), ("update_cell", c_void_p),
    ]


_lib = None


class DDHDGError(RuntimeError):
    def __init__(self, code, where, msg=""):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} ({msg})")


def load(build_if_missing: bool = True):
    """Load the CUDA library (building it with nvcc when missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise OSError(f"{LIB_PATH} is missing; run ddhdg_b200.build.build()")
        from . import build as _b

        _b.build()
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    L.ddhdg_ctx_create.argtypes = [P(ProblemDesc), P(c_void_p)]
    L.ddhdg_ctx_destroy.argtypes = [c_void_p]
    L.ddhdg_get_sizes.argtypes = [c_void_p, c_int, P(Sizes)]
    L.ddhdg_set_boundary.argtypes = [c_void_p, ip32, dp]
    L.ddhdg_set_enabled.argtypes = [c_void_p, c_int, c_int, c_int]
    L.ddhdg_assemble_condense.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_void_p]
    L.ddhdg_assemble_condense_noalloc.argtypes = L.ddhdg_assemble_condense.argtypes
    L.ddhdg_scatter.argtypes = [c_void_p] + [c_void_p] * 6 + [c_int, c_void_p]
    L.ddhdg_get_csr.argtypes = [c_void_p, c_int, P(c_void_p), P(c_void_p)]
    L.ddhdg_solve_trace.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]
    L.ddhdg_solve_condensed.argtypes = [c_void_p] * 6 + [c_int, c_void_p]
    L.ddhdg_reconstruct.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]
    L.ddhdg_assemble_condense_host.argtypes = L.ddhdg_assemble_condense.argtypes
    L.ddhdg_reconstruct_host.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    L.ddhdg_set_solver_graphs.argtypes = [c_void_p, c_int]
    L.ddhdg_trace_solver_bytes.argtypes = [c_int, P(c_int), c_int, c_int, P(c_int64)]
    L.ddhdg_release_solver.argtypes = [c_void_p, c_int]
    L.ddhdg_local_cell_system.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int64, c_void_p,
                                          c_int64] + [c_void_p] * 7
    L.ddhdg_assemble_condense_plain.argtypes = L.ddhdg_assemble_condense.argtypes
    L.ddhdg_reconstruct_plain.argtypes = L.ddhdg_reconstruct.argtypes
    L.ddhdg_sample_points.argtypes = [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_void_p, c_void_p]
    L.ddhdg_batch_create.argtypes = [P(BatchItem), c_int, c_int, P(c_void_p)]
    L.ddhdg_batch_destroy.argtypes = [c_void_p]
    L.ddhdg_batch_condense.argtypes = [c_void_p, c_void_p]
    L.ddhdg_batch_reconstruct.argtypes = [c_void_p, c_void_p]
    L.ddhdg_batch_set_shape.argtypes = [c_void_p, P(c_int), c_int]
    L.ddhdg_batch_get_shape.argtypes = [c_void_p, P(c_int), P(c_int), P(c_int), P(c_int)]
    L.ddhdg_batch_autotune.argtypes = [c_void_p, c_int, P(ctypes.c_float), c_void_p]
    L.ddhdg_batch_newton_step.argtypes = [c_void_p, dp, dp, P(c_int), c_void_p]
    L.ddhdg_batch_newton_step_begin.argtypes = [c_void_p, dp, c_void_p]
    L.ddhdg_batch_newton_step_end.argtypes = [c_void_p, c_int, dp, P(c_int), P(c_int)]
    L.ddhdg_newton.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_double, c_double, c_int,
                               c_double, P(c_int), P(c_double), c_void_p]
    L.ddhdg_last_timings.argtypes = [c_void_p, P(c_double), P(c_double), P(c_double), P(c_int)]
    L.ddhdg_project_cell.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    L.ddhdg_project_trace.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    L.ddhdg_project_density.argtypes = [c_void_p, c_int, c_double, c_void_p, c_void_p, c_void_p]
    L.ddhdg_reference_points.argtypes = [c_int, c_int, dp, dp, dp]
    L.ddhdg_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(code, where):
    if code != 0:
        msg = _lib.ddhdg_last_error().decode() if _lib is not None else ""
        raise DDHDGError(code, where, msg)
    return code
