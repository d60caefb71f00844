"""Shared set-up of the GPU parity tests: the same problem and the same
(randomly perturbed) state in the CUDA solver and in the CPU oracle."""

import numpy as np

from oracle import oracle as O
from tests import cases


def make_pair(pb, prm, adim, seed=0, perturb=1e-3, thermo_start=True, enabled=(True, True, True)):
    from ddhdg_b200.solver import NPSolver

    o = O.OracleSolver(pb, prm, adim)
    o.set_enabled_components(*enabled)
    if thermo_start:
        o.compute_local_charge_neutrality()
        o.project_quasi_fermi(1)
        o.project_quasi_fermi(2)
    rng = np.random.default_rng(seed)
    scale = np.maximum(np.abs(o.cell_state).max(0, keepdims=True), 1e-3)
    o.cell_state += perturb * scale * rng.standard_normal(o.cell_state.shape)
    if thermo_start:
        # keep the carrier densities positive: near n + p = 0 the SRH
        # denominator cancels and amplifies round-off of any implementation
        d, nb = o.dim, o.nb
        for c in (1, 2):
            blk = o.cell_block(c)
            blk[:, d] = np.abs(blk[:, d]) + 1e-6
            o.trace_state[:, c] = np.abs(o.trace_state[:, c]) + 1e-6
    o.trace_state += perturb * rng.standard_normal(o.trace_state.shape) * \
        np.maximum(np.abs(o.trace_state).max(), 1e-3)
    g = NPSolver(pb, prm, adim)
    g.set_enabled_components(*enabled)
    g.set_state(o.cell_state, o.trace_state)
    return g, o


def rel_err(a, b, floor=1e-300):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), floor)
    return float(np.abs(a - b).max() / scale)
