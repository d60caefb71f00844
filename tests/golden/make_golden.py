"""Generates the golden fixtures of tests/golden from the CPU oracle (the
reference's per-cell algorithm restated; the reference itself cannot be
built here).  Seeded inputs; rerun to regenerate:

    python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from tests import cases  # noqa: E402

CASES = {
    # name: (dim, m, k, seed)
    "diode_1d_k2_m8": (1, 8, 2, 1),
    "diode_2d_k1_m4": (2, 4, 1, 2),
    "diode_2d_k2_m4": (2, 4, 2, 3),
    "diode_3d_k1_m2": (3, 2, 1, 4),
}


def perturbed_state(o, seed):
    """The local-charge-neutrality potential with projected equilibrium
    densities, perturbed by a seeded relative 1e-3 (densities kept
    positive)."""
    o.compute_local_charge_neutrality()
    o.project_quasi_fermi(1)
    o.project_quasi_fermi(2)
    rng = np.random.default_rng(seed)
    scale = np.maximum(np.abs(o.cell_state).max(0, keepdims=True), 1e-3)
    o.cell_state += 1e-3 * scale * rng.standard_normal(o.cell_state.shape)
    for c in (1, 2):
        blk = o.cell_block(c)
        blk[:, o.dim] = np.abs(blk[:, o.dim]) + 1e-6
        o.trace_state[:, c] = np.abs(o.trace_state[:, c]) + 1e-6
    o.trace_state += 1e-3 * rng.standard_normal(o.trace_state.shape) * max(np.abs(o.trace_state).max(), 1e-3)


def compute(name):
    dim, m, k, seed = CASES[name]
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    o = O.OracleSolver(pb, prm, adim)
    perturbed_state(o, seed)
    cell, trace = o.cell_state.copy(), o.trace_state.copy()
    _, _, flag, val = o.assemble_condense()
    tt, rhs = o.condense_accurate()
    s_tt, s_rhs = o.condense_term_scale
    b_tt, _ = o.condense_block_scale
    _, b_rhs = o.condense_solve_scale
    rng = np.random.default_rng(seed + 100)
    upd = 1e-3 * rng.standard_normal((o.nfaces, 3, o.nf)) * max(np.abs(o.trace_state).max(), 1e-3)
    du = o.reconstruct_accurate(upd)
    # per-block magnitudes of the summed terms: tt [comp][comp] (tt and the
    # Schur product), rhs [comp] (through the local solve), cell update
    # [comp][flux, scalar]
    return dict(cell=cell, trace=trace, tt=tt, rhs=rhs, dflag=flag, dval=val, s_tt=s_tt, s_rhs=s_rhs,
                b_tt=b_tt, b_rhs=b_rhs, b_du=o.reconstruct_block_scale,
                update_trace=upd, update_cell=du)


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **compute(name))
        print("wrote", name)
