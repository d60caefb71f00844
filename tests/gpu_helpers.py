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


def block_rel_errs(tt, rhs, S, g, o, thermo=False):
    """Largest error of each (row component, column component) block of the
    condensed tt, and of each component block of rhs, relative to the
    magnitude of the terms summed inside that block; call
    ``o.condense_accurate`` first.  The small coupling blocks (p rows against
    n columns are ~1e-4 of the V-n block) are thus checked at their own
    scale, not at the largest block's.

    tt blocks: the summed terms tt and tc cc^-1 ct (``condense_block_scale``).
    rhs blocks: the summed terms through the local solve, |tr| + |tc| |cc^-1|
    |cc_rhs| (``condense_solve_scale``): in 3D Dirichlet cells cc^-1 cc_rhs
    is itself a cancellation of terms ~4e6 times larger than the V block of
    the result, which no FP64 solve resolves below ~1e-9 of that block.
    A block that vanishes in exact arithmetic (V rows against n columns with
    phi_linearize) holds only round-off of the other blocks: its scale is
    floored at 1e-8 of the largest block's, so it is checked to 1e-18 of
    that.  Returns (worst tt ratio, worst rhs ratio, per-block table)."""
    tt = np.asarray(tt).reshape(S.shape)
    rhs = np.asarray(rhs).reshape(g.shape)
    bt, br = o.condense_block_scale
    _, sr = o.condense_solve_scale
    bt = np.maximum(bt, 1e-8 * bt.max())
    sr = np.maximum(sr, 1e-8 * sr.max())
    ncomp = bt.shape[0]
    comp = (np.arange(S.shape[1]) // o.nf) % ncomp
    table = {}
    e_tt = e_rhs = 0.0
    for a in range(ncomp):
        ra = comp == a
        d = np.abs(rhs[:, ra] - g[:, ra]).max()
        er = float(d / max(sr[a], 1e-300))
        table[f"rhs[{a}]"] = er
        table[f"rhs[{a}] (schur terms only)"] = float(d / max(br[a], 1e-300))
        e_rhs = max(e_rhs, er)
        for b in range(ncomp):
            cb = comp == b
            d = np.abs(tt[:, ra][:, :, cb] - S[:, ra][:, :, cb]).max()
            e = float(d / max(bt[a, b], 1e-300))
            table[f"tt[{a},{b}]"] = e
            e_tt = max(e_tt, e)
    return e_tt, e_rhs, table


def cell_block_rel_err(du, acc, o):
    """Largest error of the reconstructed cell update over the blocks
    (component x {flux, scalar}), each relative to the magnitude of the
    terms summed in that block (the oracle's ``reconstruct_block_scale``;
    call ``reconstruct_accurate`` first).  Returns (worst ratio, table)."""
    d, nb = o.dim, o.nb
    a = np.asarray(du).reshape(o.ncells, 3, d + 1, nb)
    b = np.asarray(acc).reshape(o.ncells, 3, d + 1, nb)
    sc = o.reconstruct_block_scale
    table = {}
    worst = 0.0
    for c in range(3):
        for j, (name, sl) in enumerate((("flux", slice(0, d)), ("scalar", slice(d, d + 1)))):
            if sc[c, j] == 0.0:
                continue
            e = float(np.abs(a[:, c, sl] - b[:, c, sl]).max() / sc[c, j])
            table[f"{'Vnp'[c]} {name}"] = e
            worst = max(worst, e)
    return worst, table
