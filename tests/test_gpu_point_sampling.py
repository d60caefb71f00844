"""get_solution_on_a_point (src/np_solver.cpp:1637-1700) on the device
(ddhdg_sample_points) against the oracle's point evaluation of the same
state: V, n, p at seeded points inside cells, on interior faces and outside
the mesh, and the quasi Fermi potentials (include/solver.h:343-376)."""

import numpy as np
import pytest

from oracle import oracle as O
from ddhdg_b200.problem import Component
from tests import cases
from tests.gpu_helpers import make_pair

pytestmark = pytest.mark.gpu


def _points(o, rng, n=200):
    d = o.dim
    lo = np.array(o.origin[:d])
    ext = np.array(o.n[:d]) * np.array(o.h[:d])
    inside = lo + rng.random((n, d)) * ext
    # on interior faces: a coordinate on a mesh line
    faces = inside.copy()
    ax = rng.integers(0, d, n)
    line = rng.integers(1, np.array(o.n[:d])[ax])
    faces[np.arange(n), ax] = lo[ax] + line * np.array(o.h[:d])[ax]
    outside = lo + (rng.random((8, d)) * 1.2 - 0.1) * ext
    pts = np.concatenate([inside, faces, outside])
    return np.concatenate([pts, np.zeros((pts.shape[0], 3 - d))], 1)


def _qf(c, V, dens, pb):
    """compute_quasi_fermi_potential (include/solver.h:343-376), physical
    units, at the diode's constant temperature."""
    U_T = 300.0 * O.KB / O.Q
    comp = Component(c)
    edge = pb.band_edge_energy[comp] * O.EV / O.Q
    if comp == Component.n:
        return V - edge - U_T * np.log(dens / pb.band_density[comp])
    return V - edge + U_T * np.log(dens / pb.band_density[comp])


@pytest.mark.parametrize("dim,k,m", [(2, 2, 8), (3, 1, 4), (1, 3, 16), (2, 1, 12)])
def test_point_values_match_oracle(dim, k, m):
    pb, prm, adim = cases.diode(dim=dim, m=m, k=k)
    g, o = make_pair(pb, prm, adim, seed=dim + 10 * k)
    pts = _points(o, np.random.default_rng(dim * 100 + k))
    for c in (Component.V, Component.n, Component.p):
        a = g.evaluate(c, pts)
        b = o.evaluate(int(c), pts)
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max(), c
    # one point through the single-point call
    assert abs(g.get_solution_on_a_point(pts[0], Component.V) - o.evaluate(0, pts[:1])[0]) <= \
        1e-13 * abs(o.evaluate(0, pts[:1])[0]) + 1e-300


def test_quasi_fermi_potentials_match_oracle():
    pb, prm, adim = cases.diode(dim=2, m=8, k=2)
    g, o = make_pair(pb, prm, adim, seed=3)
    pts = _points(o, np.random.default_rng(5))
    V = o.evaluate(0, pts)
    for c, comp in ((1, Component.phi_n), (2, Component.phi_p)):
        dens = o.evaluate(c, pts)
        with np.errstate(invalid="ignore"):
            ref = _qf(c, V, dens, pb)
        got = g.evaluate(comp, pts)
        # the perturbed density interpolates below zero at a few points: no
        # potential there, on either side
        ok = dens > 0
        assert ok.sum() > 0.9 * ok.size
        assert np.array_equal(np.isnan(got), ~ok), comp
        assert np.abs(got[ok] - ref[ok]).max() <= 1e-12 * np.abs(ref[ok]).max() + 1e-12, comp
