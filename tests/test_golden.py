"""The oracle reproduces the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py from seeded inputs)."""

import os

import numpy as np
import pytest

from tests.golden import make_golden as mg

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(mg.CASES))
def test_oracle_reproduces_fixture(name):
    ref = np.load(os.path.join(HERE, name + ".npz"))
    got = mg.compute(name)
    assert np.array_equal(got["dflag"], ref["dflag"])
    for key in ("cell", "trace", "tt", "rhs", "dval", "update_cell", "b_tt", "b_rhs", "b_du"):
        scale = max(np.abs(ref[key]).max(), 1e-300)
        assert np.abs(got[key] - ref[key]).max() <= 1e-12 * scale, key
