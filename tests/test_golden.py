"""The committed golden fixtures (tests/golden, made by make_golden.py from
the oracle after it passed the known-answer tests) still equal the oracle's
output: a change of the oracle shows up here before it can move the GPU
parity tests."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

import make_golden  # noqa: E402


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_reproduces_golden(name):
    want = np.load(os.path.join(HERE, name + ".npz"))
    rows, walk, names, _ = make_golden.compute(name)
    assert list(want["names"]) == names
    np.testing.assert_array_equal(rows, want["rows"])
    np.testing.assert_array_equal(walk, want["walk"])
