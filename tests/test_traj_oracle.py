"""The CPU restatement of the trajectory post-processing (oracle/traj_ref.py)
against the reference's own step_tracker (golden vectors made by running it,
tests/golden/make_steps_golden.py) and against closed-form MSD cases."""
import os

import numpy as np

from oracle import traj_ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "steps_golden.npz")


def test_steps_match_reference_step_tracker():
    g = np.load(GOLDEN)
    assert list(g["out_dtypes"]) == ["float32", "float32", "float64", "float64", "float64"]
    xs, ys, dx, dy, ln, order = traj_ref.steps(g["particle"], g["x"], g["y"], float(g["pixel_size"]))
    np.testing.assert_array_equal(xs, g["out_x"])
    np.testing.assert_array_equal(ys, g["out_y"])
    # step_tracker assigns its groupby-ordered lists by position
    np.testing.assert_array_equal(dx, g["x_step"])
    np.testing.assert_array_equal(dy, g["y_step"])
    np.testing.assert_array_equal(ln, g["steplength"])
    # the golden table is frame-ordered with interleaved ids: the positional
    # assignment is not the per-row step
    assert not np.array_equal(order, np.arange(len(order)))


def test_filter_stubs_counts():
    ids = np.array([3, 1, 3, 2, 3, 1, 7])
    np.testing.assert_array_equal(traj_ref.filter_stubs(ids, 2), [1, 1, 1, 0, 1, 1, 0])
    np.testing.assert_array_equal(traj_ref.filter_stubs(ids, 3), [1, 0, 1, 0, 1, 0, 0])
    assert traj_ref.filter_stubs(ids, 0).all()


def test_msd_uniform_motion_and_gaps():
    # x = 2 f exactly (a power-of-two pixel size keeps every value exact):
    # msd(L) = (2 L mpp)^2 whatever the gaps
    f = np.array([0, 1, 2, 4, 5, 8], np.int64)
    x = (2.0 * f).astype(np.float32)
    y = np.zeros_like(x)
    ids = np.zeros(len(f), np.int64)
    out = traj_ref.imsd(ids, f, x, y, 0.5, 100)
    lags = out[:, 0].astype(int)
    # span 9 frames: lags 1..8; lag 5 has no pair (f, f+5 both present: 0-5? yes 0,5; ...)
    for lag, pid, v in out:
        assert v == np.float32((2 * lag * 0.5) ** 2)
    present = set(f.tolist())
    want = [L for L in range(1, 9) if any(a in present and a + L in present for a in range(9))]
    assert lags.tolist() == want


def test_msd_order_and_max_lagtime():
    rng = np.random.default_rng(0)
    rows = []
    for pid in [5, 2, 9]:
        for fr in range(rng.integers(3, 8), 20):
            rows.append((pid, fr, rng.normal(), rng.normal()))
    ids, f, x, y = (np.array(c) for c in zip(*rows))
    out = traj_ref.imsd(ids, f, x.astype(np.float32), y.astype(np.float32), 1.0, 4)
    assert out[:, 0].max() == 4
    keys = list(zip(out[:, 0], out[:, 1]))
    assert keys == sorted(keys)


def test_msd_refuses_two_rows_in_one_frame():
    import pytest
    with pytest.raises(ValueError):
        traj_ref.imsd([1, 1], [3, 3], np.zeros(2, np.float32), np.zeros(2, np.float32), 1.0, 10)
