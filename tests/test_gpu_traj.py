"""Trajectory post-processing on the device (gt_filter_stubs, gt_steps,
gt_imsd) against the reference's step_tracker (golden vectors) and the CPU
restatement (oracle/traj_ref.py): stub masks, steps and step lengths bit for
bit; MSD values bit for bit against the restatement's float64 left-to-right
sums (tolerance 1 float32 ulp written in the test for the rounding of the
summed means)."""
import os

import numpy as np
import pytest

from oracle import traj_ref
from tracking_optimizations_b200 import batch_rust, synth, trajectories

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "steps_golden.npz")


def test_steps_match_reference_step_tracker(gpu):
    g = np.load(GOLDEN)
    xs, ys, dx, dy, ln, order = trajectories.steps(g["particle"], g["x"], g["y"], float(g["pixel_size"]))
    np.testing.assert_array_equal(xs, g["out_x"])
    np.testing.assert_array_equal(ys, g["out_y"])
    np.testing.assert_array_equal(dx, g["x_step"])
    np.testing.assert_array_equal(dy, g["y_step"])
    np.testing.assert_array_equal(ln, g["steplength"])
    np.testing.assert_array_equal(order, np.argsort(g["particle"], kind="stable"))


def linked_table(frames=40, seed=21):
    spec = synth.scaled(synth.PLAIN_1000, frames=frames, seed=seed)
    tab, cols = batch_rust(synth.make_movie(spec), **dict(spec.params))
    names = [c[0] for c in cols]
    return {k: tab[:, names.index(k)] for k in ("frame", "y", "x", "particle")}


def assert_msd_equal(got, want):
    t, p, m = got
    assert len(t) == len(want)
    np.testing.assert_array_equal(np.round(t).astype(np.int64), want[:, 0].astype(np.int64))  # fps = 1
    np.testing.assert_array_equal(p, want[:, 1].astype(np.int64))
    np.testing.assert_allclose(m, want[:, 2], rtol=1.2e-7, atol=0)


def test_filter_stubs_steps_imsd_on_a_linked_table(gpu):
    t = linked_table()
    ids = t["particle"].astype(np.int64)
    for thr in [0, 1, 5, 20, 41]:
        np.testing.assert_array_equal(trajectories.filter_stubs(ids, thr), traj_ref.filter_stubs(ids, thr))
    _, inv, cnt = np.unique(ids, return_inverse=True, return_counts=True)
    np.testing.assert_array_equal(trajectories.filter_stubs(ids, 3, return_counts=True)[1], cnt[inv])
    keep = traj_ref.filter_stubs(ids, 10)
    ids_k, f_k, x_k, y_k = ids[keep], t["frame"][keep].astype(np.int64), t["x"][keep], t["y"][keep]
    got = trajectories.steps(ids_k, x_k, y_k, 0.18333)
    want = traj_ref.steps(ids_k, x_k, y_k, 0.18333)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    # the reference's memory dedupe can give a particle two rows in one
    # frame; trackpy's msd refuses those particles, so drop them here
    dup = np.zeros(len(ids_k), bool)
    key = ids_k * 100000 + f_k
    u, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    bad = np.unique(ids_k[cnt[inv] > 1])
    ok = ~np.isin(ids_k, bad)
    for maxlag in [1, 7, 100]:
        g = trajectories.imsd(ids_k[ok], f_k[ok], x_k[ok], y_k[ok], 0.18333, 1.0, max_lagtime=maxlag)
        w = traj_ref.imsd(ids_k[ok], f_k[ok], x_k[ok], y_k[ok], 0.18333, maxlag)
        assert_msd_equal(g, w)


def test_imsd_gaps_edge_cases(gpu):
    # a single-row particle (no lag), a particle with gaps, negative frames,
    # ids out of order
    ids = np.array([7, 3, 3, 3, 3, 11, 3, 11], np.int64)
    f = np.array([5, -2, 0, 1, 6, 0, 9, 1], np.int64)
    rng = np.random.default_rng(1)
    x = rng.normal(size=8).astype(np.float32) * 10
    y = rng.normal(size=8).astype(np.float32) * 10
    assert_msd_equal(trajectories.imsd(ids, f, x, y, 0.5, 1.0, 100), traj_ref.imsd(ids, f, x, y, 0.5, 100))
    t, p, m = trajectories.imsd(ids[:1], f[:1], x[:1], y[:1], 0.5, 1.0, 100)
    assert len(t) == 0


def test_imsd_refuses_two_rows_in_one_frame(gpu):
    with pytest.raises(Exception, match="one trajectory per particle"):
        trajectories.imsd([1, 1, 2], [3, 3, 4], np.zeros(3, np.float32), np.zeros(3, np.float32), 1.0, 1.0, 10)


def test_postprocess_chain(gpu):
    import pandas as pd

    class Params:
        duration_filter = 8
        pixel_size = 0.18333
        tracking_time = 0.036

    t = linked_table(frames=30, seed=5)
    df = pd.DataFrame({k: t[k] for k in ("frame", "y", "x", "particle")})
    ids = df["particle"].to_numpy().astype(np.int64)
    f = df["frame"].to_numpy().astype(np.int64)
    u, inv, cnt = np.unique(ids * 100000 + f, return_inverse=True, return_counts=True)
    df = df[~np.isin(ids, np.unique(ids[cnt[inv] > 1]))].reset_index(drop=True)
    full, msd_df = trajectories.postprocess(df, Params)
    keep = traj_ref.filter_stubs(df["particle"].to_numpy().astype(np.int64), 8)
    sub = df[keep]
    xs, ys, dx, dy, ln, _ = traj_ref.steps(sub["particle"].to_numpy().astype(np.int64), sub["x"], sub["y"], 0.18333)
    np.testing.assert_array_equal(full["x"].to_numpy(), xs)
    np.testing.assert_array_equal(full["steplength"].to_numpy(), ln)
    dur = full.groupby("particle")["particle"].transform(len).to_numpy()
    np.testing.assert_array_equal(full["duration"].to_numpy(), dur)
    w = traj_ref.imsd(full["particle"].to_numpy(), full["frame"].to_numpy(), xs, ys, 0.18333, dur.max())
    np.testing.assert_allclose(msd_df["time"].to_numpy(), w[:, 0].astype(np.float64) / 0.036)
    np.testing.assert_array_equal(msd_df["particle"].to_numpy(), w[:, 1].astype(np.int64))
    np.testing.assert_allclose(msd_df["msd"].to_numpy(), w[:, 2], rtol=1.2e-7, atol=0)
