"""The FP64 adjoint checker (oracle/adjoint_ref.py) checked on the CPU.

The restatement at fixed peaks must reproduce the FP32 oracle's located rows
(which the known-answer tests pin), and its two gradient checkers -- central
finite differences and torch float64 autograd -- must agree with each other.
"""
import numpy as np
import pytest

from oracle import adjoint_ref, oracle
from tracking_optimizations_b200 import synth

PARAMS = dict(diameter=7, separation=8, minmass=300.0, noise_size=1.0, smoothing_size=7)


@pytest.fixture(scope="module")
def scene():
    spec = synth.scaled(synth.PLAIN_1000, frames=2, height=64, width=96, spots=10, seed=5)
    movie = synth.make_movie(spec).astype(np.float32)
    rows, walk, _ = oracle.batch_walk(movie, **PARAMS)
    assert len(rows) >= 8
    return movie, rows, walk


def test_fixed_peak_forward_matches_located_rows(scene):
    movie, rows, walk = scene
    ref = adjoint_ref.refine(movie, walk, 7, 1.0, 7)
    np.testing.assert_array_equal(walk[:, 0], rows[:, 0].astype(np.int64))
    # FP32 located rows vs the FP64 evaluation of the same expression
    np.testing.assert_allclose(ref[:, 0], rows[:, 2], rtol=0, atol=1e-4)
    np.testing.assert_allclose(ref[:, 1], rows[:, 3], rtol=0, atol=1e-4)
    np.testing.assert_allclose(ref[:, 2], rows[:, 1], rtol=1e-5)


def test_walk_records_are_consistent(scene):
    movie, rows, walk = scene
    # the final position is within one step per axis of the last read pixel,
    # and the refined position within the 0.6 threshold plus rounding
    assert np.all(np.abs(walk[:, 3] - walk[:, 1]) <= 1)
    assert np.all(np.abs(walk[:, 4] - walk[:, 2]) <= 1)
    assert np.all(np.abs(rows[:, 2] - walk[:, 3]) < 2.0)


def test_finite_differences_agree_with_torch_fp64(scene):
    pytest.importorskip("torch")
    movie, rows, walk = scene
    rng = np.random.default_rng(1)
    up = rng.normal(size=(len(walk), 3))
    up[:, 2] *= 1e-3  # mass is ~1e3 larger than positions
    margin = adjoint_ref.clip_margin(movie, walk, 7, 1.0, 7)
    keep = margin > 1e-2
    walk, up = walk[keep], up[keep]
    g, gs, gk = adjoint_ref.torch_reference(movie, walk, up, 7, 1.0, 7)
    samples = adjoint_ref.fd_pixels(movie, walk[:4], up[:4], 7, 1.0, 7, npix=8)
    # fd_pixels sums L over the particles near each pixel: restrict the
    # torch gradient to the same particles
    g4, _, _ = adjoint_ref.torch_reference(movie, walk[:4], up[:4], 7, 1.0, 7)
    scale = max(abs(v) for *_, v in samples)
    for t, u, v, d in samples:
        assert abs(g4[t, u, v] - d) <= 1e-6 * scale
    ds, dk = adjoint_ref.fd_params(movie, walk, up, 7, 1.0, 7)
    assert abs(gs - ds) <= 1e-6 * abs(gs)
    assert abs(gk - dk) <= 1e-6 * abs(gk)


def test_circle_order_matches_centroid_loop():
    c = adjoint_ref.circle(3)
    assert len(c) == 29
    assert tuple(c[0]) == (-3, 0) and tuple(c[-1]) == (3, 0)
    assert np.all(np.diff(c[:, 0]) >= 0)
