"""The device renderer of synthetic movies (gt_synth_render).

Checks the noise model on spot-free frames (Poisson mean and variance plus
read-noise variance), that spots land where the tracks put them (located
positions within half a pixel), and that the frames do not depend on the
chunking.
"""
import numpy as np
import pytest

from tracking_optimizations_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    assert t.cuda.is_available(), "needs a CUDA device"
    return t


def test_background_statistics(torch):
    spec = synth.MovieSpec(4, 256, 256, 0, 1.2, 150.0, 1500.0, 1.5, background=100.0, read_noise=5.0, seed=3)
    m = synth.make_movie_device(spec).cpu().numpy().view(np.uint16).astype(np.float64)
    # rounding adds 1/12 to the variance
    assert abs(m.mean() - 100.0) < 0.1
    assert abs(m.var() - (100.0 + 25.0 + 1.0 / 12.0)) < 1.5
    low = synth.MovieSpec(2, 256, 256, 0, 1.2, 150.0, 1500.0, 1.5, background=3.0, read_noise=0.0, seed=4)
    z = synth.make_movie_device(low).cpu().numpy().view(np.uint16).astype(np.float64)
    assert abs(z.mean() - 3.0) < 0.05 and abs(z.var() - 3.0) < 0.1
    assert abs(np.mean(z == 0) - np.exp(-3.0)) < 0.01


def test_spots_are_located_at_their_tracks(torch):
    from tracking_optimizations_b200.gpu_tracking import batch_device

    spec = synth.MovieSpec(6, 256, 384, 60, 1.2, 600.0, 1500.0, 1.5, read_noise=5.0, seed=8,
                           params=dict(diameter=7, separation=8, minmass=300.0))
    movie = synth.make_movie_device(spec)
    rows = batch_device(movie, **spec.params).cpu().numpy()
    tracks = synth.spot_tracks(spec)
    hits = 0
    for t in range(spec.frames):
        r = rows[rows[:, 0] == t]
        for y, x, a in tracks[t]:
            if a == 0 or y < 5 or x < 5 or y > spec.height - 6 or x > spec.width - 6:
                continue
            d = np.hypot(r[:, 2] - y, r[:, 3] - x)
            hits += int(d.size > 0 and d.min() < 0.5)
    visible = sum(int(a > 0 and 5 <= y <= spec.height - 6 and 5 <= x <= spec.width - 6)
                  for t in range(spec.frames) for y, x, a in tracks[t])
    assert hits >= 0.9 * visible, (hits, visible)


def test_chunking_does_not_change_frames(torch):
    # the noise is counter-based; where spots overlap, their float sums may
    # round differently (atomic addition order), by at most one count
    spec = synth.MovieSpec(7, 64, 96, 10, 1.5, 200.0, 900.0, 1.0, read_noise=2.0, seed=12)
    a = synth.make_movie_device(spec, chunk=16).cpu().numpy().view(np.uint16).astype(np.int64)
    b = synth.make_movie_device(spec, chunk=3).cpu().numpy().view(np.uint16).astype(np.int64)
    assert np.abs(a - b).max() <= 1
    assert np.mean(a != b) < 1e-3
