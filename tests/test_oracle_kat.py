"""Known-answer tests pinning the CPU restatement (oracle/) to the reference
semantics, derived by hand from the reference source.  No golden vectors
exist in the reference (it has no tests), so these are the pins."""
import numpy as np
import pytest

from oracle import oracle


def test_dilation_sizes():
    # gpu_setup.rs:48 floor(2*sep/sqrt(2)) in f32; max_rows.wgsl:17 trunc(D/2 - 0.5)
    assert oracle.dilation(8) == (11, 5)
    assert oracle.dilation(10) == (14, 6)
    assert oracle.dilation(12) == (16, 7)
    assert oracle.dilation(1) == (1, 0)
    assert oracle.dilation(0) == (0, 0)


def test_bandpass_constant_image_vanishes():
    f = np.full((40, 50), 300.0, np.float32)
    p = oracle.bandpass(f, 7, 1.0)
    assert p.shape == f.shape
    assert (p >= 0).all()
    assert p.max() < 1e-3 * 300.0


def test_bandpass_matches_float64_formula():
    # separable Gaussian (zero-padded, normalised by the full window) minus a
    # reflect-padded boxcar / k^2, clipped at 0 (preprocess_rows/cols.wgsl)
    rng = np.random.default_rng(5)
    f = rng.integers(0, 2000, (23, 31)).astype(np.float32)
    k, s2 = 5, 1.7
    r = k // 2
    w = np.exp(-np.arange(-r, r + 1, dtype=np.float64) ** 2 / (2 * s2))
    n = w.sum()
    fp = np.pad(f.astype(np.float64), r, mode="constant")
    fr = np.pad(f.astype(np.float64), r, mode="symmetric")
    H, W = f.shape
    g_row = np.stack([sum(w[i] * fp[r:r + H, i:i + W] for i in range(k))]) [0] / n
    b_row = sum(fr[:, i:i + W] for i in range(k))
    gp = np.pad(g_row, ((r, r), (0, 0)), mode="constant")
    g = sum(w[i] * gp[i:i + H] for i in range(k)) / n
    b = sum(b_row[i:i + H] for i in range(k)) / (k * k)
    ref = np.maximum(g - b, 0)
    got = oracle.bandpass(f, k, s2)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=2e-3)


def gauss_frame(H, W, spots, sigma=1.5, bg=0.0):
    yy, xx = np.mgrid[0:H, 0:W]
    f = np.full((H, W), bg)
    for (y, x, a) in spots:
        f += a * np.exp(-((yy - y) ** 2 + (xx - x) ** 2) / (2 * sigma ** 2))
    return f.astype(np.float32)


def test_single_spot_position():
    f = gauss_frame(48, 48, [(20.3, 25.6, 1000.0)])
    tab, cols = oracle.batch(f[None], 9, minmass=10)
    assert [c[0] for c in cols] == ["frame", "mass", "y", "x"]
    assert tab.shape[0] == 1
    assert abs(tab[0, 2] - 20.3) < 0.15 and abs(tab[0, 3] - 25.6) < 0.15
    assert tab[0, 1] > 10


def test_walk_moves_to_the_centroid():
    # a spot centred between pixels: the max pixel's centroid offset is
    # > 0.6 after a shift, so the walk must move (walk_cols.wgsl:46-68)
    f = gauss_frame(48, 48, [(20.5, 25.5, 1000.0)], sigma=2.0)
    f[19, 24] += 60.0   # make the up-left pixel the local maximum
    planes = oracle.locate_planes(f, 9, minmass=1)
    ys, xs = np.nonzero(planes[0])
    assert len(ys) >= 1
    # every emitted position lies near the true centre although it is keyed
    # by its originating pixel (walk_cols.wgsl:87-91)
    for y0, x0 in zip(ys, xs):
        assert abs(planes[1, y0, x0] - 20.5) < 0.7 and abs(planes[2, y0, x0] - 25.5) < 0.7


def test_separation_tie_break_keeps_lower_raster_index():
    # two identical integer blobs 12 px apart with separation 13: their
    # neighbourhoods are translates of each other, so the masses are exactly
    # equal and execute_gpu.rs:268-276 keeps the lower pre-filter index
    f = np.zeros((40, 60), np.float32)
    blob = np.array([[10, 40, 10], [40, 200, 40], [10, 40, 10]], np.float32)
    f[19:22, 19:22] = blob
    f[19:22, 31:34] = blob
    planes = oracle.locate_planes(f, 5, separation=13, minmass=1)
    assert (planes[0] > 0).sum() == 2
    ys, xs = np.nonzero(planes[0])
    assert planes[0][ys[0], xs[0]] == planes[0][ys[1], xs[1]]
    tab, _ = oracle.batch(f[None], 5, separation=13, minmass=1)
    assert tab.shape[0] == 1 and abs(tab[0, 3] - 20) < 0.5
    g = f.copy()
    g[20, 32] += 1.0   # now the right blob is heavier and wins
    tab, _ = oracle.batch(g[None], 5, separation=13, minmass=1)
    assert tab.shape[0] == 1 and abs(tab[0, 3] - 32) < 0.5


def test_minmass_is_strict():
    f = gauss_frame(48, 48, [(24, 24, 500.0)])
    tab, _ = oracle.batch(f[None], 9, minmass=0)
    m = float(tab[0, 1])
    assert oracle.batch(f[None], 9, minmass=m)[0].shape[0] == 0
    assert oracle.batch(f[None], 9, minmass=np.nextafter(np.float32(m), np.float32(0)))[0].shape[0] == 1


def test_unimplemented_options_raise():
    f = np.zeros((1, 16, 16), np.float32)
    for name in oracle.NOT_IMPLEMENTED:
        with pytest.raises(NotImplementedError):
            oracle.batch(f, 5, **{name: 1})


def test_columns_order():
    p = oracle.resolve(9, search_range=5, cpu_processed=True, sig_radius=3, bg_radius=6, characterize=True)
    assert [c[0] for c in oracle.columns(p)] == [
        "frame", "mass", "y", "x", "particle", "Rg", "ecc", "signal", "raw_mass", "raw_bg_median",
        "raw_mass_corrected", "Rg_gpu", "raw_mass_gpu", "signal_gpu", "ecc_gpu"]


def table(frames):
    rows = []
    for t, pts in enumerate(frames):
        for (y, x) in pts:
            rows.append((t, 1.0, y, x))
    return np.array(rows, np.float32)


def relabel(ids):
    m = {}
    return [m.setdefault(i, len(m)) for i in ids]


def test_link_continuation_and_new():
    ids = oracle.link(table([[(10, 10), (50, 50)], [(11, 10.5), (80, 80)]]), 5)
    assert list(ids) == [0, 1, 0, 2]


def test_link_subnet_minimises_squared_distance():
    # sources a=(10,10), b=(10,14); dests c=(10,13), d=(10,9.5)
    # a->d (0.25) + b->c (1) beats a->c (9) + b->d (20.25)
    ids = oracle.link(table([[(10, 10), (10, 14)], [(10, 13), (10, 9.5)]]), 5)
    assert list(ids) == [0, 1, 1, 0]


def test_link_subnet_prefers_null_over_far_pair():
    # one source between two dests; only one can take it (linking.rs:404-405:
    # null costs r^2 per unmatched destination)
    ids = oracle.link(table([[(10, 10)], [(10, 11), (10, 13)]]), 5)
    assert list(ids) == [0, 0, 1]


def test_link_strict_radius():
    # exactly search_range away is not a candidate (linking.rs:97 `<`)
    ids = oracle.link(table([[(10, 10)], [(10, 15)]]), 5)
    assert list(ids) == [0, 1]


def test_link_memory_bridges_gap():
    fr = [[(10, 10), (40, 40)], [(40, 41)], [(10.5, 10.5), (40, 42)]]
    assert list(oracle.link(table(fr), 5, memory=1)) == [0, 1, 1, 0, 1]
    assert list(oracle.link(table(fr), 5, memory=0)) == [0, 1, 1, 2, 1]


def test_link_memory_expires():
    fr = [[(10, 10), (40, 40)], [(40, 41)], [(40, 42)], [(10.5, 10.5), (40, 43)]]
    assert list(oracle.link(table(fr), 5, memory=1)) == [0, 1, 1, 1, 2, 1]
    assert list(oracle.link(table(fr), 5, memory=2)) == [0, 1, 1, 1, 0, 1]


def test_link_frame_subsetter_groups():
    # groups are runs of equal column-0 values (linking.rs:33-61): a repeated
    # frame value after another value starts a new group, and gaps in frame
    # numbers are not empty frames
    rows = np.array([[5, 1, 10, 10], [5, 1, 30, 30], [9, 1, 10.5, 10], [5, 1, 11, 10]], np.float32)
    assert list(oracle.link(rows, 3)) == [0, 1, 0, 0]


def test_fp64_twin_agrees():
    from tracking_optimizations_b200 import synth
    mv = synth.make_movie(synth.scaled(synth.PLAIN_SMALL, frames=2))
    p = dict(synth.PLAIN_SMALL.params)
    a, _ = oracle.batch(mv, **p)
    b, _ = oracle.batch(mv, fp64=True, **p)
    assert a.shape[0] == b.shape[0]
    np.testing.assert_allclose(a[:, 2:4], b[:, 2:4], atol=1e-3)
    np.testing.assert_allclose(a[:, 1], b[:, 1], rtol=1e-4)
