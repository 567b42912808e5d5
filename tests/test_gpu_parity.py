"""Parity of the CUDA path (through the C ABI) with the CPU restatement.

Integer/index results (detected features, counts, trajectory IDs) must be
identical; positions, masses and the characterisation columns are also
compared for exact equality, because the kernels evaluate every value with
the oracle's operation order (explicit fused multiply-adds only).  Each case
also states the error of the FP32 result against the FP64 oracle.
"""
import os

import numpy as np
import pytest

from oracle import oracle
from tracking_optimizations_b200 import _native, batch_rust, link_rust, synth

pytestmark = pytest.mark.gpu

NTHREADS = 8


def assert_tables_equal(got, want, cols):
    g, gc = got
    w, wc = want
    assert gc == wc == cols if cols is not None else gc == wc
    assert g.shape == w.shape, (g.shape, w.shape)
    if g.size:
        bad = ~((g == w) | (np.isnan(g) & np.isnan(w)))
        if bad.any():
            r, c = np.argwhere(bad)[0]
            raise AssertionError(f"first mismatch row {r} col {gc[c]}: gpu {g[r]} vs oracle {w[r]}")


def fp64_error(table, movie, params):
    """max |dx|, |dy| (px) and max relative mass error against the FP64 oracle."""
    ref, _ = oracle.batch(movie, nthreads=NTHREADS, fp64=True, **params)
    if table.shape[0] == 0 or ref.shape[0] == 0:
        return 0.0, 0.0
    # match rows by frame and nearest position
    errs, merr = [], []
    for t in np.unique(table[:, 0]):
        a = table[table[:, 0] == t]
        b = ref[ref[:, 0] == t]
        if len(b) == 0:
            continue
        d = (a[:, None, 2] - b[None, :, 2]) ** 2 + (a[:, None, 3] - b[None, :, 3]) ** 2
        j = d.argmin(1)
        ok = d[np.arange(len(a)), j] < 0.25
        errs.append(np.sqrt(d[np.arange(len(a)), j][ok]))
        merr.append(np.abs(a[ok, 1] - b[j[ok], 1]) / np.abs(b[j[ok], 1]))
    e = np.concatenate(errs) if errs else np.zeros(1)
    m = np.concatenate(merr) if merr else np.zeros(1)
    return float(e.max(initial=0)), float(m.max(initial=0))


def check(movie, **params):
    d = params.pop("diameter")
    got = batch_rust(movie, d, **params)
    want = oracle.batch(movie, d, nthreads=NTHREADS, **params)
    assert_tables_equal(got, want, None)
    return got


def test_plain_small_exact(gpu):
    spec = synth.PLAIN_SMALL
    mv = synth.make_movie(spec)
    params = dict(spec.params, cpu_processed=True)
    tab, cols = check(mv, **params)
    assert _native.last_stats()["locate_kernel"] == 2, "specialised TMA locate kernel not used"
    assert [c[0] for c in cols] == ["frame", "mass", "y", "x", "particle", "Rg", "ecc", "signal"]
    assert tab.shape[0] > 300
    pos_err, mass_err = fp64_error(tab, mv, dict(spec.params))
    print(f"plain_small: rows={tab.shape[0]} fp64 pos err={pos_err:.2e} px mass rel err={mass_err:.2e}")
    assert pos_err < 1e-3 and mass_err < 1e-4


def test_plain_512_scaled_exact(gpu):
    spec = synth.scaled(synth.PLAIN_1000, frames=12)
    mv = synth.make_movie(spec)
    tab, _ = check(mv, **dict(spec.params, cpu_processed=True))
    assert _native.last_stats()["locate_kernel"] == 2, "specialised TMA locate kernel not used"
    assert tab.shape[0] > 12 * 300


def test_float32_input_exact(gpu):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=4, seed=7)
    mv = synth.make_movie(spec).astype(np.float32)
    mv += np.random.default_rng(0).random(mv.shape, dtype=np.float32)  # non-integer pixels
    check(mv, **dict(spec.params, cpu_processed=True))


def test_u16_and_f32_agree(gpu):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=3, seed=11)
    mv = synth.make_movie(spec)
    a = batch_rust(mv, 9, minmass=500, search_range=5)
    b = batch_rust(mv.astype(np.float32), 9, minmass=500, search_range=5)
    assert_tables_equal(a, b, None)


@pytest.mark.parametrize("H,W", [(37, 53), (64, 64), (130, 70), (33, 257)])
def test_odd_sizes(gpu, H, W):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=3, height=H, width=W, seed=H * W)
    mv = synth.make_movie(spec)
    check(mv, **dict(spec.params, cpu_processed=True))


@pytest.mark.parametrize("kw", [
    dict(diameter=5), dict(diameter=7, separation=4), dict(diameter=8), dict(diameter=11, smoothing_size=13),
    dict(diameter=9, max_iterations=1), dict(diameter=9, max_iterations=0), dict(diameter=9, max_iterations=30),
    dict(diameter=9, noise_size=2.5), dict(diameter=9, smoothing_size=4), dict(diameter=3, separation=2),
    dict(diameter=1), dict(diameter=9, minmass=-5.0),
])
def test_parameter_variants(gpu, kw):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=2, height=96, width=128, seed=3)
    mv = synth.make_movie(spec)
    check(mv, cpu_processed=True, **kw)


def test_characterize_and_raw_columns(gpu):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=3, seed=5)
    mv = synth.make_movie(spec)
    tab, cols = check(mv, diameter=9, minmass=500, characterize=True, cpu_processed=True, sig_radius=4.0,
                      bg_radius=8.0, gap_radius=1.0, search_range=5.0)
    assert cols[-1][0] == "ecc_gpu"


def test_raw_signal_even_annulus(gpu):
    spec = synth.scaled(synth.PLAIN_SMALL, frames=2, seed=6)
    mv = synth.make_movie(spec)
    check(mv, diameter=9, minmass=500, sig_radius=2.5, bg_radius=6.0)


@pytest.mark.parametrize("rows", [64, 32])
def test_candidate_flood_exact(gpu, rows):
    """A checkerboard makes every other pixel an equal (non-strict) local
    maximum: thousands of candidates per tile, more than the locate kernel
    walks itself (the rest go to the fallback walk)."""
    mv = np.full((2, 96, 160), 1000, np.uint16)
    yy, xx = np.mgrid[0:96, 0:160]
    board = np.where((yy + xx) % 2 == 0, 1200, 800).astype(np.uint16)
    mv[0, 8:90, 4:150] = board[8:90, 4:150]
    mv[1, 20:60, 70:140] = board[20:60, 70:140]
    try:
        _native.set_option("locate_tile_rows", rows)
        tab, _ = check(mv, diameter=7, minmass=10.0, search_range=3.0, cpu_processed=True)
        st = _native.last_stats()
        assert st["locate_kernel"] == 2
    finally:
        _native.set_option("locate_tile_rows", 64)
    assert st["candidates"] > 4000  # records before the separation filter
    assert tab.shape[0] >= 10


def test_blank_and_saturated_frames(gpu):
    mv = np.zeros((3, 64, 80), np.uint16)
    mv[1, 20:30, 30:40] = 65535     # saturated plateau: many equal maxima
    mv[2] = 100
    tab, _ = check(mv, diameter=7, search_range=3.0, cpu_processed=True)
    assert (tab[:, 0] == 0).sum() == 0


@pytest.mark.parametrize("memory", [1, 2, 3])
@pytest.mark.parametrize("seed", [21, 22])
def test_memory_linking_exact(gpu, memory, seed):
    spec = synth.MovieSpec(30, 160, 160, 60, 1.3, 200, 1200, 1.6, read_noise=5.0, blink=0.15, seed=seed)
    mv = synth.make_movie(spec)
    tab, _ = check(mv, diameter=7, minmass=200, search_range=5.0, memory=memory)
    st = _native.last_stats()
    print(f"memory={memory}: link fixed-point passes {st['link_iterations']}")


def test_linking_across_upload_chunks_exact(gpu):
    """Host frames are uploaded, finalized and linked in chunks of 16 frames
    here (the linker in frame windows); memory 4 with frequent blinking
    reaches across the chunk boundaries, and the last chunk has 2 frames."""
    spec = synth.MovieSpec(50, 128, 160, 50, 1.3, 200, 1200, 1.6, read_noise=5.0, blink=0.3, seed=77)
    mv = synth.make_movie(spec)
    check(mv, diameter=7, minmass=200, search_range=5.0, memory=4)
    st = _native.last_stats()
    assert st["link_iterations"] >= 1


def test_dense_linking_subnets_exact(gpu):
    # DENSE_LINK density (20000 spots per 2048^2) on 512^2: many 2-12 subnets
    spec = synth.scaled(synth.DENSE_LINK, frames=8, height=512, width=512, seed=31)
    mv = synth.make_movie(spec)
    check(mv, **spec.params)


def test_link_rust_matches_oracle(gpu):
    rng = np.random.default_rng(4)
    rows = []
    pos = rng.uniform(0, 200, (80, 2))
    for t in range(25):
        keep = rng.random(len(pos)) > 0.1
        for (y, x) in pos[keep]:
            rows.append((t, 1.0, y, x))
        pos = pos + rng.normal(0, 2.0, pos.shape)
    rows = np.array(rows, np.float32)
    for mem in [None, 0, 1, 3]:
        g = link_rust(rows, 6.0, mem)
        w = oracle.link(rows, 6.0, mem)
        np.testing.assert_array_equal(g, w)
    # frame-value quirks of FrameSubsetter: leading non-zero frame, repeats
    quirky = rows.copy()
    quirky[:, 0] += 3
    np.testing.assert_array_equal(link_rust(quirky, 6.0, 2), oracle.link(quirky, 6.0, 2))


@pytest.mark.parametrize("opt", [("locate_tile_rows", 32), ("force_generic", 1)])
def test_locate_kernel_variants_agree(gpu, opt):
    """The specialised kernel at both tile heights and the generic kernel
    produce identical tables."""
    spec = synth.scaled(synth.PLAIN_1000, frames=6, seed=41)
    mv = synth.make_movie(spec)
    params = dict(spec.params, cpu_processed=True, characterize=True)
    base = batch_rust(mv, **params)
    try:
        _native.set_option(*opt)
        other = batch_rust(mv, **params)
    finally:
        _native.set_option("locate_tile_rows", 64)
        _native.set_option("force_generic", 0)
    assert_tables_equal(other, base, None)


def test_full_size_plain_1000(gpu):
    """All 1000 frames of 512^2 (the throughput workload) on the GPU against
    the oracle over the whole movie: every row, column and trajectory id."""
    spec = synth.PLAIN_1000
    mv = synth.make_movie(spec)
    params = dict(spec.params, cpu_processed=True)
    got = batch_rust(mv, **params)
    assert got[0].shape[0] > 1000 * 300
    d = params.pop("diameter")
    want = oracle.batch(mv, d, nthreads=os.cpu_count() or NTHREADS, **params)
    assert_tables_equal(got, want, None)


def test_full_size_dense_linking(gpu):
    """The dense linking stress at full size: 200 frames of 2048^2 with 20000
    spots, step 2.5 px, search_range 7, memory 3, diameter 9 -- every row and
    trajectory id against the oracle."""
    spec = synth.DENSE_LINK
    mv = synth.make_movie_device(spec).cpu().numpy().view(np.uint16)  # 838 Mpx: rendered on the device
    params = dict(spec.params)
    got = batch_rust(mv, **params)
    st = _native.last_stats()
    assert got[0].shape[0] > 200 * 12000
    d = params.pop("diameter")
    want = oracle.batch(mv, d, nthreads=os.cpu_count() or NTHREADS, **params)
    assert_tables_equal(got, want, None)
    print(f"dense linking: {got[0].shape[0]} rows, {int(got[0][:, 4].max()) + 1} trajectories, "
          f"link passes {st['link_iterations']}, link {st['ms_link']:.2f} ms")


def test_tables_alive_across_calls_keep_their_contents():
    # host tables come from a pool of page-locked blocks: a table still
    # referenced must never be handed to a later call
    spec = synth.scaled(synth.PLAIN_SMALL, frames=6, seed=5)
    movie = synth.make_movie(spec)
    other = synth.make_movie(synth.scaled(synth.PLAIN_SMALL, frames=6, seed=6))
    params = dict(spec.params)
    d = params.pop("diameter")
    want_a, _ = oracle.batch(movie, d, nthreads=NTHREADS, **params)
    want_b, _ = oracle.batch(other, d, nthreads=NTHREADS, **params)
    held = []
    for i in range(6):
        held.append((i, batch_rust(movie if i % 2 == 0 else other, d, **params)[0]))
        if i == 3:
            del held[:2]  # released blocks go back to the pool and are reused
    for i, tab in held:
        np.testing.assert_array_equal(tab, want_a if i % 2 == 0 else want_b, err_msg=f"call {i}")


def tiny_movie(H, W, seed):
    """Three frames of H x W: read noise and a few bright Gaussian spots."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W]
    mv = rng.normal(200.0, 8.0, (3, H, W))
    for t in range(3):
        for _ in range(max(2, H * W // 25)):
            cy, cx = rng.uniform(0, H), rng.uniform(0, W)
            mv[t] += 3000.0 * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * 1.2 ** 2))
    return np.clip(mv, 0, 65535).astype(np.uint16)


@pytest.mark.parametrize("diameter", [5, 7])
@pytest.mark.parametrize("H,W", [(5, 40), (40, 5), (7, 7), (9, 13), (16, 8), (12, 30)])
def test_tiny_frames(gpu, H, W, diameter):
    """Frames narrower or shorter than a tile's halo: one tile covers the
    frame, and a boxcar window can reach both frame edges (the specialised
    kernel repairs the reflect padding of such tiles after its row pass)."""
    mv = tiny_movie(H, W, H * 100 + W)
    tab, _ = check(mv, diameter=diameter, minmass=50.0, search_range=3.0, cpu_processed=True)
    assert _native.last_stats()["locate_kernel"] in (1, 2)
