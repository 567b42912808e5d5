"""Batched uneven movies (gt_batch_many_device) on the GPU.

Every movie of a batch must get exactly the table that the one-movie path
(gt_batch_device) returns for it: movies of different sizes, pixel types and
parameters (specialised and generic locate kernels, linking with and
without memory, no linking, cpu_processed / characterize columns), on the
first call (graph built) and on a replay of the cached graph; a movie whose
per-frame capacity overflows is rerun through the one-movie path.
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


def _movie(torch, T, H, W, spots, seed, f32=False):
    spec = synth.scaled(synth.PLAIN_1000, frames=T, height=H, width=W, spots=spots, seed=seed)
    m = synth.make_movie(spec)
    if f32:
        return torch.from_numpy(m.astype(np.float32)).cuda()
    return torch.from_numpy(m.view(np.int16)).cuda()


@pytest.fixture(scope="module")
def movies(torch):
    return [
        (_movie(torch, 12, 128, 128, 20, 1), dict(diameter=7, separation=8, minmass=300.0, search_range=5.0,
                                                  memory=2, cpu_processed=True)),
        (_movie(torch, 5, 96, 200, 30, 2), dict(diameter=5, minmass=200.0, search_range=4.0)),
        (_movie(torch, 30, 256, 256, 120, 3), dict(diameter=9, minmass=400.0, search_range=6.0, memory=1)),
        (_movie(torch, 7, 64, 64, 8, 4, f32=True), dict(diameter=7, minmass=300.0, characterize=True)),
        (_movie(torch, 40, 128, 256, 60, 5), dict(diameter=7, separation=8, minmass=300.0, search_range=5.0,
                                                  memory=3)),
        (_movie(torch, 3, 300, 180, 40, 6), dict(diameter=11, minmass=500.0, noise_size=1.5, smoothing_size=9,
                                                 search_range=7.0)),
        (_movie(torch, 9, 128, 128, 25, 7), dict(diameter=7, separation=8, minmass=300.0, sig_radius=4.0,
                                                 bg_radius=7.0)),
    ]


def _plain(torch, movies):
    from tracking_optimizations_b200.gpu_tracking import batch_device

    return [batch_device(fr, **p).cpu().numpy() for fr, p in movies]


def test_batch_equals_per_movie_calls(torch, movies):
    from tracking_optimizations_b200.batched import batch_many, output_buffers

    want = _plain(torch, movies)
    assert all(len(w) > 0 for w in want)
    outs = output_buffers(movies)
    got, st = batch_many(movies, return_stats=True, outs=outs)
    assert st["batch_graph"] in (0, 1), st
    print(f"batched: graph={st['batch_graph']} launches={st['launches']} link passes={st['link_iterations']} "
          f"ms={st['ms_total']:.3f} fallbacks={st['batch_fallbacks']}")
    for i, ((tab, names), w) in enumerate(zip(got, want)):
        np.testing.assert_array_equal(tab.cpu().numpy(), w, err_msg=f"movie {i}")
    # replay of the cached graph (same frames, parameters and outputs)
    for o in outs:
        o.fill_(-1.0)
    got2, st2 = batch_many(movies, return_stats=True, outs=outs)
    if st["batch_graph"] == 1:
        assert st2["batch_graph"] == 2
    for i, ((tab, names), w) in enumerate(zip(got2, want)):
        np.testing.assert_array_equal(tab.cpu().numpy(), w, err_msg=f"movie {i} (replay)")


def test_batch_after_other_calls_and_reordered(torch, movies):
    # another call reuses the workspace between two batched calls; a
    # different movie order builds a new graph
    from tracking_optimizations_b200.batched import batch_many

    want = _plain(torch, movies)
    order = [3, 0, 6, 2, 5, 1, 4]
    got = batch_many([movies[i] for i in order])
    for (tab, _), i in zip(got, order):
        np.testing.assert_array_equal(tab.cpu().numpy(), want[i], err_msg=f"movie {i}")
    _plain(torch, movies[:1])
    got = batch_many([movies[i] for i in order])
    for (tab, _), i in zip(got, order):
        np.testing.assert_array_equal(tab.cpu().numpy(), want[i], err_msg=f"movie {i} after a plain call")


def test_capacity_overflow_falls_back(torch, movies):
    # pure noise with diameter 3 and separation 1: more candidates per frame
    # than the batched plan's first capacity
    from tracking_optimizations_b200.batched import batch_many

    rng = np.random.default_rng(0)
    noise = torch.from_numpy(rng.poisson(100.0, (2, 512, 512)).astype(np.float32)).cuda()
    params = dict(diameter=3, separation=1, minmass=0.0)
    mix = [movies[0], (noise, params)]
    want = _plain(torch, mix)
    assert len(want[1]) > 2 * 4096
    got, st = batch_many(mix, return_stats=True)
    assert st["batch_fallbacks"] == 1
    for (tab, _), w in zip(got, want):
        np.testing.assert_array_equal(tab.cpu().numpy(), w)


def test_batch_rejects_bad_movie(torch, movies):
    from tracking_optimizations_b200.batched import batch_many

    bad = (movies[0][0], dict(diameter=7, percentile=50.0))
    with pytest.raises(NotImplementedError, match="percentile"):
        batch_many([movies[1], bad])


def test_large_movie_linked_by_its_own_launch(torch, movies):
    # a dense 2048^2 movie with memory 3: its linker scratch would cap a
    # shared launch, so it is linked alone; the small movie shares the
    # multi-movie launch
    from tracking_optimizations_b200.batched import batch_many, output_buffers

    spec = synth.scaled(synth.DENSE_LINK, frames=6, seed=61)
    dense = (synth.make_movie_device(spec), dict(spec.params))
    mix = [movies[0], dense, movies[4]]
    want = _plain(torch, mix)
    outs = output_buffers(mix)
    for rep in range(2):
        got, st = batch_many(mix, return_stats=True, outs=outs)
        assert st["batch_fallbacks"] == 0
        for i, ((tab, _), w) in enumerate(zip(got, want)):
            np.testing.assert_array_equal(tab.cpu().numpy(), w, err_msg=f"movie {i} (call {rep})")
