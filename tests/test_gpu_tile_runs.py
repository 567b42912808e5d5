"""Runs of tiles per CTA in the specialised locate kernel.

A CTA of locate_fast_kernel locates a run of consecutive output tiles: while
one or two warps walk a tile's candidates and emit its records, the other
warps start the next tile's row pass, and the next raw tile is copied in
behind the current one.  The default run length depends on the size of a
launch (small test movies get one tile per CTA), so these tests set it
(context option ``locate_tiles_per_cta``) and compare every row and
trajectory id with the oracle.  They cover:

* runs that end inside a frame and runs that cross frames (3, 8);
* tiles with no candidates, tiles with more candidates than two walker
  warps take (the run then waits for the walks), and a flood of equal
  maxima (more candidates than the CTA has threads);
* a frame width whose rows are not a multiple of 16 bytes, where the raw
  tiles are staged without TMA;
* 32-row tiles (256 threads).
"""
import numpy as np
import pytest

from oracle import oracle
from tracking_optimizations_b200 import _native, batch_rust, synth

pytestmark = pytest.mark.gpu

NTHREADS = 8


def movie(width):
    spec = synth.scaled(synth.PLAIN_1000, frames=9, height=200, width=width, spots=120, seed=31)
    mv = synth.make_movie(spec)
    h = mv.shape[1]
    yy, xx = np.mgrid[0:h, 0:width]
    board = np.where((yy + xx) % 2 == 0, 1200, 800).astype(np.uint16)
    mv[3] = 1000
    mv[3, 10:150, 20:width - 20] = board[10:150, 20:width - 20]  # a flood of equal maxima
    mv[5] = 0                                                   # a blank frame
    mv[6, 40:60, 40:140] = board[40:60, 40:140]                  # 60-100 candidates in a few tiles
    return mv, dict(spec.params)


@pytest.mark.parametrize("rows", [64, 32])
@pytest.mark.parametrize("per_cta", [1, 3, 8])
@pytest.mark.parametrize("width", [320, 300])
def test_tile_runs_match_oracle(gpu, per_cta, width, rows):
    mv, params = movie(width)
    d = params.pop("diameter")
    params["cpu_processed"] = True
    want = oracle.batch(mv, d, nthreads=NTHREADS, **params)
    _native.set_option("locate_tiles_per_cta", per_cta)
    _native.set_option("locate_tile_rows", rows)
    try:
        got = batch_rust(mv, d, **params)
        st = _native.last_stats()
    finally:
        _native.set_option("locate_tiles_per_cta", 0)
        _native.set_option("locate_tile_rows", 64)
    # 2: tiles staged by TMA; 1: staged by the threads (rows of 600 bytes)
    assert st["locate_kernel"] == (2 if width == 320 else 1)
    assert got[1] == want[1]
    assert got[0].shape == want[0].shape
    same = (got[0] == want[0]) | (np.isnan(got[0]) & np.isnan(want[0]))
    assert same.all(), f"first mismatch at {np.argwhere(~same)[0]}"
    assert st["candidates"] > 4000  # the flood frame
    assert (want[0][:, 0] == 5).sum() == 0 and (want[0][:, 0] == 0).sum() > 50


@pytest.mark.parametrize("diameter", [5, 9, 11])
def test_tile_runs_other_diameters(gpu, diameter):
    """Two processed planes (diameters 5, 7, 11) and one (9), in runs of 4."""
    mv, params = movie(320)
    params.update(diameter=diameter, separation=diameter + 1, smoothing_size=diameter)
    params.pop("diameter")
    params["cpu_processed"] = True
    want = oracle.batch(mv, diameter, nthreads=NTHREADS, **params)
    _native.set_option("locate_tiles_per_cta", 4)
    try:
        got = batch_rust(mv, diameter, **params)
        st = _native.last_stats()
    finally:
        _native.set_option("locate_tiles_per_cta", 0)
    assert st["locate_kernel"] == 2
    assert got[1] == want[1]
    assert got[0].shape == want[0].shape
    same = (got[0] == want[0]) | (np.isnan(got[0]) & np.isnan(want[0]))
    assert same.all(), f"first mismatch at {np.argwhere(~same)[0]}"
