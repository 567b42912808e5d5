"""Error paths of the device code, made to happen without a fault.

* The linker's per-subnetwork search budget: a context option lowers it so
  that a small dense subnetwork exceeds it; the call must report
  GT_ERR_SUBNET_BUDGET and return no table, and the context must link
  correctly again once the budget is restored.
* The bounded wait for a tile staged by TMA in the specialised locate
  kernel: a test switch issues no copy, so the barrier never completes and
  the wait runs out after a short iteration limit; every CTA returns, the
  call reports GT_ERR_DEVICE_TIMEOUT, and the next call on the same context
  gives the normal result.
"""
import numpy as np
import pytest

from oracle import oracle
from tracking_optimizations_b200 import _native, gpu_tracking, synth

pytestmark = pytest.mark.gpu


def dense_subnet_table():
    """Two frames of 6 particles 1 px apart, shifted by 0.3 px: with
    search_range 5 every source reaches every destination (one 6 x 6
    subnetwork)."""
    rng = np.random.default_rng(11)
    base = np.array([[10.0 + i % 3, 10.0 + i // 3] for i in range(6)], np.float32)
    rows = []
    for f in range(2):
        pos = base + (0.3 * f + rng.uniform(-0.05, 0.05, base.shape)).astype(np.float32)
        for y, x in pos:
            rows.append([f, 1000.0, y, x])
    return np.array(rows, np.float32)


def test_subnet_budget_error_then_recovery(gpu):
    table = dense_subnet_table()
    want = oracle.link(table, 5.0)
    _native.set_option("subnet_budget", 8)
    try:
        with pytest.raises(_native.GtError) as e:
            gpu_tracking.link_rust(table, 5.0)
        assert e.value.status == _native.GT_ERR_SUBNET_BUDGET
        # the locate+link path reports it the same way, with no table
        movie = synth.make_movie(synth.scaled(synth.PLAIN_SMALL, frames=2))
        _native.set_option("subnet_budget", 1)
        with pytest.raises(_native.GtError) as e2:
            gpu_tracking.batch_rust(movie, 9, minmass=500.0, search_range=30.0)
        assert e2.value.status == _native.GT_ERR_SUBNET_BUDGET
    finally:
        _native.set_option("subnet_budget", 0)  # back to the default
    np.testing.assert_array_equal(gpu_tracking.link_rust(table, 5.0), want)


@pytest.mark.parametrize("per_cta", [0, 4])
def test_tile_copy_timeout_then_recovery(gpu, per_cta):
    """The withheld copy of a CTA's first tile runs out of its bounded wait;
    with runs of 4 tiles per CTA the CTA then issues no further copies,
    skips the later waits and still reaches every barrier."""
    movie = synth.make_movie(synth.scaled(synth.PLAIN_1000, frames=4, seed=9))
    params = dict(minmass=300.0, separation=8)
    want, _ = gpu_tracking.batch_rust(movie, 7, **params)
    assert _native.last_stats()["locate_kernel"] == 2  # the TMA-staged kernel ran
    _native.set_option("locate_tiles_per_cta", per_cta)
    _native.set_option("test_withhold_tile_copy", 1)
    try:
        with pytest.raises(_native.GtError) as e:
            gpu_tracking.batch_rust(movie, 7, **params)
        assert e.value.status == _native.GT_ERR_DEVICE_TIMEOUT
    finally:
        _native.set_option("test_withhold_tile_copy", 0)
    try:
        got, _ = gpu_tracking.batch_rust(movie, 7, **params)
    finally:
        _native.set_option("locate_tiles_per_cta", 0)
    np.testing.assert_array_equal(got, want)
