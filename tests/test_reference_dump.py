"""The oracle against the reference's own output: the mass plane its GPU path
wrote over gpu-tracking/inp (tests/golden/reference_dump.npz, made by
tests/golden/make_reference_dump.py from gpu-tracking/masses.bin).

The dump was made with Gaussian taps normalised on the host
(kernels.rs:86-97); the oracle's ``normalized_taps`` form reproduces it bit
for bit.  The live shaders normalise inside the passes instead
(preprocess_rows.wgsl:52, preprocess_cols.wgsl:54); that form is held to a
mass tolerance of 1e-4 relative against the same dump.
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_dump.npz")


@pytest.fixture(scope="module")
def dump():
    return np.load(GOLDEN)


def ulps(a, b):
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def test_oracle_reproduces_reference_mass_plane(dump):
    inp = dump["inp"].astype(np.float32)
    c = oracle.centers(inp, 9, normalized_taps=True)
    mass = np.ascontiguousarray(c[2])
    idx = dump["sample_idx"]
    assert np.array_equal(mass.reshape(-1)[idx].view(np.uint32), dump["sample_mass"].view(np.uint32))
    # all 419,200 pixels, bit for bit
    assert hashlib.sha256(mass.tobytes()).hexdigest() == str(dump["masses_sha256"])


def test_oracle_rows_carry_reference_masses(dump):
    """Every located row's mass is the dump's mass at its walk's last-read
    pixel (walk_cols.wgsl:69-73)."""
    inp = dump["inp"].astype(np.float32)
    tab, walk, cols = oracle.batch_walk(inp[None], 9, separation=10, minmass=0.0, normalized_taps=True)
    assert np.array_equal(walk, dump["walk"])
    mass = tab[:, [n for n, _ in cols].index("mass")]
    assert len(mass) > 1000
    assert np.array_equal(mass.view(np.uint32), dump["walk_mass"].view(np.uint32))


def test_live_normalisation_within_tolerance_of_reference(dump):
    """The live shaders' in-pass normalisation against the dump: within
    1e-4 relative wherever the mass is at least 10 (every minmass the
    workloads use is far above), 2e-3 absolute everywhere (a few ulps of the
    pixel-scale bandpass terms summed over the circle); the measured gap is
    printed."""
    inp = dump["inp"].astype(np.float32)
    live = oracle.centers(inp, 9)[2].reshape(-1)[dump["sample_idx"]]
    ref = dump["sample_mass"]
    big = ref >= 10.0
    rel = np.abs(live[big].astype(np.float64) - ref[big]) / ref[big]
    u = ulps(live[big], ref[big])
    absd = np.abs(live.astype(np.float64) - ref)
    print(f"live form vs dump: max rel {rel.max():.3g} (mass >= 10), max abs {absd.max():.3g}, "
          f"median ulp {np.median(u):.0f}, identical {np.mean(u == 0):.3f}")
    assert rel.max() <= 1e-4
    assert absd.max() <= 2e-3
