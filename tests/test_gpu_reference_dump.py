"""The CUDA locate kernels against the reference's own output: every row
located on gpu-tracking/inp carries, bit for bit, the mass that the
reference's GPU wrote into its mass plane (gpu-tracking/masses.bin) at that
row's last-read pixel (walk_cols.wgsl:69-73).

The dump was made with Gaussian taps normalised on the host
(kernels.rs:86-97); the context option ``normalized_taps`` selects that form.
Fixture: tests/golden/reference_dump.npz (tests/golden/make_reference_dump.py).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_dump.npz")


@pytest.mark.parametrize("dtype", ["u16", "f32"])
@pytest.mark.parametrize("kernel", ["fast", "generic"])
def test_located_masses_equal_reference_dump(gpu, dtype, kernel):
    torch = pytest.importorskip("torch")
    from tracking_optimizations_b200 import _native, adjoint

    d = np.load(GOLDEN)
    inp = d["inp"]
    frames = inp.astype(np.uint16).view(np.int16) if dtype == "u16" else inp.astype(np.float32)
    t = torch.from_numpy(np.ascontiguousarray(frames[None])).cuda()
    _native.set_option("normalized_taps", 1)
    _native.set_option("force_generic", int(kernel == "generic"))
    try:
        rows, walk, names = adjoint.locate_with_walk(t, 9, separation=10, minmass=0.0)
        stats = _native.last_stats()
    finally:
        _native.set_option("normalized_taps", 0)
        _native.set_option("force_generic", 0)
    rows = rows.cpu().numpy()
    walk = walk.cpu().numpy()
    # the specialised kernel takes u16 frames only
    assert stats["locate_kernel"] == (0 if kernel == "generic" or dtype == "f32" else 2)
    np.testing.assert_array_equal(walk, d["walk"])
    mass = np.ascontiguousarray(rows[:, [n for n, _ in names].index("mass")])
    assert len(mass) == len(d["walk_mass"]) > 1000
    assert np.array_equal(mass.view(np.uint32), d["walk_mass"].view(np.uint32))
