"""The CUDA path against the committed golden fixtures (tests/golden):
bit-exact tables (frame, mass, y, x, particle ids and the extra columns) and
walk records, through the reference-facing entry points."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

import make_golden  # noqa: E402
from tracking_optimizations_b200 import gpu_tracking, synth  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_cuda_path_matches_golden(name):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "needs a CUDA device"
    from tracking_optimizations_b200 import adjoint

    want = np.load(os.path.join(HERE, name + ".npz"))
    spec, extra = make_golden.CASES[name]
    params = dict(spec.params)
    params.update(extra)
    params = {k: v for k, v in params.items() if v is not None}
    movie = synth.make_movie(spec)
    rows, cols = gpu_tracking.batch_rust(movie, **params)
    assert [c for c, _ in cols] == list(want["names"])
    np.testing.assert_array_equal(rows, want["rows"])
    frames = torch.from_numpy(movie.view(np.int16)).cuda()
    lp = {k: v for k, v in params.items()
          if k not in ("sig_radius", "bg_radius", "gap_radius", "characterize", "cpu_processed")}
    d = lp.pop("diameter")
    _, walk, _ = adjoint.locate_with_walk(frames, d, **lp)
    np.testing.assert_array_equal(walk.cpu().numpy(), want["walk"])
