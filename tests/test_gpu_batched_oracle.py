"""The batched uneven-movie path (gt_batch_many_device) against the oracle,
on a slice of the 64-movie uneven workload (synth.batch_workload): nine of
its movies truncated to 6 frames, covering every diameter (5, 7, 9, 11),
memory 0-3, frames from 128x128 to 2048x4096 (the densest movie of the
workload, 22,004 spots per frame) -- every row and trajectory id bit for
bit, in one call that runs them as parallel graph branches with a shared
linker launch."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle
from tracking_optimizations_b200 import batched, synth

pytestmark = pytest.mark.gpu

PICK = [7, 54, 4, 14, 11, 13, 2, 12, 48]  # indices into synth.batch_workload()


def test_batched_slice_matches_oracle(gpu):
    specs = synth.batch_workload()
    chosen = [synth.scaled(specs[i], frames=6) for i in PICK]
    assert {s.params["diameter"] for s in chosen} == {5, 7, 9, 11}
    assert {s.params["memory"] for s in chosen} == {0, 1, 2, 3}
    assert any(s.height == 2048 and s.width == 4096 for s in chosen)
    host = [synth.make_movie(s) for s in chosen]
    movies = [(torch.from_numpy(m.view(np.int16)).cuda(), dict(s.params)) for m, s in zip(host, chosen)]
    got, stats = batched.batch_many(movies, return_stats=True)
    for k, (m, s) in enumerate(zip(host, chosen)):
        params = dict(s.params)
        d = params.pop("diameter")
        want, cols = oracle.batch(m, d, nthreads=os.cpu_count() or 8, **params)
        table, names = got[k]
        assert [c for c, _ in names] == [c for c, _ in cols]
        np.testing.assert_array_equal(table.cpu().numpy(), want, err_msg=f"movie {PICK[k]}")
    print(f"batched slice: {sum(g[0].shape[0] for g in got)} rows, fallbacks {stats['batch_fallbacks']}")
