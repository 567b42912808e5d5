"""Regenerates the golden fixtures of this directory from the oracle.

The reference cannot run here (Rust host, WGSL through wgpu), so the
fixtures are the oracle's outputs on the seeded workloads, pinned once the
oracle passed the known-answer tests (tests/test_oracle_kat.py): the CPU
suite checks that the oracle still reproduces them, the GPU suite that the
CUDA path does.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle  # noqa: E402
from tracking_optimizations_b200 import synth  # noqa: E402

CASES = {
    # 10 x 256^2 u16, 50 spots, d 9, sep 10, k 9, minmass 500, sr 5, memory 0
    "plain_small": (synth.PLAIN_SMALL, dict(cpu_processed=True)),
    # 40 frames of the 512^2 spot model (500 spots, read noise, blinking), memory 2
    "plain_512_40": (synth.scaled(synth.PLAIN_1000, frames=40), dict(cpu_processed=True)),
    # same movie, characterize columns and raw signal/background columns, no linking
    "plain_512_8_columns": (synth.scaled(synth.PLAIN_1000, frames=8),
                            dict(characterize=True, sig_radius=4.0, bg_radius=7.0, gap_radius=1.0,
                                 search_range=None, memory=None)),
}


def compute(name):
    spec, extra = CASES[name]
    params = dict(spec.params)
    params.update(extra)
    params = {k: v for k, v in params.items() if v is not None}
    movie = synth.make_movie(spec)
    rows, cols = oracle.batch(movie, nthreads=os.cpu_count() or 1, **params)
    _, walk, _ = oracle.batch_walk(movie.astype(np.float32), nthreads=os.cpu_count() or 1,
                                   **{k: v for k, v in params.items()
                                      if k not in ("sig_radius", "bg_radius", "gap_radius", "characterize",
                                                   "cpu_processed")})
    return rows, walk, [c for c, _ in cols], params


def main():
    for name in CASES:
        rows, walk, names, params = compute(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), rows=rows, walk=walk, names=np.array(names))
        print(name, rows.shape, walk.shape)


if __name__ == "__main__":
    main()
