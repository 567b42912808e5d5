"""Generates tests/golden/reference_dump.npz from the reference's own dump of
its GPU mass plane.

The reference repository holds two files written by its GPU path:
``gpu-tracking/inp`` (a 524 x 800 float32 frame, the grey-lion image, whole
numbers 0..255) and ``gpu-tracking/masses.bin`` (the 524 x 800 float32
``masses`` buffer that centers.wgsl:23-109 wrote over it, with diameter 9,
smoothing_size 9, noise_size 1 and Gaussian taps normalised on the host as
kernels.rs:86-97 does).  The mass plane itself (1.7 MB, incompressible) is
kept only as its SHA-256 digest plus the values the tests read:

* ``inp``: the frame as uint8 (exact: every value is a whole number 0..255);
* ``masses_sha256``: digest of the dump's float32 bytes, row-major;
* ``sample_idx`` / ``sample_mass``: 8192 seeded pixel indices and the dump's
  masses there (diagnostics when the digest differs);
* ``walk`` / ``walk_mass``: the walk records {frame, last-read row, column,
  final row, column} of the rows located on ``inp`` with diameter 9,
  separation 10, minmass 0 (the oracle's walk, which is what the reference's
  walk_cols.wgsl reads), and the dump's mass at each last-read pixel -- the
  mass that row must carry.

Run once where the reference tree is present:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_reference_dump.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
H, W = 524, 800
PARAMS = dict(diameter=9, separation=10, minmass=0.0, normalized_taps=True)


def main():
    ref_root = os.environ.get("REFERENCE_ROOT") or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not ref_root:
        sys.exit("set REFERENCE_ROOT (or pass the reference checkout as the first argument)")
    base = os.path.join(ref_root, "gpu-tracking")
    inp = np.fromfile(os.path.join(base, "inp"), dtype=np.float32).reshape(H, W)
    raw = open(os.path.join(base, "masses.bin"), "rb").read()
    masses = np.frombuffer(raw, dtype=np.float32).reshape(H, W)
    if not (np.array_equal(inp, np.round(inp)) and inp.min() >= 0 and inp.max() <= 255):
        sys.exit("inp is not whole numbers 0..255")

    sys.path.insert(0, ROOT)
    from oracle import oracle
    _, walk, _ = oracle.batch_walk(inp[None], PARAMS["diameter"], separation=PARAMS["separation"],
                                   minmass=PARAMS["minmass"], normalized_taps=True)
    walk_mass = masses[walk[:, 1], walk[:, 2]]
    rng = np.random.default_rng(0)
    sample_idx = np.sort(rng.choice(H * W, size=8192, replace=False)).astype(np.int64)
    np.savez_compressed(
        os.path.join(HERE, "reference_dump.npz"),
        inp=inp.astype(np.uint8),
        masses_sha256=np.array(hashlib.sha256(raw).hexdigest()),
        sample_idx=sample_idx,
        sample_mass=masses.reshape(-1)[sample_idx],
        walk=walk.astype(np.int32),
        walk_mass=walk_mass.astype(np.float32),
    )
    print(f"{len(walk)} located rows, {len(sample_idx)} sampled pixels")


if __name__ == "__main__":
    main()
