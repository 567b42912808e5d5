"""Seeded synthetic Gaussian-spot movies (uint16) for parity tests and the
benchmark.

The reference measures on a lab movie that is not in its repository; these
movies stand in for it with the workload shapes of the benchmark
configurations: Poisson background (optionally plus Gaussian read noise),
isotropic Gaussian spots A*exp(-r^2 / (2 sigma^2)) sampled at pixel centres,
Brownian motion per axis per frame, optional blinking, rounded and clipped to
[0, 65535].
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class MovieSpec:
    frames: int
    height: int
    width: int
    spots: int
    sigma: float
    amp_lo: float
    amp_hi: float
    step: float
    background: float = 100.0
    read_noise: float = 0.0
    blink: float = 0.0
    seed: int = 0
    params: dict = field(default_factory=dict)


# Plain method, CPU-runnable: 10 x 256^2, 50 spots.
PLAIN_SMALL = MovieSpec(10, 256, 256, 50, 1.5, 200.0, 1000.0, 1.0, seed=0,
                        params=dict(diameter=9, separation=10, noise_size=1.0, smoothing_size=9,
                                    minmass=500.0, max_iterations=10, search_range=5.0, memory=0))

# Plain method, throughput on 1 GPU: 1000 x 512^2, 500 spots, read noise, blinking.
PLAIN_1000 = MovieSpec(1000, 512, 512, 500, 1.2, 150.0, 1500.0, 1.5, read_noise=5.0, blink=0.02, seed=1,
                       params=dict(diameter=7, separation=8, noise_size=1.0, smoothing_size=7,
                                   minmass=300.0, search_range=5.0, memory=2))

# Dense linking stress: 200 x 2048^2, 20000 spots, step 2.5, search_range 7, memory 3.
DENSE_LINK = MovieSpec(200, 2048, 2048, 20000, 1.5, 150.0, 1500.0, 2.5, read_noise=5.0, seed=3,
                       params=dict(diameter=9, search_range=7.0, memory=3))


def scaled(spec, frames=None, height=None, width=None, spots=None, seed=None):
    """Same spot model at another size (spot count scales with area unless given)."""
    h = height or spec.height
    w = width or spec.width
    n = spots if spots is not None else max(1, int(round(spec.spots * h * w / (spec.height * spec.width))))
    return MovieSpec(frames or spec.frames, h, w, n, spec.sigma, spec.amp_lo, spec.amp_hi, spec.step,
                     spec.background, spec.read_noise, spec.blink, spec.seed if seed is None else seed,
                     dict(spec.params))


def make_movie(spec, return_truth=False):
    """Render a movie; optionally also the true positions (T, N, 2) and visibility."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    T, H, W, N = spec.frames, spec.height, spec.width, spec.spots
    pos = np.stack([rng.uniform(0, H - 1, N), rng.uniform(0, W - 1, N)], axis=1)
    amp = rng.uniform(spec.amp_lo, spec.amp_hi, N)
    R = int(np.ceil(4 * spec.sigma))
    off = np.arange(-R, R + 1)
    dy, dx = np.meshgrid(off, off, indexing="ij")
    movie = np.empty((T, H, W), np.uint16)
    truth = np.empty((T, N, 2))
    vis = np.empty((T, N), bool)
    inv2s2 = 1.0 / (2.0 * spec.sigma ** 2)
    for t in range(T):
        img = rng.poisson(spec.background, (H, W)).astype(np.float64)
        if spec.read_noise > 0:
            img += rng.normal(0.0, spec.read_noise, (H, W))
        on = rng.random(N) >= spec.blink
        truth[t] = pos
        vis[t] = on
        p = pos[on]
        a = amp[on]
        cy = np.rint(p[:, 0]).astype(np.int64)
        cx = np.rint(p[:, 1]).astype(np.int64)
        rows = cy[:, None, None] + dy[None]
        cols = cx[:, None, None] + dx[None]
        val = a[:, None, None] * np.exp(-((rows - p[:, 0, None, None]) ** 2 +
                                          (cols - p[:, 1, None, None]) ** 2) * inv2s2)
        ok = (rows >= 0) & (rows < H) & (cols >= 0) & (cols < W)
        np.add.at(img, (rows[ok], cols[ok]), val[ok])
        movie[t] = np.clip(np.rint(img), 0, 65535).astype(np.uint16)
        pos = pos + rng.normal(0.0, spec.step, (N, 2))
        # reflect at the borders
        for k, lim in ((0, H - 1), (1, W - 1)):
            c = pos[:, k]
            c = np.where(c < 0, -c, c)
            c = np.where(c > lim, 2 * lim - c, c)
            pos[:, k] = np.clip(c, 0, lim)
    if return_truth:
        return movie, truth, vis
    return movie
