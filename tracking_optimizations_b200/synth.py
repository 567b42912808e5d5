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
        img += np.bincount((rows[ok] * W + cols[ok]).ravel(), weights=val[ok].ravel(),
                           minlength=H * W).reshape(H, W)
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


def batch_workload(n=64, seed=2):
    """Uneven movies for the batched path: side in {128, 256, 384, 512,
    1024, 2048}, aspect 1 or 2, T ~ U{10..500}, 0.5-3 spots per 1000 px^2,
    diameter in {5, 7, 9, 11} with separation = diameter + 1, search_range ~
    U(3, 8); spot model of PLAIN_1000 (sigma 1.2, A ~ U(150, 1500), step 1.5,
    Poisson 100 + read noise 5, 2 % blinking).  Parameters the workload
    leaves open: minmass = 6 d^2 (300 for d = 7, as PLAIN_1000) and memory ~
    U{0..3}.  About 23 Gpx (47 GB of u16) in total: render with
    make_movie_device."""
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for i in range(n):
        side = int(rng.choice([128, 256, 384, 512, 1024, 2048]))
        aspect = int(rng.choice([1, 2]))
        H, W = side, side * aspect
        T = int(rng.integers(10, 501))
        density = float(rng.uniform(0.5, 3.0))
        d = int(rng.choice([5, 7, 9, 11]))
        params = dict(diameter=d, separation=d + 1, minmass=float(6 * d * d),
                      search_range=float(rng.uniform(3.0, 8.0)), memory=int(rng.integers(0, 4)))
        specs.append(MovieSpec(T, H, W, max(1, int(round(density * H * W / 1000.0))), 1.2, 150.0, 1500.0, 1.5,
                               read_noise=5.0, blink=0.02, seed=seed * 1000 + i, params=params))
    return specs


def spot_tracks(spec):
    """(T, N, 3) float32 (y, x, amplitude) of every spot in every frame, the
    motion model of make_movie (uniform start, Brownian steps reflected at
    the borders, amplitude 0 while blinked off), from its own seeded
    stream."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    T, H, W, N = spec.frames, spec.height, spec.width, spec.spots
    pos = np.stack([rng.uniform(0, H - 1, N), rng.uniform(0, W - 1, N)], axis=1)
    amp = rng.uniform(spec.amp_lo, spec.amp_hi, N)
    out = np.empty((T, N, 3), np.float32)
    for t in range(T):
        on = rng.random(N) >= spec.blink
        out[t, :, 0] = pos[:, 0]
        out[t, :, 1] = pos[:, 1]
        out[t, :, 2] = np.where(on, amp, 0.0)
        pos = pos + rng.normal(0.0, spec.step, (N, 2))
        for k, lim in ((0, H - 1), (1, W - 1)):
            c = pos[:, k]
            c = np.where(c < 0, -c, c)
            c = np.where(c > lim, 2 * lim - c, c)
            pos[:, k] = np.clip(c, 0, lim)
    return out


def make_movie_device(spec, device="cuda", chunk=16):
    """Render ``spec`` on the device (libgt gt_synth_render: Philox4x32-10
    noise, the make_movie spot model).  Returns a (T, H, W) int16 CUDA
    tensor holding the u16 pixels."""
    import ctypes

    import torch

    from . import _native

    tracks = torch.from_numpy(spot_tracks(spec)).to(device)
    T, H, W = spec.frames, spec.height, spec.width
    out = torch.empty((T, H, W), dtype=torch.int16, device=device)
    scratch = torch.empty((min(chunk, T), H, W), dtype=torch.float32, device=device)
    rc = _native.load().gt_synth_render(ctypes.c_void_p(tracks.data_ptr()), spec.spots, T, H, W, spec.sigma,
                                        spec.background, spec.read_noise, spec.seed, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(scratch.data_ptr()), min(chunk, T),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        raise RuntimeError(f"gt_synth_render failed ({rc})")
    torch.cuda.current_stream().synchronize()
    return out
