"""Adjoint of bandpass + refinement at fixed peaks on the GPU.

Checks, through the C ABI (via tracking_optimizations_b200.adjoint):
* the walk records of gt_batch_device_walk equal the oracle's, and the
  fixed-peak forward reproduces the located rows bit for bit;
* dL/dframes against FP64 central differences (step 1e-3, 32 random pixels
  per particle) and against a torch float64 autograd gradient, and
  dL/dnoise_size, dL/dsmoothing_size (box normalisation 1/k^2 relaxed) the
  same way, all at <= 1e-4 relative error;
* the propagated localisation uncertainty against the FP64 Jacobian and a
  Monte Carlo estimate;
* 50 Adam steps calibrating noise_size to a target made by the forward
  model at a known noise_size (an interior optimum), repeatable bit for
  bit.

Particles whose circle holds a bandpass value within 1e-2 of the clip are
left out of the gradient comparisons: an FP32 and an FP64 evaluation may
disagree about the clip there, and so may the two sides of a finite
difference.  The tests count them.
"""
import ctypes

import numpy as np
import pytest

from oracle import adjoint_ref, oracle
from tracking_optimizations_b200 import _native, synth

pytestmark = pytest.mark.gpu

D, K, S = 7, 7, 1.0
PARAMS = dict(separation=8, minmass=300.0)
REL = 1e-4


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    assert t.cuda.is_available(), "needs a CUDA device"
    return t


@pytest.fixture(scope="module")
def adj(torch):
    from tracking_optimizations_b200 import adjoint

    return adjoint


@pytest.fixture(scope="module")
def scene(torch, adj):
    spec = synth.scaled(synth.PLAIN_1000, frames=3, height=96, width=128, spots=24, seed=11)
    movie = synth.make_movie(spec)
    f32 = movie.astype(np.float32)
    frames = torch.from_numpy(f32).cuda()
    rows, walk, names = adj.locate_with_walk(frames, D, noise_size=S, smoothing_size=K, **PARAMS)
    return f32, frames, rows, walk


def test_walk_records_match_oracle_and_forward_is_bit_exact(torch, adj, scene):
    f32, frames, rows, walk = scene
    want_rows, want_walk, _ = oracle.batch_walk(f32, D, noise_size=S, smoothing_size=K, **PARAMS)
    np.testing.assert_array_equal(rows.cpu().numpy(), want_rows)
    np.testing.assert_array_equal(walk.cpu().numpy(), want_walk)
    yxm = adj.refine(frames, walk, D, noise_size=S, smoothing_size=K, **PARAMS)
    r = rows.cpu().numpy()
    np.testing.assert_array_equal(yxm.cpu().numpy(), r[:, [2, 3, 1]])


def test_forward_from_u16_walk_matches(torch, adj, scene):
    # walks found by the specialised u16 kernel drive the f32 adjoint
    f32, frames, rows, walk = scene
    u16 = torch.from_numpy(f32.astype(np.uint16).view(np.int16)).cuda()
    rows16, walk16, _ = adj.locate_with_walk(u16, D, noise_size=S, smoothing_size=K, **PARAMS)
    assert torch.equal(walk16, walk)
    yxm = adj.refine(frames, walk16, D, noise_size=S, smoothing_size=K, **PARAMS)
    np.testing.assert_array_equal(yxm.cpu().numpy(), rows16.cpu().numpy()[:, [2, 3, 1]])


def _kept(f32, walk_np):
    margin = adjoint_ref.clip_margin(f32, walk_np, D, S, K)
    keep = margin > 1e-2
    assert keep.mean() > 0.8, f"too many near-clip particles: {np.sum(~keep)} of {len(keep)}"
    return keep


def _gpu_backward(torch, adj, frames, walk, up):
    fr = frames.clone().requires_grad_(True)
    ns = torch.tensor(S, dtype=torch.float64, device="cuda", requires_grad=True)
    ks = torch.tensor(float(K), dtype=torch.float64, device="cuda", requires_grad=True)
    yxm = adj.refine(fr, walk, D, noise_size=ns, smoothing_size=ks, **PARAMS)
    (yxm.double() * torch.from_numpy(up).cuda()).sum().backward()
    return fr.grad.cpu().numpy(), float(ns.grad), float(ks.grad)


def test_pixel_gradient_vs_torch_fp64(torch, adj, scene):
    f32, frames, rows, walk = scene
    wn = walk.cpu().numpy()
    keep = _kept(f32, wn)
    wk = wn[keep]
    rng = np.random.default_rng(3)
    up = rng.normal(size=(len(wk), 3))
    up[:, 2] *= 1e-3
    g_gpu, gs_gpu, gk_gpu = _gpu_backward(torch, adj, frames, torch.from_numpy(wk).cuda(), up)
    g_ref, gs_ref, gk_ref = adjoint_ref.torch_reference(f32, wk, up, D, S, K)
    scale = np.abs(g_ref).max()
    err = np.abs(g_gpu - g_ref).max()
    print(f"pixel grad: max |err| / max |g| = {err / scale:.3e}; ds {gs_gpu:.6e} vs {gs_ref:.6e}; "
          f"dk {gk_gpu:.6e} vs {gk_ref:.6e}")
    assert err <= REL * scale
    # element-wise on every pixel whose gradient is at least 1 % of the largest
    big = np.abs(g_ref) >= 1e-2 * scale
    assert np.all(np.abs(g_gpu - g_ref)[big] <= REL * np.abs(g_ref)[big] + 1e-6 * scale)
    assert abs(gs_gpu - gs_ref) <= REL * abs(gs_ref)
    assert abs(gk_gpu - gk_ref) <= REL * abs(gk_ref)
    # no gradient outside the particles' windows
    assert np.all(g_gpu[g_ref == 0] == 0)


def test_pixel_gradient_interior_tiles_vs_torch_fp64(torch, adj):
    """A frame wide and tall enough for transpose tiles away from every edge
    (the register-blocked interior passes) besides the edge tiles."""
    spec = synth.scaled(synth.PLAIN_1000, frames=2, height=160, width=256, spots=60, seed=19)
    f32 = synth.make_movie(spec).astype(np.float32)
    frames = torch.from_numpy(f32).cuda()
    rows, walk, names = adj.locate_with_walk(frames, D, noise_size=S, smoothing_size=K, **PARAMS)
    wn = walk.cpu().numpy()
    wk = wn[_kept(f32, wn)]
    assert len(wk) > 40
    rng = np.random.default_rng(8)
    up = rng.normal(size=(len(wk), 3))
    up[:, 2] *= 1e-3
    g_gpu, gs_gpu, gk_gpu = _gpu_backward(torch, adj, frames, torch.from_numpy(wk).cuda(), up)
    g_ref, gs_ref, gk_ref = adjoint_ref.torch_reference(f32, wk, up, D, S, K)
    scale = np.abs(g_ref).max()
    big = np.abs(g_ref) >= 1e-2 * scale
    assert np.abs(g_gpu - g_ref).max() <= REL * scale
    assert np.all(np.abs(g_gpu - g_ref)[big] <= REL * np.abs(g_ref)[big] + 1e-6 * scale)
    assert abs(gs_gpu - gs_ref) <= REL * abs(gs_ref)
    assert abs(gk_gpu - gk_ref) <= REL * abs(gk_ref)


def test_pixel_gradient_vs_central_differences(torch, adj, scene):
    f32, frames, rows, walk = scene
    wn = walk.cpu().numpy()
    wk = wn[_kept(f32, wn)][:12]
    rng = np.random.default_rng(4)
    up = rng.normal(size=(len(wk), 3))
    up[:, 2] *= 1e-3
    g_gpu, gs_gpu, gk_gpu = _gpu_backward(torch, adj, frames, torch.from_numpy(wk).cuda(), up)
    samples = adjoint_ref.fd_pixels(f32, wk, up, D, S, K, npix=32, h=1e-3, seed=5)
    fd = np.array([d for *_, d in samples])
    got = np.array([g_gpu[t, u, v] for t, u, v, _ in samples])
    scale = np.abs(fd).max()
    print(f"FD pixel samples {len(samples)}: max |err| / max |g| = {np.abs(got - fd).max() / scale:.3e}")
    assert np.all(np.abs(got - fd) <= REL * np.maximum(np.abs(fd), 1e-2 * scale))
    ds, dk = adjoint_ref.fd_params(f32, wk, up, D, S, K, h=1e-3)
    assert abs(gs_gpu - ds) <= REL * abs(ds)
    assert abs(gk_gpu - dk) <= REL * abs(dk)


def test_config4_gradient_vs_central_differences(torch, adj):
    """The differentiation workload itself: 256 frames of 512 x 512 f32
    with the throughput movie's spot model, diameter 7.  24 particles
    sampled across the frames (away from the clip), dL/dpixel against FP64
    central differences (step 1e-3) on 32 random pixels of each particle's
    window, and dL/dnoise_size, dL/dsmoothing_size likewise."""
    spec = synth.scaled(synth.PLAIN_1000, frames=256, seed=31)
    f32 = synth.make_movie(spec).astype(np.float32)
    frames = torch.from_numpy(f32).cuda()
    rows, walk, _ = adj.locate_with_walk(frames, D, noise_size=S, smoothing_size=K, **PARAMS)
    wn = walk.cpu().numpy()
    assert len(wn) > 256 * 300
    rng = np.random.default_rng(12)
    pick = np.sort(rng.choice(len(wn), size=64, replace=False))
    wk = wn[pick]
    wk = wk[_kept(f32, wk)][:24]
    assert len(wk) == 24 and len(np.unique(wk[:, 0])) > 12
    up = rng.normal(size=(len(wk), 3))
    up[:, 2] *= 1e-3
    g_gpu, gs_gpu, gk_gpu = _gpu_backward(torch, adj, frames, torch.from_numpy(wk).cuda(), up)
    samples = adjoint_ref.fd_pixels(f32, wk, up, D, S, K, npix=32, h=1e-3, seed=13)
    fd = np.array([d for *_, d in samples])
    got = np.array([g_gpu[t, u, v] for t, u, v, _ in samples])
    scale = np.abs(fd).max()
    print(f"config[4] FD samples {len(samples)}: max |err| / max |g| = {np.abs(got - fd).max() / scale:.3e}")
    assert len(samples) == 24 * 32
    assert np.all(np.abs(got - fd) <= REL * np.maximum(np.abs(fd), 1e-2 * scale))
    # parameter derivatives on the particles whose circle stays 0.1 from the
    # clip: a step of 1e-3 in smoothing_size moves the boxcar term by
    # 2 B / k * 1e-3 (about 0.04 here), which must not carry a pixel across
    # the clip inside the central difference
    far = adjoint_ref.clip_margin(f32, wk, D, S, K) > 0.1
    assert far.sum() >= 12
    wf, uf = wk[far], up[far]
    _, gs_gpu, gk_gpu = _gpu_backward(torch, adj, frames, torch.from_numpy(wf).cuda(), uf)
    ds, dk = adjoint_ref.fd_params(f32, wf, uf, D, S, K, h=1e-3)
    assert abs(gs_gpu - ds) <= REL * abs(ds)
    assert abs(gk_gpu - dk) <= REL * abs(dk)


def test_uncertainty_vs_fp64_jacobian(torch, adj, scene):
    f32, frames, rows, walk = scene
    wn = walk.cpu().numpy()
    wk = wn[_kept(f32, wn)][:8]
    sd = adj.uncertainty(frames, torch.from_numpy(wk).cuda(), D, gain=1.0, read_noise=5.0, noise_size=S,
                         smoothing_size=K, **PARAMS).cpu().numpy()
    ref = adjoint_ref.uncertainty(f32, wk, D, S, K, gain=1.0, read_noise=5.0)
    np.testing.assert_allclose(sd, ref, rtol=REL)


def test_uncertainty_matches_monte_carlo(torch, adj):
    # one spot, 400 noise realisations, positions refined at one fixed walk
    rng = np.random.default_rng(9)
    H = W = 48
    yy, xx = np.mgrid[0:H, 0:W]
    clean = 100.0 + 600.0 * np.exp(-((yy - 24.3) ** 2 + (xx - 23.6) ** 2) / (2 * 1.2 ** 2))
    n = 400
    movie = (rng.poisson(clean, (n, H, W)) + rng.normal(0, 5.0, (n, H, W))).astype(np.float32)
    frames = torch.from_numpy(movie).cuda()
    _, walk0, _ = adj.locate_with_walk(frames[:1], D, noise_size=S, smoothing_size=K, **PARAMS)
    assert walk0.shape[0] == 1
    walk = walk0.repeat(n, 1)
    walk[:, 0] = torch.arange(n, dtype=torch.int32, device="cuda")
    yxm = adj.refine(frames, walk, D, noise_size=S, smoothing_size=K, **PARAMS).cpu().numpy()
    sd = adj.uncertainty(frames, walk, D, gain=1.0, read_noise=5.0, noise_size=S, smoothing_size=K,
                         **PARAMS).cpu().numpy()
    emp = yxm.std(axis=0, ddof=1)
    pred = np.sqrt((sd ** 2).mean(axis=0))
    print(f"Monte Carlo sd {emp} vs propagated {pred}")
    np.testing.assert_allclose(pred, emp, rtol=0.12)


def test_adam_calibrates_noise_size(torch, adj):
    """Calibration with a known interior optimum: the target positions are
    the forward model's own at noise_size 1.6 (fixed peaks of a 6-frame
    256 x 256 scene); 50 Adam steps from noise_size 3.0 must end within one
    step of a 61-point log grid of the loss minimum (which lies at 1.6) and
    with at least 98 % of the achievable loss improvement.  The parameter
    gradient is reduced in a fixed order, so a second run repeats the
    trajectory exactly."""
    S_TRUE = 1.6
    spec = synth.scaled(synth.PLAIN_1000, frames=6, height=256, width=256, spots=120, seed=21)
    frames = torch.from_numpy(synth.make_movie(spec).astype(np.float32)).cuda()
    rows, walk, _ = adj.locate_with_walk(frames, D, noise_size=S, smoothing_size=K, **PARAMS)
    assert walk.shape[0] > 400
    tgt = adj.refine(frames, walk, D, noise_size=S_TRUE, smoothing_size=K, **PARAMS)[:, :2].clone()
    s_fit, losses = adj.calibrate_noise_size(frames, walk, tgt, D, noise_size=3.0, steps=50, lr=0.08,
                                             smoothing_size=K, **PARAMS)
    s_fit2, losses2 = adj.calibrate_noise_size(frames, walk, tgt, D, noise_size=3.0, steps=50, lr=0.08,
                                               smoothing_size=K, **PARAMS)
    assert s_fit2 == s_fit and losses2 == losses

    def loss_at(s):
        yxm = adj.refine(frames, walk, D, noise_size=s, smoothing_size=K, **PARAMS)
        return float(((yxm[:, :2] - tgt) ** 2).sum(dim=1).mean())

    grid = np.sort(np.append(np.exp(np.linspace(np.log(0.5), np.log(4.0), 61)), S_TRUE))
    gl = np.array([loss_at(s) for s in grid])
    best = grid[np.argmin(gl)]
    step = np.log(4.0 / 0.5) / 60
    final = loss_at(s_fit)
    print(f"noise_size 3.0 -> {s_fit:.4f} (grid best {best:.4f}, truth {S_TRUE}); loss {losses[0]:.3e} -> "
          f"{final:.3e} (grid min {gl.min():.3e})")
    assert len(losses) == 50
    assert 0.5 < best < 4.0, "the optimum lies inside the grid"
    assert abs(np.log(s_fit) - np.log(best)) <= step
    assert final <= gl.min() + 0.02 * (losses[0] - gl.min())


def test_full_size_backward_is_linear(torch, adj):
    # 256 frames of 512 x 512 f32: gradients of two upstreams add up
    spec = synth.scaled(synth.PLAIN_1000, frames=256, seed=31)
    movie = synth.make_movie(spec)
    frames = torch.from_numpy(movie.astype(np.float32)).cuda()
    rows, walk, _ = adj.locate_with_walk(frames, D, noise_size=S, smoothing_size=K, **PARAMS)
    n = walk.shape[0]
    assert n > 256 * 300
    yxm = adj.refine(frames, walk, D, noise_size=S, smoothing_size=K, **PARAMS)
    assert torch.equal(yxm, rows[:, [2, 3, 1]])
    lib = _native.load()
    ctx = _native.context(0)
    p = _native.make_params(D, noise_size=S, smoothing_size=K, **PARAMS)
    g1 = torch.randn((n, 3), device="cuda")
    g2 = torch.randn((n, 3), device="cuda")

    def back(g):
        gi = torch.empty_like(frames)
        gp = torch.empty(2, dtype=torch.float64, device="cuda")
        st = lib.gt_adjoint_backward(ctx, ctypes.c_void_p(frames.data_ptr()), 256, 512, 512, ctypes.byref(p),
                                     ctypes.c_void_p(walk.data_ptr()), n, ctypes.c_void_p(g.data_ptr()),
                                     ctypes.c_void_p(gi.data_ptr()), ctypes.c_void_p(gp.data_ptr()), None)
        _native.check(st, ctx)
        return gi, gp

    a, pa = back(g1)
    b, pb = back(g2)
    c, pc = back(g1 + g2)
    assert torch.isfinite(c).all()
    scale = c.abs().max()
    assert (c - (a + b)).abs().max() <= 1e-5 * scale
    assert torch.allclose(pc, pa + pb, rtol=1e-5)
    stats = _native.last_stats(0)
    assert stats["ms_adjoint_dense"] > 0 and stats["ms_adjoint_particles"] > 0


def test_adjoint_rejects_bad_input(torch, adj, scene):
    f32, frames, rows, walk = scene
    bad = walk.clone()
    bad[0, 1] = 10_000
    with pytest.raises(ValueError, match="walk record"):
        adj.refine(frames, bad, D, noise_size=S, smoothing_size=K, **PARAMS)
    with pytest.raises(NotImplementedError, match="diameter"):
        adj.refine(frames, walk, 33, noise_size=S, smoothing_size=K, separation=34)
    with pytest.raises(NotImplementedError, match="percentile"):
        adj.refine(frames, walk, D, percentile=50.0, **PARAMS)
