"""Differentiable refinement at fixed peaks.

The located (y, x, mass) of a feature is, once its walk is fixed, a smooth
function of the frame pixels and of ``noise_size`` away from the bandpass
clip (gpu-tracking/src/shaders/preprocess_rows.wgsl:14-53,
preprocess_cols.wgsl:14-61, centers.wgsl:23-109, walk_cols.wgsl:38-74):

    R = G_s * I - B_k * I,   P = max(R, 0)
    mass = sum_circle P,  y = final_row + sum i P / mass,  x = final_col + sum j P / mass

evaluated at the walk's last-read pixel.  ``RefineAtPeaks`` wraps the CUDA
forward and adjoint kernels of libgt (gt_adjoint_forward / _backward) as a
``torch.autograd.Function``:

* gradients flow to the frames (f32), to ``noise_size`` (the Gaussian
  variance) and to ``smoothing_size`` through the declared relaxation: the box
  normalisation 1/k^2 is treated as continuous in k while the window and the
  Gaussian tap count stay fixed (dR/dk = 2 B / k);
* the clip at 0 takes subgradient 0;
* peaks (walk records) are inputs, not differentiated.

``uncertainty`` propagates pixel noise (Poisson scaled by a gain, plus read
noise) through the same Jacobian.  ``calibrate_noise_size`` fits
``noise_size`` to known positions with Adam through this Function.

PyTorch provides device memory, the current stream and autograd only: all
arithmetic runs in libgt's kernels.
"""
import ctypes

import torch

from . import _native

WALK_COLS = 5  # frame, last-read row, last-read column, final row, final column


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _device_index(t):
    return t.device.index if t.device.index is not None else torch.cuda.current_device()


def _check_frames(frames, dtypes):
    if not isinstance(frames, torch.Tensor) or not frames.is_cuda:
        raise TypeError("frames must be a CUDA tensor")
    if frames.dim() == 2:
        frames = frames.unsqueeze(0)
    if frames.dim() != 3:
        raise ValueError("frames must be (T, H, W) or (H, W)")
    if frames.dtype not in dtypes:
        raise TypeError(f"frames dtype must be one of {dtypes}")
    return frames.contiguous()


def locate_with_walk(frames, diameter, **params):
    """Locate (and link, when ``search_range`` is given) device-resident frames.

    ``frames``: (T, H, W) CUDA tensor, float32, or int16/uint16 holding u16
    pixels.  Returns ``(rows, walk, names)``: the gpu_tracking.batch table as
    an (n, ncols) float32 CUDA tensor, the (n, 5) int32 walk records that the
    adjoint functions take, and the column names.
    """
    u16 = [torch.int16] + ([torch.uint16] if hasattr(torch, "uint16") else [])
    frames = _check_frames(frames, [torch.float32] + u16)
    dtype = _native.GT_F32 if frames.dtype == torch.float32 else _native.GT_U16
    T, H, W = frames.shape
    from .gpu_tracking import column_names

    names = column_names(diameter, **params)
    ncols = len(names)
    lib = _native.load()
    dev = _device_index(frames)
    ctx = _native.context(dev)
    p = _native.make_params(diameter, **params)
    cap = max(1024, T * H * W // 256)
    for _ in range(2):
        rows = torch.empty((cap, ncols), dtype=torch.float32, device=frames.device)
        walk = torch.empty((cap, WALK_COLS), dtype=torch.int32, device=frames.device)
        n = ctypes.c_int64()
        st = lib.gt_batch_device_walk(ctx, _ptr(frames), dtype, T, H, W, ctypes.byref(p), _ptr(rows), cap,
                                      ctypes.byref(n), _ptr(walk), _stream())
        _native.check(st, ctx)
        if n.value <= cap:
            return rows[: n.value], walk[: n.value], names
        cap = n.value
    raise RuntimeError("row count changed between two identical calls")


def _params(diameter, noise_size, smoothing_size, params):
    kw = dict(params)
    kw["noise_size"] = float(noise_size)
    if smoothing_size is not None:
        kw["smoothing_size"] = int(round(float(smoothing_size)))
    return _native.make_params(diameter, **kw)


def _walk(walk):
    if walk.dtype != torch.int32 or walk.dim() != 2 or walk.shape[1] != WALK_COLS:
        raise ValueError("walk must be an (n, 5) int32 tensor")
    return walk.contiguous()


class RefineAtPeaks(torch.autograd.Function):
    """(frames, noise_size, smoothing_size) -> (n, 3) [y, x, mass] at fixed walks.

    ``noise_size`` and ``smoothing_size`` are 0-d float64 tensors (their
    values select the forward's parameters; smoothing_size is rounded to the
    integer window).  ``opts`` carries the remaining gpu_tracking.batch
    parameters (``diameter`` included).
    """

    @staticmethod
    def forward(ctx, frames, noise_size, smoothing_size, walk, opts):
        frames = _check_frames(frames, [torch.float32])
        walk = _walk(walk)
        opts = dict(opts)
        diameter = opts.pop("diameter")
        p = _params(diameter, noise_size.item(), smoothing_size.item(), opts)
        T, H, W = frames.shape
        n = walk.shape[0]
        out = torch.empty((n, 3), dtype=torch.float32, device=frames.device)
        lib = _native.load()
        gctx = _native.context(_device_index(frames))
        st = lib.gt_adjoint_forward(gctx, _ptr(frames), T, H, W, ctypes.byref(p), _ptr(walk), n, _ptr(out),
                                    _stream())
        _native.check(st, gctx)
        ctx.save_for_backward(frames, walk)
        ctx.p = p
        ctx.shape = (T, H, W)
        ctx.params_dtype = (noise_size.dtype, smoothing_size.dtype)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        frames, walk = ctx.saved_tensors
        T, H, W = ctx.shape
        g = grad_out.contiguous().to(torch.float32)
        n = walk.shape[0]
        grad_frames = torch.empty((T, H, W), dtype=torch.float32, device=frames.device)
        grad_par = torch.empty(2, dtype=torch.float64, device=frames.device)
        lib = _native.load()
        gctx = _native.context(_device_index(frames))
        st = lib.gt_adjoint_backward(gctx, _ptr(frames), T, H, W, ctypes.byref(ctx.p), _ptr(walk), n, _ptr(g),
                                     _ptr(grad_frames), _ptr(grad_par), _stream())
        _native.check(st, gctx)
        gs = grad_par[0].to(ctx.params_dtype[0])
        gk = grad_par[1].to(ctx.params_dtype[1])
        return grad_frames, gs, gk, None, None


def refine(frames, walk, diameter, noise_size=None, smoothing_size=None, **params):
    """Differentiable (y, x, mass) of the walks over ``frames`` ((T, H, W) f32).

    ``noise_size`` / ``smoothing_size`` may be floats or 0-d tensors with
    ``requires_grad``; defaults follow gpu_tracking.batch (1 and diameter).
    Returns an (n, 3) float32 tensor.
    """
    dev = frames.device
    ns = noise_size if isinstance(noise_size, torch.Tensor) else torch.tensor(
        1.0 if noise_size is None else float(noise_size), dtype=torch.float64)
    ks = smoothing_size if isinstance(smoothing_size, torch.Tensor) else torch.tensor(
        float(diameter if smoothing_size is None else smoothing_size), dtype=torch.float64)
    opts = dict(params)
    opts["diameter"] = diameter
    return RefineAtPeaks.apply(frames, ns.to(dev) if ns.device != dev else ns,
                               ks.to(dev) if ks.device != dev else ks, walk, opts)


def uncertainty(frames, walk, diameter, gain=1.0, read_noise=0.0, **params):
    """Standard deviations of (y, x, mass) per walk under pixel variance
    gain * max(I, 0) + read_noise^2, by linear propagation through the
    refinement's Jacobian.  Returns an (n, 3) float32 CUDA tensor."""
    frames = _check_frames(frames, [torch.float32])
    walk = _walk(walk)
    T, H, W = frames.shape
    n = walk.shape[0]
    p = _native.make_params(diameter, **params)
    out = torch.empty((n, 3), dtype=torch.float32, device=frames.device)
    lib = _native.load()
    gctx = _native.context(_device_index(frames))
    st = lib.gt_adjoint_uncertainty(gctx, _ptr(frames), T, H, W, ctypes.byref(p), _ptr(walk), n, float(gain),
                                    float(read_noise), _ptr(out), _stream())
    _native.check(st, gctx)
    return out


def calibrate_noise_size(frames, walk, target_yx, diameter, noise_size=1.0, steps=50, lr=0.05, lr_min_frac=0.1,
                         **params):
    """Fit ``noise_size`` so that the refined positions of ``walk`` approach
    ``target_yx`` ((n, 2), e.g. simulated ground truth): Adam on the mean
    squared position error through RefineAtPeaks.  The Gaussian variance is
    optimised in log space so that it stays positive; the learning rate
    decays from ``lr`` to ``lr * lr_min_frac`` on a cosine schedule.
    Returns ``(noise_size, losses)`` with one loss per step (before the
    update).  The parameter gradient is reduced in a fixed order, so the
    same inputs give the same trajectory."""
    import math

    dev = frames.device
    target = target_yx.to(device=dev, dtype=torch.float32)
    log_s = torch.tensor(float(noise_size), dtype=torch.float64, device=dev).log().requires_grad_(True)
    ks = torch.tensor(float(params.pop("smoothing_size", diameter)), dtype=torch.float64, device=dev)
    opt = torch.optim.Adam([log_s], lr=lr)
    losses = []
    for i in range(steps):
        for g in opt.param_groups:
            g["lr"] = lr * (lr_min_frac + (1.0 - lr_min_frac) * 0.5 * (1.0 + math.cos(math.pi * i / steps)))
        opt.zero_grad()
        yxm = refine(frames, walk, diameter, noise_size=log_s.exp(), smoothing_size=ks, **params)
        loss = ((yxm[:, :2] - target) ** 2).sum(dim=1).mean()
        loss.backward()
        losses.append(float(loss.item()))
        opt.step()
    return float(log_s.exp().item()), losses
