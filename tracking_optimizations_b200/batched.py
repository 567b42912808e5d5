"""Many movies of uneven size and parameters in one call (gt_batch_many_device).

The reference locates and links one movie per call
(gpu-tracking/src/lib.rs:94-121 batch_rust -> execute_gpu.rs:372-440).  This
entry point takes a list of device-resident movies, each with its own
gpu_tracking.batch keyword arguments, and runs them as one CUDA graph: the
movies' locate / ordering / output kernels as parallel graph branches and all
linking in one cooperative kernel.  Every movie's table equals the one
``gpu_tracking.batch_rust`` returns for it.

Torch supplies device memory and the current stream only.
"""
import ctypes

import torch

from . import _native
from .gpu_tracking import column_names


def _dtype(t):
    if t.dtype == torch.float32:
        return _native.GT_F32
    if t.dtype == torch.int16 or (hasattr(torch, "uint16") and t.dtype == torch.uint16):
        return _native.GT_U16
    raise TypeError("frames must be float32, or int16/uint16 holding u16 pixels")


def output_buffers(movies):
    """Output tensors sized for ``movies`` (see batch_many's ``outs``)."""
    outs = []
    for fr, params in movies:
        kw = dict(params)
        diameter = kw.pop("diameter")
        T, H, W = fr.shape
        cap = max(1024, T * max(64, H * W // 256))
        outs.append(torch.empty((cap, len(column_names(diameter, **kw))), dtype=torch.float32, device=fr.device))
    return outs


def batch_many(movies, device=None, return_stats=False, outs=None):
    """``movies``: list of ``(frames, params)`` with ``frames`` a (T, H, W)
    CUDA tensor and ``params`` a dict of gpu_tracking.batch keyword arguments
    (``diameter`` included).  Returns a list of ``(table, names)`` with
    ``table`` an (n, ncols) float32 CUDA tensor; with ``return_stats`` also
    the call's gt_last_stats dict.

    The CUDA graph of a batch is cached and replayed while the frames,
    parameters and output buffers stay the same: pass the same ``outs``
    (from ``output_buffers``) to successive calls to replay it; the returned
    tables are then views of those buffers."""
    if not movies:
        return ([], {}) if return_stats else []
    frames0 = movies[0][0]
    dev = frames0.device
    index = dev.index if dev.index is not None else torch.cuda.current_device()
    lib = _native.load()
    ctx = _native.context(index if device is None else device)
    arr = (_native.GtMovie * len(movies))()
    keep = []
    names_all = []
    for i, (fr, params) in enumerate(movies):
        if not fr.is_cuda or fr.dim() != 3:
            raise ValueError(f"movie {i}: frames must be a (T, H, W) CUDA tensor")
        fr = fr.contiguous()
        kw = dict(params)
        diameter = kw.pop("diameter")
        names = column_names(diameter, **kw)
        T, H, W = fr.shape
        if outs is not None:
            out = outs[i]
            if out.dim() != 2 or out.shape[1] != len(names) or out.dtype != torch.float32 or not out.is_contiguous():
                raise ValueError(f"movie {i}: output buffer must be a contiguous (rows, {len(names)}) float32 tensor")
            cap = out.shape[0]
        else:
            cap = max(1024, T * max(64, H * W // 256))
            out = torch.empty((cap, len(names)), dtype=torch.float32, device=fr.device)
        m = arr[i]
        m.frames = fr.data_ptr()
        m.dtype = _dtype(fr)
        m.T, m.H, m.W = T, H, W
        m.params = _native.make_params(diameter, **kw)
        m.out = out.data_ptr()
        m.out_rows = cap
        keep.append((fr, out))
        names_all.append(names)
    st = lib.gt_batch_many_device(ctx, arr, len(movies), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _native.check(st, ctx)
    stats = _native.last_stats(index if device is None else device)
    result = []
    for i, (fr, out) in enumerate(keep):
        n = arr[i].nrows
        if n > out.shape[0]:
            # more rows than the guessed capacity: this movie alone again
            from .gpu_tracking import batch_device

            out = batch_device(fr, **movies[i][1])
            result.append((out, names_all[i]))
            continue
        result.append((out[:n], names_all[i]))
    return (result, stats) if return_stats else result
