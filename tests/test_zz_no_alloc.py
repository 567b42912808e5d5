"""gt_locate_frame_static: locating one frame with no memory allocation.

Callers that cannot allocate -- code running while a CUDA stream is being
captured, processes whose device memory belongs to another framework's pool,
acquisition loops that forbid allocation once running -- get this entry
point: all its scratch is one fixed __device__ array inside libgt.so.  The
test calls it through the C ABI and checks that its rows equal those of the
regular entry point (gt_batch_device, which allocates its workspace) for the
same frame, on two calls in a row, since the shared scratch keeps the
previous call's contents.
"""
import ctypes

import numpy as np
import pytest

from tracking_optimizations_b200 import _native, synth

pytestmark = pytest.mark.gpu

PARAMS = dict(diameter=7, separation=8, minmass=300.0, cpu_processed=True)


def regular(lib, ctx, d_frame, H, W, params, ncols, torch):
    out = torch.zeros((H * W // 16, ncols), dtype=torch.float32, device="cuda")
    n = ctypes.c_int64()
    st = lib.gt_batch_device(ctx, ctypes.c_void_p(d_frame.data_ptr()), _native.GT_U16, 1, H, W,
                             ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), out.shape[0],
                             ctypes.byref(n), None)
    _native.check(st, ctx)
    return out[: n.value].cpu().numpy()


def static(lib, d_frame, H, W, params, ncols, torch, fill):
    out = torch.full((H * W // 16, ncols), fill, dtype=torch.float32, device="cuda")
    n = ctypes.c_int64(-1)
    st = lib.gt_locate_frame_static(ctypes.c_void_p(d_frame.data_ptr()), _native.GT_U16, H, W,
                                    ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), out.shape[0],
                                    ctypes.byref(n), None)
    if st != _native.GT_OK:
        raise _native.GtError(st, lib.gt_last_error(None).decode())
    return out[: n.value].cpu().numpy()


def test_static_entry_matches_regular_entry_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "needs a CUDA device"
    lib = _native.load()
    ctx = _native.context(0)
    params = _native.make_params(**PARAMS)
    ncols = 7
    spec = synth.scaled(synth.PLAIN_1000, frames=2, seed=77)
    movie = synth.make_movie(spec)
    H, W = movie.shape[1:]
    frames = [torch.from_numpy(movie[i].view(np.int16).copy()).cuda() for i in range(2)]
    want = [regular(lib, ctx, f, H, W, params, ncols, torch) for f in frames]
    assert all(len(w) > 300 for w in want)
    # two calls in a row on different frames, then the first frame again:
    # each must match although the scratch holds the previous call's data
    for i, fill in [(0, 0.0), (1, -1.0), (0, 7.0)]:
        got = static(lib, frames[i], H, W, params, ncols, torch, fill)
        np.testing.assert_array_equal(got, want[i])


def test_static_entry_rejects_oversize_frames():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    params = _native.make_params(**PARAMS)
    frame = torch.zeros((2048, 1024), dtype=torch.int16, device="cuda")
    with pytest.raises(_native.GtError, match="static scratch"):
        static(lib, frame, 2048, 1024, params, 7, torch, 0.0)
    linked = _native.make_params(search_range=5.0, **PARAMS)
    with pytest.raises(_native.GtError, match="linking"):
        static(lib, frame[:64, :64].contiguous(), 64, 64, linked, 7, torch, 0.0)
