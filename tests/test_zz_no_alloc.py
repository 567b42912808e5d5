"""gt_locate_frame_static: locating one frame with no memory allocation.

Callers that cannot allocate device memory get this entry point: processes
whose device memory belongs to another framework's pool (a cudaMalloc beside
it can fail or fragment it) and acquisition loops that forbid allocation
once running.  All its scratch is one fixed __device__ array inside
libgt.so.  The tests call it through the C ABI and check that its rows equal
those of the regular entry point (gt_batch_device, which allocates its
workspace) for the same frame, on two calls in a row, since the shared
scratch keeps the previous call's contents.  The file is collected last, so
that a run stopping at its first failure has run every other test.
"""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from tracking_optimizations_b200 import _native, synth

pytestmark = pytest.mark.gpu

# (name, params, frame dtype): the specialised u16 kernel, float frames and a
# diameter without a specialised kernel (generic kernel), and the extra
# columns whose scratch slices differ (GPU characterisation, raw signal and
# annulus background)
CASES = [
    ("fast_u16", dict(diameter=7, separation=8, minmass=300.0, cpu_processed=True), "u16"),
    ("f32_frame", dict(diameter=7, separation=8, minmass=300.0, cpu_processed=True), "f32"),
    ("generic_d13", dict(diameter=13, minmass=300.0), "u16"),
    ("extra_columns", dict(diameter=9, minmass=300.0, characterize=True, cpu_processed=True, sig_radius=3.0,
                           bg_radius=6.0, gap_radius=1.0), "u16"),
]


def ncols_of(params):
    from tracking_optimizations_b200.gpu_tracking import column_names
    p = dict(params)
    d = p.pop("diameter")
    return len(column_names(d, **p))


def to_device(torch, frame, dtype):
    if dtype == "u16":
        return torch.from_numpy(frame.view(np.int16).copy()).cuda(), _native.GT_U16
    return torch.from_numpy(frame.astype(np.float32)).cuda(), _native.GT_F32


def regular(lib, ctx, d_frame, dt, H, W, params, ncols, torch):
    out = torch.zeros((H * W // 16, ncols), dtype=torch.float32, device="cuda")
    n = ctypes.c_int64()
    st = lib.gt_batch_device(ctx, ctypes.c_void_p(d_frame.data_ptr()), dt, 1, H, W,
                             ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), out.shape[0],
                             ctypes.byref(n), None)
    _native.check(st, ctx)
    return out[: n.value].cpu().numpy()


def static(lib, d_frame, dt, H, W, params, ncols, torch, fill):
    out = torch.full((H * W // 16, ncols), fill, dtype=torch.float32, device="cuda")
    n = ctypes.c_int64(-1)
    st = lib.gt_locate_frame_static(ctypes.c_void_p(d_frame.data_ptr()), dt, H, W,
                                    ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), out.shape[0],
                                    ctypes.byref(n), None)
    if st != _native.GT_OK:
        raise _native.GtError(st, lib.gt_last_error(None).decode())
    return out[: n.value].cpu().numpy()


@pytest.mark.parametrize("name,kw,dtype", CASES, ids=[c[0] for c in CASES])
def test_static_entry_matches_regular_entry_twice(name, kw, dtype):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "needs a CUDA device"
    lib = _native.load()
    ctx = _native.context(0)
    params = _native.make_params(**kw)
    ncols = ncols_of(kw)
    spec = synth.scaled(synth.PLAIN_1000, frames=2, seed=77)
    movie = synth.make_movie(spec)
    H, W = movie.shape[1:]
    frames = [to_device(torch, movie[i], dtype) for i in range(2)]
    want = [regular(lib, ctx, f, dt, H, W, params, ncols, torch) for f, dt in frames]
    assert all(len(w) > 100 for w in want)
    # two calls in a row on different frames, then the first frame again:
    # each must match although the scratch holds the previous call's data
    for i, fill in [(0, 0.0), (1, -1.0), (0, 7.0)]:
        f, dt = frames[i]
        got = static(lib, f, dt, H, W, params, ncols, torch, fill)
        np.testing.assert_array_equal(got, want[i])


def test_static_entry_rejects_oversize_frames():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    kw = CASES[0][1]
    params = _native.make_params(**kw)
    frame = torch.zeros((2048, 1024), dtype=torch.int16, device="cuda")
    with pytest.raises(_native.GtError, match="static scratch"):
        static(lib, frame, _native.GT_U16, 2048, 1024, params, 7, torch, 0.0)
    linked = _native.make_params(search_range=5.0, **kw)
    with pytest.raises(_native.GtError, match="linking"):
        static(lib, frame[:64, :64].contiguous(), _native.GT_U16, 64, 64, linked, 7, torch, 0.0)


def test_static_entry_reports_capacity():
    """A frame with more features than the scratch holds (32768): diameter 3
    and separation 1 make every positive pixel of a noise frame a feature."""
    torch = pytest.importorskip("torch")
    lib = _native.load()
    rng = np.random.default_rng(5)
    frame = rng.integers(0, 4000, size=(1024, 1024), dtype=np.uint16)
    d_frame = torch.from_numpy(frame.view(np.int16)).cuda()
    params = _native.make_params(diameter=3, separation=1, minmass=0.0)
    with pytest.raises(_native.GtError, match="32768") as e:
        static(lib, d_frame, _native.GT_U16, 1024, 1024, params, 4, torch, 0.0)
    assert e.value.status == _native.GT_ERR_CAPACITY
    # the scratch is usable again afterwards
    kw = CASES[0][1]
    small = synth.make_movie(synth.scaled(synth.PLAIN_1000, frames=1, seed=3))[0]
    f, dt = to_device(torch, small, "u16")
    H, W = small.shape
    got = static(lib, f, dt, H, W, _native.make_params(**kw), 7, torch, 0.0)
    want = regular(lib, _native.context(0), f, dt, H, W, _native.make_params(**kw), 7, torch)
    np.testing.assert_array_equal(got, want)


def test_static_entry_leaves_other_errors_visible():
    """After a successful static call, a failing context-free call still
    reports its own message through gt_last_error(NULL)."""
    torch = pytest.importorskip("torch")
    lib = _native.load()
    kw = CASES[0][1]
    small = synth.make_movie(synth.scaled(synth.PLAIN_1000, frames=1, seed=3))[0]
    f, dt = to_device(torch, small, "u16")
    static(lib, f, dt, small.shape[0], small.shape[1], _native.make_params(**kw), 7, torch, 0.0)
    T, H, W = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    with tempfile.TemporaryDirectory() as tmp:
        missing = os.path.join(tmp, "missing.tif").encode()
        st = lib.gt_file_info(missing, 0, 0, ctypes.byref(T), ctypes.byref(H), ctypes.byref(W))
    assert st != _native.GT_OK
    msg = lib.gt_last_error(None).decode()
    assert "missing.tif" in msg
