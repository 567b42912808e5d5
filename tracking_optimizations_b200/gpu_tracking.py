"""Module-level functions of the reference's pyo3 module `gpu_tracking`
(gpu-tracking/src/lib.rs:44-236), backed by libgt.so on a B200.

Same names, positional order and defaults:
  batch_rust(pyarr, diameter, minmass, maxsize, separation, noise_size,
             smoothing_size, threshold, invert, percentile, topn, preprocess,
             max_iterations, characterize, filter_close, search_range, memory,
             cpu_processed, sig_radius, bg_radius, gap_radius)
      -> (float32 array [rows, cols], [(name, type), ...])
  link_rust(pyarr, search_range, memory=None) -> uint64 array
  batch_file_rust(filename, diameter, channel=None, ...) -> as batch_rust
  parse_ets(path) -> {channel: uint16 array}
The reference accepts float32 frames only (lib.rs:50); uint16 frames are
accepted as well.  Unsupported options raise NotImplementedError as the
reference's `not_implemented!` does (lib.rs:28-39, 73-74).
"""
import ctypes
import os
import weakref

import numpy as np

from . import _native

PARAM_ORDER = ["minmass", "maxsize", "separation", "noise_size", "smoothing_size", "threshold", "invert",
               "percentile", "topn", "preprocess", "max_iterations", "characterize", "filter_close",
               "search_range", "memory", "cpu_processed", "sig_radius", "bg_radius", "gap_radius"]


def _frames_array(pyarr):
    arr = np.asarray(pyarr)
    if arr.ndim != 3:
        raise ValueError(f"expected a (frames, rows, cols) array, got shape {arr.shape}")
    if arr.dtype == np.uint16:
        dtype = _native.GT_U16
    elif arr.dtype == np.float32:
        dtype = _native.GT_F32
    else:
        raise TypeError(f"frames must be float32 or uint16, got {arr.dtype}")
    if not arr.flags["C_CONTIGUOUS"]:
        # execute_gpu.rs:497-499 rejects non-standard layouts
        raise ValueError("Array is not standard layout")
    return arr, dtype


def batch_rust(pyarr, diameter, minmass=None, maxsize=None, separation=None, noise_size=None,
               smoothing_size=None, threshold=None, invert=None, percentile=None, topn=None, preprocess=None,
               max_iterations=None, characterize=None, filter_close=None, search_range=None, memory=None,
               cpu_processed=None, sig_radius=None, bg_radius=None, gap_radius=None, device=0):
    """Locate (and link when search_range is given) features in every frame."""
    arr, dtype = _frames_array(pyarr)
    vals = dict(minmass=minmass, maxsize=maxsize, separation=separation, noise_size=noise_size,
                smoothing_size=smoothing_size, threshold=threshold, invert=invert, percentile=percentile,
                topn=topn, preprocess=preprocess, max_iterations=max_iterations, characterize=characterize,
                filter_close=filter_close, search_range=search_range, memory=memory,
                cpu_processed=cpu_processed, sig_radius=sig_radius, bg_radius=bg_radius,
                gap_radius=gap_radius)
    params = _native.make_params(diameter, **vals)
    lib = _native.load()
    ctx = _native.context(device)
    tab = _native.GtTable()
    T, H, W = arr.shape
    st = lib.gt_batch(ctx, arr.ctypes.data_as(ctypes.c_void_p), dtype, T, H, W, ctypes.byref(params),
                      ctypes.byref(tab))
    _native.check(st, ctx)
    try:
        n, c = tab.nrows, tab.ncols
        cols = [(tab.names[i].value.decode(), tab.types[i].value.decode()) for i in range(c)]
        out = _adopt_table(lib, tab, n, c)
    except BaseException:
        lib.gt_table_free(ctypes.byref(tab))
        raise
    return out, cols


def _adopt_table(lib, tab, n, c):
    """The (n, c) float32 table that libgt allocated, as a numpy array that
    owns it: no copy; gt_table_free runs when the array is collected."""
    buf = (ctypes.c_float * max(n * c, 1)).from_address(ctypes.addressof(tab.data.contents))
    keep = _native.GtTable()
    ctypes.pointer(keep)[0] = tab
    weakref.finalize(buf, lib.gt_table_free, ctypes.byref(keep))
    return np.frombuffer(buf, dtype=np.float32, count=n * c).reshape(n, c)


def batch_device(frames, diameter, **params):
    """gt_batch_device on a (T, H, W) CUDA tensor (float32, or int16/uint16
    holding u16 pixels) on the current stream; returns the table as an
    (n, ncols) float32 CUDA tensor."""
    import torch

    if not frames.is_cuda or frames.dim() != 3:
        raise ValueError("frames must be a (T, H, W) CUDA tensor")
    fr = frames.contiguous()
    dtype = _native.GT_F32 if fr.dtype == torch.float32 else _native.GT_U16
    if fr.dtype not in (torch.float32, torch.int16) and not (hasattr(torch, "uint16") and fr.dtype == torch.uint16):
        raise TypeError("frames must be float32, or int16/uint16 holding u16 pixels")
    ncols = len(column_names(diameter, **params))
    p = _native.make_params(diameter, **params)
    lib = _native.load()
    index = fr.device.index if fr.device.index is not None else torch.cuda.current_device()
    ctx = _native.context(index)
    T, H, W = fr.shape
    cap = max(1024, T * max(64, H * W // 256))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        out = torch.empty((cap, ncols), dtype=torch.float32, device=fr.device)
        n = ctypes.c_int64()
        st = lib.gt_batch_device(ctx, ctypes.c_void_p(fr.data_ptr()), dtype, T, H, W, ctypes.byref(p),
                                 ctypes.c_void_p(out.data_ptr()), cap, ctypes.byref(n), stream)
        _native.check(st, ctx)
        if n.value <= cap:
            return out[: n.value]
        cap = n.value
    raise RuntimeError("row count changed between two identical calls")


def batch_file_rust(filename, diameter, channel=None, minmass=None, maxsize=None, separation=None, noise_size=None,
                    smoothing_size=None, threshold=None, invert=None, percentile=None, topn=None, preprocess=None,
                    max_iterations=None, characterize=None, filter_close=None, search_range=None, memory=None,
                    cpu_processed=None, sig_radius=None, bg_radius=None, gap_radius=None, device=0):
    """Locate (and link) the frames of a .tif/.tiff or .ets movie file
    (lib.rs:124-200 -> execute_gpu.rs:510-542); `channel` selects the ETS
    channel (0 by default) and is ignored for TIFF."""
    vals = dict(minmass=minmass, maxsize=maxsize, separation=separation, noise_size=noise_size,
                smoothing_size=smoothing_size, threshold=threshold, invert=invert, percentile=percentile,
                topn=topn, preprocess=preprocess, max_iterations=max_iterations, characterize=characterize,
                filter_close=filter_close, search_range=search_range, memory=memory,
                cpu_processed=cpu_processed, sig_radius=sig_radius, bg_radius=bg_radius,
                gap_radius=gap_radius)
    params = _native.make_params(diameter, **vals)
    lib = _native.load()
    ctx = _native.context(device)
    tab = _native.GtTable()
    st = lib.gt_batch_file(ctx, os.fsencode(filename), 0 if channel is None else 1,
                           0 if channel is None else int(channel), ctypes.byref(params), ctypes.byref(tab))
    _native.check(st, ctx)
    try:
        n, c = tab.nrows, tab.ncols
        cols = [(tab.names[i].value.decode(), tab.types[i].value.decode()) for i in range(c)]
        out = _adopt_table(lib, tab, n, c)
    except BaseException:
        lib.gt_table_free(ctypes.byref(tab))
        raise
    return out, cols


def read_file(path, channel=None):
    """The frames of a movie file as gt_batch_file reads them: (T, H, W)
    uint16 (for ETS, H = dims[0] and W = dims[1])."""
    lib = _native.load()
    T, H, W = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    hc, ch = (0, 0) if channel is None else (1, int(channel))
    _native.check(lib.gt_file_info(os.fsencode(path), hc, ch, ctypes.byref(T), ctypes.byref(H), ctypes.byref(W)), None)
    out = np.empty((T.value, H.value, W.value), np.uint16)
    _native.check(lib.gt_file_read(os.fsencode(path), hc, ch, out.ctypes.data_as(ctypes.c_void_p), out.size), None)
    return out


def parse_ets(path):
    """{channel: uint16 array (frames, dims[1], dims[0])} of an ETS file
    (lib.rs:215-232)."""
    lib = _native.load()
    n, d0, d1 = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    _native.check(lib.gt_ets_channels(os.fsencode(path), None, None, 0, ctypes.byref(n), ctypes.byref(d0),
                                      ctypes.byref(d1)), None)
    chans = np.empty(n.value, np.int32)
    frames = np.empty(n.value, np.int32)
    _native.check(lib.gt_ets_channels(os.fsencode(path), chans.ctypes.data_as(ctypes.c_void_p),
                                      frames.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n),
                                      ctypes.byref(d0), ctypes.byref(d1)), None)
    out = {}
    for c, f in zip(chans.tolist(), frames.tolist()):
        a = np.empty((f, d1.value, d0.value), np.uint16)
        if f:
            _native.check(lib.gt_file_read(os.fsencode(path), 1, c, a.ctypes.data_as(ctypes.c_void_p), a.size),
                          None)
        out[c] = a
    return out


def link_rust(pyarr, search_range, memory=None, device=0):
    """Link a (frame, mass, y, x, ...) float32 table; returns uint64 IDs."""
    arr = np.ascontiguousarray(np.asarray(pyarr, dtype=np.float32))
    if arr.ndim != 2 or arr.shape[1] < 4:
        raise ValueError("expected an (n, >=4) float32 table")
    lib = _native.load()
    ctx = _native.context(device)
    ids = np.empty(arr.shape[0], dtype=np.uint64)
    st = lib.gt_link(ctx, arr.ctypes.data_as(ctypes.c_void_p), arr.shape[0], arr.shape[1], float(search_range),
                     0 if memory is None else 1, 0 if memory is None else int(memory),
                     ids.ctypes.data_as(ctypes.c_void_p))
    _native.check(st, ctx)
    return ids


def column_names(diameter=9, **kw):
    """execute_gpu.rs:197-226 column list for a parameter set."""
    params = _native.make_params(diameter, **kw)
    buf = ctypes.create_string_buffer(1024)
    n = _native.load().gt_column_names(ctypes.byref(params), buf, 1024)
    if n < 0:
        _native.check(-n, None)
    return [tuple(x.split(":")) for x in buf.value.decode().split(",")]
