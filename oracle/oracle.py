"""ctypes wrapper of liboracle.so, the CPU restatement of the reference path.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path, never part
of it.  Parity against the reference binary is unpinned (the reference can
neither be built nor run here; see gt_oracle.h).  Defaults follow
gpu-tracking/src/lib.rs:77-91, restated here independently of the product.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OrParams(ctypes.Structure):
    _fields_ = [
        ("diameter", ctypes.c_int32), ("minmass", ctypes.c_float), ("separation", ctypes.c_int32),
        ("noise_size", ctypes.c_float), ("smoothing_size", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
        ("characterize", ctypes.c_int32), ("cpu_processed", ctypes.c_int32),
        ("has_search_range", ctypes.c_int32), ("search_range", ctypes.c_float), ("memory", ctypes.c_int32),
        ("has_sig_radius", ctypes.c_int32), ("sig_radius", ctypes.c_float),
        ("has_bg_radius", ctypes.c_int32), ("bg_radius", ctypes.c_float), ("gap_radius", ctypes.c_float),
        ("normalized_taps", ctypes.c_int32),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "gt_oracle.cpp")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        fp = ctypes.POINTER(ctypes.c_float)
        lib.or_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrParams),
                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(fp), ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_int)]
        lib.or_batch_u16.argtypes = lib.or_batch.argtypes
        lib.or_batch_walk.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(OrParams), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p]
        lib.or_link.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                ctypes.c_void_p]
        lib.or_bandpass.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_int, ctypes.c_void_p]
        lib.or_centers.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrParams),
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.or_centers.restype = None
        lib.or_bandpass.restype = None
        lib.or_locate_planes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrParams),
                                         ctypes.c_void_p]
        lib.or_locate_planes.restype = None
        lib.or_dilation.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        lib.or_dilation.restype = None
        lib.or_free.argtypes = [ctypes.c_void_p]
        lib.or_free.restype = None
        _lib = lib
    return _lib


NOT_IMPLEMENTED = ("maxsize", "threshold", "invert", "percentile", "topn", "preprocess")


def resolve(diameter, minmass=None, maxsize=None, separation=None, noise_size=None, smoothing_size=None,
            threshold=None, invert=None, percentile=None, topn=None, preprocess=None, max_iterations=None,
            characterize=None, filter_close=None, search_range=None, memory=None, cpu_processed=None,
            sig_radius=None, bg_radius=None, gap_radius=None, normalized_taps=False):
    """lib.rs:73-91: reject unimplemented options, apply the defaults.

    normalized_taps selects the host-normalised Gaussian taps of
    kernels.rs:86-97 (the form of the reference's mass-plane dump) instead of
    the live shaders' in-pass normalisation."""
    loc = dict(maxsize=maxsize, threshold=threshold, invert=invert, percentile=percentile, topn=topn,
               preprocess=preprocess)
    for name in NOT_IMPLEMENTED:
        if loc[name] is not None:
            raise NotImplementedError(f"{name} is not implemented")
    p = OrParams()
    p.diameter = int(diameter)
    p.minmass = 0.0 if minmass is None else float(minmass)
    p.separation = int(diameter) + 1 if separation is None else int(separation)
    p.noise_size = 1.0 if noise_size is None else float(noise_size)
    p.smoothing_size = int(diameter) if smoothing_size is None else int(smoothing_size)
    p.max_iterations = 10 if max_iterations is None else int(max_iterations)
    p.characterize = int(bool(characterize)) if characterize is not None else 0
    p.cpu_processed = int(bool(cpu_processed)) if cpu_processed is not None else 0
    p.has_search_range = int(search_range is not None)
    p.search_range = 0.0 if search_range is None else float(search_range)
    p.memory = 0 if memory is None else int(memory)
    p.has_sig_radius = int(sig_radius is not None)
    p.sig_radius = 0.0 if sig_radius is None else float(sig_radius)
    p.has_bg_radius = int(bg_radius is not None)
    p.bg_radius = 0.0 if bg_radius is None else float(bg_radius)
    p.gap_radius = 0.0 if gap_radius is None else float(gap_radius)
    p.normalized_taps = int(bool(normalized_taps))
    return p


def columns(p):
    """execute_gpu.rs:197-226."""
    c = [("frame", "int"), ("mass", "float"), ("y", "float"), ("x", "float")]
    if p.has_search_range:
        c.append(("particle", "int"))
    if p.cpu_processed:
        c += [("Rg", "float"), ("ecc", "float"), ("signal", "float")]
    if p.has_sig_radius:
        c.append(("raw_mass", "float"))
    if p.has_bg_radius:
        c += [("raw_bg_median", "float"), ("raw_mass_corrected", "float")]
    if p.characterize:
        c += [("Rg_gpu", "float"), ("raw_mass_gpu", "float"), ("signal_gpu", "float"), ("ecc_gpu", "float")]
    return c


def batch(video, diameter, nthreads=1, fp64=False, **kw):
    """Oracle counterpart of batch_rust: (float32 table, column list)."""
    p = resolve(diameter, **kw)
    if p.has_bg_radius and not p.has_sig_radius:
        raise ValueError("bg_radius requires sig_radius")
    arr = np.ascontiguousarray(video)
    if arr.dtype not in (np.uint16, np.float32):
        raise TypeError("frames must be uint16 or float32")
    T, H, W = arr.shape
    lib = load()
    out = ctypes.POINTER(ctypes.c_float)()
    nr = ctypes.c_int64()
    nc = ctypes.c_int()
    fn = lib.or_batch_u16 if arr.dtype == np.uint16 else lib.or_batch
    st = fn(arr.ctypes.data_as(ctypes.c_void_p), T, H, W, ctypes.byref(p), int(nthreads), int(fp64),
            ctypes.byref(out), ctypes.byref(nr), ctypes.byref(nc))
    try:
        n, c = nr.value, nc.value
        tab = np.ctypeslib.as_array(out, shape=(max(n, 1) * c,))[: n * c].copy().reshape(n, c)
    finally:
        lib.or_free(out)
    if st == 4:
        raise RuntimeError("subnet search budget exceeded")
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    return tab, columns(p)


def batch_walk(video, diameter, nthreads=1, **kw):
    """FP32 batch on float32 frames plus the (n, 5) int32 walk records
    {frame, last-read row, last-read column, final row, final column}."""
    p = resolve(diameter, **kw)
    arr = np.ascontiguousarray(video, dtype=np.float32)
    T, H, W = arr.shape
    lib = load()
    out = ctypes.POINTER(ctypes.c_float)()
    wk = ctypes.POINTER(ctypes.c_int32)()
    nr = ctypes.c_int64()
    nc = ctypes.c_int()
    st = lib.or_batch_walk(arr.ctypes.data_as(ctypes.c_void_p), T, H, W, ctypes.byref(p), int(nthreads),
                           ctypes.byref(out), ctypes.byref(nr), ctypes.byref(nc), ctypes.byref(wk))
    try:
        n, c = nr.value, nc.value
        tab = np.ctypeslib.as_array(out, shape=(max(n, 1) * c,))[: n * c].copy().reshape(n, c)
        walk = np.ctypeslib.as_array(wk, shape=(max(n, 1) * 5,))[: n * 5].copy().reshape(n, 5)
    finally:
        lib.or_free(out)
        lib.or_free(wk)
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    return tab, walk, columns(p)


def link(table, search_range, memory=None):
    """Oracle counterpart of link_rust."""
    arr = np.ascontiguousarray(np.asarray(table, dtype=np.float32))
    ids = np.empty(arr.shape[0], np.uint64)
    st = load().or_link(arr.ctypes.data_as(ctypes.c_void_p), arr.shape[0], arr.shape[1], float(search_range),
                        0 if memory is None else int(memory), ids.ctypes.data_as(ctypes.c_void_p))
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    return ids


def bandpass(frame, smoothing_size, noise_size, normalized_taps=False):
    f = np.ascontiguousarray(frame, dtype=np.float32)
    out = np.empty_like(f)
    load().or_bandpass(f.ctypes.data_as(ctypes.c_void_p), f.shape[0], f.shape[1], int(smoothing_size),
                       float(noise_size), int(bool(normalized_taps)), out.ctypes.data_as(ctypes.c_void_p))
    return out


def centers(frame, diameter, **kw):
    """Dense (c0, c1, mass) planes of centers.wgsl at every pixel."""
    p = resolve(diameter, **kw)
    f = np.ascontiguousarray(frame, dtype=np.float32)
    out = np.zeros((3,) + f.shape, np.float32)
    load().or_centers(f.ctypes.data_as(ctypes.c_void_p), f.shape[0], f.shape[1], ctypes.byref(p),
                      out[0].ctypes.data_as(ctypes.c_void_p), out[1].ctypes.data_as(ctypes.c_void_p),
                      out[2].ctypes.data_as(ctypes.c_void_p))
    return out


def locate_planes(frame, diameter, **kw):
    p = resolve(diameter, **kw)
    f = np.ascontiguousarray(frame, dtype=np.float32)
    planes = np.zeros((3,) + f.shape, np.float32)
    load().or_locate_planes(f.ctypes.data_as(ctypes.c_void_p), f.shape[0], f.shape[1], ctypes.byref(p),
                            planes.ctypes.data_as(ctypes.c_void_p))
    return planes


def dilation(separation):
    d, o = ctypes.c_int(), ctypes.c_int()
    load().or_dilation(int(separation), ctypes.byref(d), ctypes.byref(o))
    return d.value, o.value
