"""Trajectory post-processing of a linked table, on the device.

The lab pipeline (all_cleaned_up/hatzakis_lab_tracking.py:216-232) runs,
after linking: ``trackpy.filter_stubs`` (line 217), ``step_tracker``
(lines 53-83), a per-particle duration (line 223) and ``mp_imsd`` (lines
199-214, trackpy.msd per particle) stacked to (time, particle, msd) rows
(lines 230-232).  The functions here compute the same results with the CUDA
kernels of libgt (gt_filter_stubs, gt_steps, gt_imsd in include/gt.h);
``postprocess`` chains them the way ``tracker`` does.

Particles are taken in pandas' groupby order: ascending id, the rows of a
particle in table order.
"""
import ctypes

import numpy as np

from . import _native


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ids(a):
    a = np.asarray(a)
    if a.dtype.kind == "f":
        if not np.all(np.isfinite(a)) or np.any(a != np.round(a)):
            raise ValueError("particle ids must be integers")
    return _i64(a)


def filter_stubs(ids, threshold=100, device=0, return_counts=False):
    """Boolean mask of the rows whose particle occurs in at least
    ``threshold`` rows (trackpy.filter_stubs as the lab pipeline calls it);
    with ``return_counts`` also the number of rows of each row's particle."""
    ids = _ids(ids)
    n = len(ids)
    keep = np.zeros(n, np.uint8)
    count = np.zeros(n, np.int64)
    nk = ctypes.c_int64()
    lib = _native.load()
    ctx = _native.context(device)
    _native.check(lib.gt_filter_stubs(ctx, _ptr(ids), n, int(threshold), _ptr(keep), _ptr(count),
                                      ctypes.byref(nk)), ctx)
    return (keep.view(bool), count) if return_counts else keep.view(bool)


def steps(ids, x, y, mpp, device=0):
    """step_tracker's arithmetic: returns ``(xs, ys, x_step, y_step,
    steplength, order)`` -- xs, ys = x * mpp, y * mpp (float32, table order);
    the steps (float64) in groupby order, ``order[j]`` the table row of entry
    j."""
    ids, x, y = _ids(ids), _f32(x), _f32(y)
    n = len(ids)
    if len(x) != n or len(y) != n:
        raise ValueError("ids, x and y must have the same length")
    xs, ys = np.empty(n, np.float32), np.empty(n, np.float32)
    xst, yst, ln = np.empty(n, np.float64), np.empty(n, np.float64), np.empty(n, np.float64)
    order = np.empty(n, np.int64)
    lib = _native.load()
    ctx = _native.context(device)
    _native.check(lib.gt_steps(ctx, _ptr(ids), _ptr(x), _ptr(y), n, float(mpp), _ptr(xs), _ptr(ys), _ptr(xst),
                               _ptr(yst), _ptr(ln), _ptr(order)), ctx)
    return xs, ys, xst, yst, ln, order


def step_tracker(df, params):
    """hatzakis_lab_tracking.py:53-83 on a pandas DataFrame with columns x, y
    and particle: scales x and y by ``params.pixel_size`` in place and adds
    x_step, y_step and steplength.  As the lab function does, the step
    columns receive the groupby-ordered values by position (they line up with
    the rows only when the table is sorted by particle).  Returns ``df``."""
    xs, ys, xst, yst, ln, _ = steps(df["particle"].to_numpy(), df["x"].to_numpy(), df["y"].to_numpy(),
                                   params.pixel_size)
    df["x"] = xs
    df["y"] = ys
    df["x_step"] = xst
    df["y_step"] = yst
    df["steplength"] = ln
    return df


def imsd(ids, frames, x, y, mpp, fps, max_lagtime=100, device=0):
    """trackpy.msd per particle, concatenated and stacked as mp_imsd and
    tracker() do: returns ``(time, particle, msd)`` arrays, one entry per
    (lag, particle) with at least one pair, ordered by lag then particle;
    time = lag / fps (float64), particle int64, msd float32."""
    ids, frames, x, y = _ids(ids), _i64(frames), _f32(x), _f32(y)
    n = len(ids)
    if not (len(frames) == len(x) == len(y) == n):
        raise ValueError("ids, frames, x and y must have the same length")
    tab = _native.GtTable()
    lib = _native.load()
    ctx = _native.context(device)
    _native.check(lib.gt_imsd(ctx, _ptr(ids), _ptr(frames), _ptr(x), _ptr(y), n, float(mpp), int(max_lagtime),
                              ctypes.byref(tab)), ctx)
    try:
        m = tab.nrows
        a = np.ctypeslib.as_array(tab.data, shape=(max(m, 1) * 3,))[: m * 3].reshape(m, 3).copy()
    finally:
        lib.gt_table_free(ctypes.byref(tab))
    lag = a[:, 0].astype(np.float64)
    return lag / float(fps), a[:, 1].astype(np.int64), a[:, 2]


def postprocess(df, params):
    """The steps of tracker() after linking (hatzakis_lab_tracking.py:
    217-232) on a linked pandas DataFrame (columns frame, x, y, particle):
    filter_stubs(duration_filter), step_tracker, integer particle ids, the
    per-particle duration, and the MSD of every particle with max_lagtime =
    the longest duration, mpp = pixel_size and fps = tracking_time, on the
    step_tracker-scaled positions -- as tracker() passes them.  Returns
    ``(full_tracked, msd_df)`` with msd_df's columns time, particle, msd."""
    import pandas as pd

    ids = _ids(df["particle"].to_numpy())
    keep, count = filter_stubs(ids, params.duration_filter, return_counts=True)
    cols = {c: df[c].to_numpy()[keep] for c in df.columns}
    ids = ids[keep]
    xs, ys, xst, yst, ln, _ = steps(ids, cols["x"], cols["y"], params.pixel_size)
    cols["x"], cols["y"] = xs, ys
    # step_tracker's columns (by position), the integer particle ids of
    # transform(int) and groupby(...).transform(len) -- a particle's rows
    # are all kept or all dropped, so its count is its duration
    cols.update(x_step=xst, y_step=yst, steplength=ln, particle=ids, duration=count[keep])
    full = pd.DataFrame(cols, index=df.index[keep])
    maxlag = int(cols["duration"].max()) if len(ids) else 0
    t, p, m = imsd(ids, cols["frame"], xs, ys, params.pixel_size, float(params.tracking_time), max_lagtime=maxlag)
    return full, pd.DataFrame({"time": t, "particle": p, "msd": m})
