"""CPU restatement of the trajectory post-processing after linking -- TEST
INFRASTRUCTURE ONLY (the checker for gt_filter_stubs / gt_steps / gt_imsd);
nothing in the product imports it.

The lab pipeline (all_cleaned_up/hatzakis_lab_tracking.py:216-232) runs,
after linking:

* ``trackpy.filter_stubs(tracks, threshold)`` (line 217).  trackpy is an
  external dependency that is not in the reference tree and whose version the
  reference does not pin; restated here from its published definition: keep
  the rows of the particles that occur in at least ``threshold`` rows, in
  table order.  Parity against trackpy itself is unpinned.
* ``step_tracker`` (lines 53-83), the reference's own code: x, y scaled by
  the pixel size in float32 (the float32 column times a Python float), then
  per particle (pandas groupby order: ascending id, rows of a particle in
  table order) the difference to the particle's previous row (0 for its
  first row) and ``np.sqrt(y**2 + x**2)`` -- in float64, because
  ``tolist()`` turns the float32 values into Python floats.  Pinned by the
  reference function itself (tests/golden/make_steps_golden.py runs it).
* ``mp_imsd`` (lines 199-214): ``trackpy.msd(traj, mpp, fps, max_lagtime)``
  per particle, concatenated, the 'msd' column unstacked, lag time =
  lag / fps, then stacked to (time, particle, msd) rows by ``tracker``
  (lines 230-232).  trackpy.msd restated from its published definition:
  positions ``traj[['x', 'y']] * mpp`` (float32) reindexed to every frame
  from the particle's first to its last (gaps NaN); for lag L in
  1 .. min(max_lagtime, span - 1), <x^2> = nanmean of the squared x
  differences over the pairs with both frames present, likewise <y^2>;
  msd = <x^2> + <y^2>; lags without a pair give NaN, which ``stack`` drops.
  Two rows of one particle in one frame are refused ("more than one
  trajectory per particle").  The means are formed here from float32
  squares summed left to right in float64, then rounded to float32 (trackpy
  sums in float32 pairwise; the difference is within float32 rounding).
"""
import numpy as np


def filter_stubs(ids, threshold):
    ids = np.asarray(ids, dtype=np.int64)
    _, inv, cnt = np.unique(ids, return_inverse=True, return_counts=True)
    return cnt[inv] >= threshold


def steps(ids, x, y, mpp):
    """(xs, ys, x_step, y_step, steplength, order): xs, ys in table order,
    the steps in groupby order, order = table row of each groupby entry."""
    ids = np.asarray(ids, dtype=np.int64)
    m = np.float32(mpp)
    xs = np.asarray(x, dtype=np.float32) * m
    ys = np.asarray(y, dtype=np.float32) * m
    order = np.argsort(ids, kind="stable")
    g = ids[order]
    same = np.zeros(len(g), bool)
    same[1:] = g[1:] == g[:-1]
    xo, yo = xs[order].astype(np.float64), ys[order].astype(np.float64)
    dx = np.zeros(len(g), np.float64)
    dy = np.zeros(len(g), np.float64)
    dx[1:] = xo[1:] - xo[:-1]
    dy[1:] = yo[1:] - yo[:-1]
    dx[~same] = 0
    dy[~same] = 0
    length = np.sqrt(dy * dy + dx * dx)
    return xs, ys, dx, dy, length, order


def imsd(ids, frames, x, y, mpp, max_lagtime):
    """(lag, particle, msd) rows ordered by lag then particle (NaN lags
    dropped), as float32 arrays."""
    ids = np.asarray(ids, dtype=np.int64)
    frames = np.asarray(frames, dtype=np.int64)
    m = np.float32(mpp)
    xs = np.asarray(x, dtype=np.float32) * m
    ys = np.asarray(y, dtype=np.float32) * m
    out = []
    for pid in np.unique(ids):
        sel = np.nonzero(ids == pid)[0]
        f = frames[sel]
        if len(np.unique(f)) != len(f):
            raise ValueError("more than one trajectory per particle")
        f0 = f.min()
        span = int(f.max() - f0 + 1)
        px = np.full(span, np.nan, np.float32)
        py = np.full(span, np.nan, np.float32)
        px[f - f0] = xs[sel]
        py[f - f0] = ys[sel]
        for lag in range(1, min(int(max_lagtime), span - 1) + 1):
            dx = px[lag:] - px[:-lag]
            dy = py[lag:] - py[:-lag]
            ok = ~np.isnan(dx)
            cnt = int(ok.sum())
            if cnt == 0:
                continue
            sx = np.cumsum((dx[ok] * dx[ok]).astype(np.float64))[-1]
            sy = np.cumsum((dy[ok] * dy[ok]).astype(np.float64))[-1]
            v = np.float32(sx / cnt) + np.float32(sy / cnt)
            out.append((lag, pid, v))
    if not out:
        return np.zeros((0, 3), np.float32)
    out.sort(key=lambda r: (r[0], r[1]))
    return np.array(out, dtype=np.float32)
