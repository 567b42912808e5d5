"""Generates tests/golden/steps_golden.npz by running the reference's own
``step_tracker`` (all_cleaned_up/hatzakis_lab_tracking.py:53-83) on a seeded
synthetic linked table.

The reference module imports trackpy, matplotlib and skimage at the top,
which are not installed, so only the function's own source is taken from the
module (by its syntax tree) and executed with numpy and pandas -- the code
that runs is the reference's, unchanged.  Run once where the reference tree
is present:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_steps_golden.py

The table: 60 frames, particle ids interleaved within each frame (so that
step_tracker's positional assignment of its groupby-ordered lists is visible),
trajectories starting and ending at different frames, pixel size 0.18333
(the lab default, hatzakis_lab_tracking.py:27).
"""
import ast
import os
import sys

import numpy as np
import pandas as pd

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_step_tracker(ref_root):
    path = os.path.join(ref_root, "all_cleaned_up", "hatzakis_lab_tracking.py")
    tree = ast.parse(open(path).read(), path)
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "step_tracker")
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np, "pd": pd}
    exec(compile(mod, path, "exec"), ns)
    return ns["step_tracker"]


def table(seed=3):
    rng = np.random.default_rng(seed)
    rows = []
    for pid in range(12):
        start = int(rng.integers(0, 30))
        length = int(rng.integers(2, 30))
        y, x = rng.uniform(20, 480, 2)
        for f in range(start, min(60, start + length)):
            if rng.random() < 0.1 and f != start:
                continue  # a gap (linking memory)
            y += rng.normal(0, 1.5)
            x += rng.normal(0, 1.5)
            rows.append((f, pid, np.float32(y), np.float32(x)))
    rows.sort(key=lambda r: (r[0], (r[1] * 7) % 12))  # frame order, ids interleaved
    f, p, y, x = (np.array(c) for c in zip(*rows))
    return f.astype(np.int64), p.astype(np.int64), y.astype(np.float32), x.astype(np.float32)


def main(ref_root):
    step_tracker = reference_step_tracker(ref_root)

    class Params:
        pixel_size = 0.18333

    f, p, y, x = table()
    df = pd.DataFrame({"frame": f, "y": y, "x": x, "particle": p.astype(np.float32)})
    out = step_tracker(df.copy(), Params)
    np.savez_compressed(os.path.join(HERE, "steps_golden.npz"), frame=f, particle=p, y=y, x=x,
                        pixel_size=np.float64(Params.pixel_size),
                        out_x=out["x"].to_numpy(np.float32), out_y=out["y"].to_numpy(np.float32),
                        x_step=out["x_step"].to_numpy(), y_step=out["y_step"].to_numpy(),
                        steplength=out["steplength"].to_numpy(),
                        out_dtypes=np.array([str(out[c].dtype) for c in ["x", "y", "x_step", "y_step",
                                                                          "steplength"]]))
    print("wrote", os.path.join(HERE, "steps_golden.npz"), len(f), "rows")


if __name__ == "__main__":
    ref_root = os.environ.get("REFERENCE_ROOT") or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not ref_root:
        sys.exit("set REFERENCE_ROOT (or pass the reference checkout as the first argument)")
    main(ref_root)
