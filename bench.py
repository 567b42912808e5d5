#!/usr/bin/env python
"""Benchmark of gpu_tracking's locate-and-link hot path on B200.

Workload: one movie of 1000 frames of 512x512 uint16 (seeded synthetic
Gaussian spots: Poisson background 100 + read noise 5, 500 spots/frame,
sigma 1.2, amplitude U(150, 1500), Brownian 1.5 px, 2 % blinking) with
diameter 7, separation 8, noise_size 1, smoothing_size 7, minmass 300,
search_range 5, memory 2, cpu_processed=True.  A step = locate + link of the
whole movie.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun: every rank processes its own movie (weak scaling,
no collective on the data path); the time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "locate+link frames/s at 512²×1000 u16"


def workload():
    from tracking_optimizations_b200 import synth
    spec = synth.PLAIN_1000
    params = dict(spec.params, cpu_processed=True)
    return spec, params


def config_dict(spec, params, world):
    return {
        "workload": "plain locate+link, 1000 frames x 512x512 uint16 per GPU, synthetic Gaussian spots "
                    "(500/frame, sigma 1.2, Poisson 100 + read noise 5, 2% blinking)",
        "frames": spec.frames, "height": spec.height, "width": spec.width, "spots": spec.spots,
        "params": params, "parallelism": f"replicas x{world}",
        "l2": "inputs larger than L2 (524 MB movie per step)",
    }


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(movie, params, budget_s=12.0):
    """The oracle port (CPU restatement of the reference path) on host cores:
    locate multi-threaded over frames, linking sequential, on a bounded
    sample of the workload's frames."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    oracle.batch(movie[:4], nthreads=cores, **params)
    per = (time.perf_counter() - t0) / 4
    n = int(min(len(movie), max(8, budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    oracle.batch(movie[:n], nthreads=cores, **params)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"first {n} frames of the workload movie, locate on {cores} threads + sequential link"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path, restated (oracle port), on
    the host cores; rank 0 alone."""
    if rank != 0:
        return
    spec, params = workload()
    from tracking_optimizations_b200 import synth
    cores = os.cpu_count() or 1
    sample = 200
    movie = synth.make_movie(synth.scaled(spec, frames=sample))
    from oracle import oracle
    for _ in range(args.warmup):
        oracle.batch(movie[:8], nthreads=cores, **params)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.batch(movie[:sample], nthreads=cores, **params)
    dt = time.perf_counter() - t0
    value = sample * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(spec, params, 1),
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} frames of the workload per step (CPU restatement of the "
                                   "reference shaders + Rust post-process/linker; the reference binary "
                                   "cannot be built here)"},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--frames", type=int, default=None,
                    help="smaller movie of the same spot model (profiling captures only)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from tracking_optimizations_b200 import _native, batch_rust, synth

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    spec, params = workload()
    rspec = synth.scaled(spec, frames=args.frames, seed=spec.seed + rank)
    movie = synth.make_movie(rspec)
    T, H, W = movie.shape
    lib = _native.load()
    ctx = _native.context(local)
    gp = _native.make_params(**params)
    d_frames = torch.from_numpy(movie.view(np.int16)).to(f"cuda:{local}")
    ncols = 8
    cap_rows = T * 1024
    d_out = torch.empty((cap_rows, ncols), dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()
    nrows = ctypes.c_int64()

    def step():
        st = lib.gt_batch_device(ctx, ctypes.c_void_p(d_frames.data_ptr()), _native.GT_U16, T, H, W,
                                 ctypes.byref(gp), ctypes.c_void_p(d_out.data_ptr()), cap_rows,
                                 ctypes.byref(nrows), ctypes.c_void_p(stream.cuda_stream))
        _native.check(st, ctx)

    for _ in range(max(3, args.warmup)):
        step()
    assert nrows.value <= cap_rows
    stats = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
            stats.append(_native.last_stats(local))
        ev1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    t = torch.tensor([ms], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * T / (ms_max / 1e3)

    # end to end through the public API: pinned host frames in, table out
    e2e_value, tab, pinned = None, None, None
    if not args.no_e2e:
        pinned = torch.from_numpy(movie).pin_memory()
        host_in = pinned.numpy()
        batch_rust(host_in, **params)
        if world > 1:
            dist.barrier()
        e2e_steps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            tab, cols = batch_rust(host_in, **params)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        te = torch.tensor([e2e_s], device=f"cuda:{local}")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_value = world * T / float(te.item())

    if rank == 0:
        loc_ms = float(np.median([s["ms_locate"] for s in stats]))
        cands = stats[-1]["candidates"]
        rows = stats[-1]["particles"]
        # algorithmic bytes of one locate launch: frames read once (u16) +
        # candidate records written (80 B each)
        loc_bytes = T * H * W * 2 + cands * 80
        peak, kind = peaks()
        achieved = loc_bytes / (loc_ms / 1e3) / 1e9
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "locate_traffic.json")) as f:
                tr = json.load(f)
            traffic = tr["dram_bytes_per_frame"] * T
        except Exception:
            pass
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16 in / f32 compute", "data": "synthetic",
            "config": config_dict(spec, params, world),
            "roofline": {"bound": "hbm", "kernel": "locate_tiles_kernel", "achieved": achieved, "peak": peak,
                         "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": loc_bytes, "launch_ms": loc_ms},
            "stages_ms": {k: float(np.median([s[k] for s in stats]))
                          for k in ["ms_locate", "ms_finalize", "ms_link", "ms_assemble", "ms_total"]},
            "link_iterations": stats[-1]["link_iterations"], "fallback_walks": stats[-1]["fallback_walks"],
            "candidates_per_frame": cands / T, "particles_per_frame": rows / T,
            "gpu_launches": int(sum(s["launches"] for s in stats)),
            "e2e": None if e2e_value is None else {
                "value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": int(movie.nbytes),
                "d2h_bytes_per_step": int(tab.nbytes), "timing": "host clock around synchronous calls",
                "pinned_input": True},
            "clocks": clk.summary(),
        }
        if args.frames is not None:
            line["config"]["frames"] = T
            line["config"]["workload"] = f"profiling capture: {T} frames of the same spot model"
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(movie, params)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
