#!/usr/bin/env python
"""Benchmark of gpu_tracking's locate-and-link hot path on B200.

Workload: one movie of 1000 frames of 512x512 uint16 (seeded synthetic
Gaussian spots: Poisson background 100 + read noise 5, 500 spots/frame,
sigma 1.2, amplitude U(150, 1500), Brownian 1.5 px, 2 % blinking) with
diameter 7, separation 8, noise_size 1, smoothing_size 7, minmass 300,
search_range 5, memory 2, cpu_processed=True.  A step = locate + link of the
whole movie.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload locate-link|adjoint|batched|file|postprocess|dense-link]

The other workloads print one line each: the adjoint of bandpass + refine
at fixed peaks (256 x 512x512 f32), 64 uneven movies in one graph launch
against per-movie calls, the movie from a multi-page TIFF file, and the
lab pipeline's post-processing (stub filter, step lengths, per-particle
MSD) of the movie's linked table.

N > 1 runs under torchrun: every rank processes its own movie (weak scaling,
no collective on the data path); the time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "locate+link frames/s at 512²×1000 u16"
LOCATE_KERNELS = {0: "locate_tiles_kernel", 1: "locate_fast_kernel", 2: "locate_fast_kernel (TMA staging)"}


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


def max_over_ranks(x, world, device):
    """The largest x over all ranks (every rank gets it); x itself at N=1."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, ms_max):
    """Whole-job units/s: every rank processed units_per_rank, the job took
    the slowest rank's time (replicas, weak scaling)."""
    return world * units_per_rank / (ms_max / 1e3)


def locate_traffic(frames):
    """DRAM bytes (read + write) of one locate launch over `frames` frames:
    the per-frame figure of the committed ncu capture of the same kernel on
    300 frames of this workload (profiles/locate_fast_kernel_300x512.md),
    scaled by the frame count (traffic is per frame)."""
    try:
        with open(os.path.join(ROOT, "profiles", "locate_fast_kernel_300x512.md")) as f:
            for line in f:
                if line.startswith("dram_bytes_per_frame:"):
                    return int(line.split(":")[1]) * frames
    except OSError:
        pass
    return None


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only) by a
    background thread every ~2 ms, kept for the samples taken inside the
    timed region (between __enter__ and __exit__)."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self.handle = None
        self.thread = None
        self.stop = None
        self.t0 = self.t1 = None

    def _open(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            self.handle = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        self.reasons_fn = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

    def _run(self):
        while not self.stop.is_set():
            try:
                mhz = self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM)
                rs = self.reasons_fn(self.handle)
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        import threading

        try:
            self._open()
        except Exception:
            self.handle = None
            return self
        self.stop = threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        deadline = time.perf_counter() + 2.0
        while not self.samples and time.perf_counter() < deadline:
            time.sleep(0.001)
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *a):
        self.t1 = time.perf_counter()
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=2)
        try:
            if self.handle is not None:
                self.nvml.nvmlShutdown()
        except Exception:
            pass

    def summary(self):
        if self.handle is None or self.t0 is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        inside = [x for x in self.samples if self.t0 <= x[0] <= self.t1]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = sorted({n for _, _, rs in inside for n, bit in self.REASONS if rs & bit})
        return {"sm_mhz": float(np.median([m for _, m, _ in inside])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(inside), "source": "NVML every ~2 ms in the timed region"}


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


def run_adjoint(args, rank, world, local):
    """--workload adjoint: one step = the fixed-peak forward plus its adjoint
    (gt_adjoint_forward + gt_adjoint_backward) over 256 frames of 512 x 512
    f32 with the locate workload's spot model; peaks from one locate before
    timing.  Algorithmic bytes per frame: the frame re-read (H*W*4) plus the
    gradient write (H*W*4)."""
    import torch

    from tracking_optimizations_b200 import _native, adjoint, synth

    torch.cuda.set_device(local)
    spec, params = workload()
    rspec = synth.scaled(spec, frames=args.frames or 256, seed=spec.seed + 100 + rank)
    movie = synth.make_movie(rspec).astype(np.float32)
    T, H, W = movie.shape
    dev = f"cuda:{local}"
    frames = torch.from_numpy(movie).to(dev)
    aparams = {k: v for k, v in params.items() if k not in ("search_range", "memory", "cpu_processed")}
    d = aparams.pop("diameter")
    rows, walk, _ = adjoint.locate_with_walk(frames, d, **aparams)
    n = walk.shape[0]
    lib = _native.load()
    ctx = _native.context(local)
    gp = _native.make_params(d, **aparams)
    yxm = torch.empty((n, 3), dtype=torch.float32, device=dev)
    gup = torch.randn((n, 3), device=dev, generator=torch.Generator(device=dev).manual_seed(0))
    gI = torch.empty_like(frames)
    gpar = torch.empty(2, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st_f, st_b = [], []

    def step():
        _native.check(lib.gt_adjoint_forward(ctx, P(frames), T, H, W, ctypes.byref(gp), P(walk), n, P(yxm), sp),
                      ctx)
        st_f.append(_native.last_stats(local))
        _native.check(lib.gt_adjoint_backward(ctx, P(frames), T, H, W, ctypes.byref(gp), P(walk), n, P(gup),
                                              P(gI), P(gpar), sp), ctx)
        st_b.append(_native.last_stats(local))

    for _ in range(max(3, args.warmup)):
        step()
    assert torch.equal(yxm, rows[:, [2, 3, 1]]), "fixed-peak forward differs from the located rows"
    st_f.clear()
    st_b.clear()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    # end to end: pinned host frames in, host gradient out, through the
    # autograd Function
    pinned = torch.from_numpy(movie).pin_memory()
    host_grad = torch.empty((T, H, W), dtype=torch.float32).pin_memory()

    def e2e_step():
        fr = pinned.to(dev, non_blocking=True).requires_grad_(True)
        out = adjoint.refine(fr, walk, d, **aparams)
        out.backward(gup)
        host_grad.copy_(fr.grad, non_blocking=True)
        torch.cuda.synchronize()

    e2e_step()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if rank != 0:
        return
    med = lambda xs, k: float(np.median([x[k] for x in xs]))  # noqa: E731
    dense_ms = med(st_b, "ms_adjoint_dense")
    alg = T * H * W * 8
    peak, kind = peaks()
    achieved = alg / (ms / 1e3) / 1e9
    line = {
        "metric": "adjoint frames/s (fixed-peak forward + backward, 256 x 512x512 f32)",
        "value": T / (ms / 1e3), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"adjoint at fixed peaks, {T} frames x {H}x{W} float32, {n} particles, "
                               "locate spot model; gt_adjoint_forward + gt_adjoint_backward per step",
                   "frames": T, "height": H, "width": W, "particles": n, "params": dict(aparams, diameter=d),
                   "l2": f"inputs larger than L2 ({movie.nbytes >> 20} MB frames + gradient per step)"},
        "roofline": {"bound": "hbm", "kernel": "whole step (frame re-read + gradient write)",
                     "achieved": achieved, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "algorithmic_bytes": alg},
        "stages_ms": {"forward_particles": med(st_f, "ms_adjoint_particles"),
                      "backward_particles": med(st_b, "ms_adjoint_particles"),
                      "backward_dense": dense_ms,
                      "dense_achieved_gbs": T * H * W * 12 / (dense_ms / 1e3) / 1e9},
        "gpu_launches": int(sum(x["launches"] for x in st_f + st_b)) // max(1, len(st_f)) * args.steps,
        "e2e": {"value": T / (e2e_ms / 1e3), "unit": "frames/s", "h2d_bytes_per_step": int(movie.nbytes),
                "d2h_bytes_per_step": int(movie.nbytes), "timing": "CUDA events around H2D + autograd + D2H"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_batched(args, rank, world, local):
    """--workload batched: 64 uneven movies (synth.batch_workload, rendered
    on the device), located and linked by one gt_batch_many_device call per
    step (a replayed CUDA graph), against the plain path: one
    gt_batch_device call per movie.  value = aggregate frames/s of the
    batched call; the plain path's figure and the ratio are reported
    beside it."""
    import torch

    from tracking_optimizations_b200 import _native, batched, synth

    torch.cuda.set_device(local)
    specs = synth.batch_workload()
    if args.frames:
        specs = specs[: args.frames]
    t0 = time.perf_counter()
    movies = [(synth.make_movie_device(s, f"cuda:{local}"), dict(s.params)) for s in specs]
    gen_s = time.perf_counter() - t0
    outs = batched.output_buffers(movies)
    lib = _native.load()
    ctx = _native.context(local)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    arr = (_native.GtMovie * len(movies))()
    plain_params = []
    for i, ((fr, params), out) in enumerate(zip(movies, outs)):
        kw = dict(params)
        d = kw.pop("diameter")
        m = arr[i]
        m.frames = fr.data_ptr()
        m.dtype = _native.GT_U16
        m.T, m.H, m.W = fr.shape
        m.params = _native.make_params(d, **kw)
        m.out = out.data_ptr()
        m.out_rows = out.shape[0]
        plain_params.append(m.params)
    nrows = ctypes.c_int64()
    plain_rows = [0] * len(movies)

    def plain_step():
        for i, ((fr, _), out) in enumerate(zip(movies, outs)):
            T, H, W = fr.shape
            _native.check(lib.gt_batch_device(ctx, ctypes.c_void_p(fr.data_ptr()), _native.GT_U16, T, H, W,
                                              ctypes.byref(plain_params[i]), ctypes.c_void_p(out.data_ptr()),
                                              out.shape[0], ctypes.byref(nrows), sp), ctx)
            plain_rows[i] = nrows.value

    stats = []

    def batch_step():
        _native.check(lib.gt_batch_many_device(ctx, arr, len(movies), sp), ctx)
        stats.append(_native.last_stats(local))

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    for _ in range(max(3, args.warmup)):
        plain_step()
    plain_ms = timed(plain_step, args.steps)
    for _ in range(max(3, args.warmup)):
        batch_step()
    assert [arr[i].nrows for i in range(len(movies))] == plain_rows, "batched row counts differ from plain"
    stats.clear()
    with Clocks(local) as clk:
        batch_ms = timed(batch_step, args.steps)
    frames = sum(s.frames for s in specs)
    px = sum(s.frames * s.height * s.width for s in specs)
    # the same comparison per class of frame size: which movies bound the ratio
    classes = {"small (<= 256x512)": lambda s: s.height * s.width <= 256 * 512,
               "medium (<= 1024x1024)": lambda s: 256 * 512 < s.height * s.width <= 1024 * 1024,
               "large (> 1024x1024)": lambda s: s.height * s.width > 1024 * 1024}
    per_class = {}
    for name, pred in classes.items():
        idx = [i for i, s in enumerate(specs) if pred(s)]
        if not idx:
            continue
        sub = (_native.GtMovie * len(idx))()
        for j, i in enumerate(idx):
            sub[j] = arr[i]

        def plain_c():
            for i in idx:
                fr, _ = movies[i]
                T, H, W = fr.shape
                _native.check(lib.gt_batch_device(ctx, ctypes.c_void_p(fr.data_ptr()), _native.GT_U16, T, H, W,
                                                  ctypes.byref(plain_params[i]),
                                                  ctypes.c_void_p(outs[i].data_ptr()), outs[i].shape[0],
                                                  ctypes.byref(nrows), sp), ctx)

        def batch_c():
            _native.check(lib.gt_batch_many_device(ctx, sub, len(idx), sp), ctx)

        for _ in range(2):
            plain_c()
            batch_c()
        pm, bm = timed(plain_c, max(1, args.steps // 2)), timed(batch_c, max(1, args.steps // 2))
        cf = sum(specs[i].frames for i in idx)
        per_class[name] = {"movies": len(idx), "frames": cf,
                           "gpx": sum(specs[i].frames * specs[i].height * specs[i].width for i in idx) / 1e9,
                           "plain_ms": pm, "batched_ms": bm, "batched_over_plain": pm / bm,
                           "plain_frames_per_s": cf / (pm / 1e3), "batched_frames_per_s": cf / (bm / 1e3)}
    if rank != 0:
        return
    peak, kind = peaks()
    alg = px * 2 + sum(plain_rows) * 80
    line = {
        "metric": "batched locate+link frames/s, 64 uneven movies (one graph launch per step)",
        "value": frames / (batch_ms / 1e3), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": batch_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16 in / f32 compute", "data": "synthetic (rendered on the device)",
        "config": {"workload": f"{len(specs)} movies, {frames} frames, {px / 1e9:.2f} Gpx u16 "
                               "(sides 128-2048, aspect 1-2, T 10-500, d 5-11, sep d+1, sr 3-8)",
                   "movies": len(specs), "frames": frames, "gpx": px / 1e9,
                   "l2": "inputs larger than L2", "generation_s": gen_s},
        "plain": {"value": frames / (plain_ms / 1e3), "ms_per_step": plain_ms,
                  "calls_per_step": len(specs)},
        "batched_over_plain": plain_ms / batch_ms,
        "per_class": per_class,
        "roofline": {"bound": "hbm", "kernel": "whole batched step", "achieved": alg / (batch_ms / 1e3) / 1e9,
                     "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": alg / (batch_ms / 1e3) / 1e9 / peak, "traffic": None, "algorithmic_bytes": alg},
        "batch_stats": {"graph": stats[-1]["batch_graph"], "launches": stats[-1]["launches"],
                        "link_passes": stats[-1]["link_iterations"], "fallbacks": stats[-1]["batch_fallbacks"],
                        "rows": sum(plain_rows)},
        "gpu_launches": int(sum(x["launches"] for x in stats)),
        "e2e": None,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_file(args, rank, world, local):
    """--workload file: the throughput movie written as an uncompressed
    multi-page u16 TIFF (untimed; it then sits in the page cache), located
    and linked from the file by gpu_tracking.batch_file_rust per step:
    decode on host threads into pinned memory, chunked upload overlapped
    with the locate kernels, linking, table back to the host."""
    import shutil
    import tempfile

    import torch
    from PIL import Image

    from tracking_optimizations_b200 import _native, gpu_tracking, synth

    torch.cuda.set_device(local)
    spec, params = workload()
    rspec = synth.scaled(spec, frames=args.frames or spec.frames, seed=spec.seed + rank)
    movie = synth.make_movie(rspec)
    T, H, W = movie.shape
    tmp = tempfile.mkdtemp(prefix="gt_bench_")
    try:
        path = os.path.join(tmp, "movie.tif")
        imgs = [Image.frombytes("I;16", (W, H), f.tobytes()) for f in movie]
        imgs[0].save(path, save_all=True, append_images=imgs[1:])
        del imgs
        for _ in range(max(3, args.warmup)):
            tab, _ = gpu_tracking.batch_file_rust(path, device=local, **params)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            tab, _ = gpu_tracking.batch_file_rust(path, device=local, **params)
        dt = (time.perf_counter() - t0) / args.steps
        stats = _native.last_stats(local)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    dt_max = max_over_ranks(dt, world, f"cuda:{local}")
    if rank != 0:
        return
    line = {
        "metric": "locate+link frames/s from a multi-page u16 TIFF file (512x512 x 1000)",
        "value": aggregate_rate(T, world, dt_max * 1e3), "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": dt_max * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16 in / f32 compute",
        "data": "synthetic, written to an uncompressed TIFF (page cache)",
        "config": dict(config_dict(spec, params, world), workload=f"file ingest: {T} frames x {H}x{W} u16 TIFF "
                       "-> batch_file_rust"),
        "stages_ms": {k: stats[k] for k in ["ms_locate", "ms_finalize", "ms_link", "ms_assemble", "ms_total"]},
        "rows": int(tab.shape[0]),
        "e2e": {"value": aggregate_rate(T, world, dt_max * 1e3), "unit": "frames/s",
                "h2d_bytes_per_step": int(movie.nbytes), "d2h_bytes_per_step": int(tab.nbytes),
                "timing": "host clock around batch_file_rust (file decode included)"},
    }
    print(json.dumps(line), flush=True)


def run_dense(args, rank, world, local):
    """--workload dense-link: the dense linking stress movie (200 frames of
    2048x2048 u16, 20,000 spots per frame, sigma 1.5, Brownian 2.5 px,
    diameter 9, search_range 7, memory 3), rendered on the device; one step
    = one gt_batch_device call (locate + link); the line reports the
    linker's share and its fixed-point passes."""
    import torch

    from tracking_optimizations_b200 import _native, synth

    torch.cuda.set_device(local)
    spec = synth.scaled(synth.DENSE_LINK, frames=args.frames or synth.DENSE_LINK.frames,
                        seed=synth.DENSE_LINK.seed + rank)
    params = dict(spec.params)
    fr = synth.make_movie_device(spec, f"cuda:{local}")
    T, H, W = fr.shape
    lib = _native.load()
    ctx = _native.context(local)
    gp = _native.make_params(**params)
    out = torch.empty((T * 30000, 5), dtype=torch.float32, device=f"cuda:{local}")
    nrows = ctypes.c_int64()
    stream = torch.cuda.current_stream()

    def step():
        _native.check(lib.gt_batch_device(ctx, ctypes.c_void_p(fr.data_ptr()), _native.GT_U16, T, H, W,
                                          ctypes.byref(gp), ctypes.c_void_p(out.data_ptr()), out.shape[0],
                                          ctypes.byref(nrows), ctypes.c_void_p(stream.cuda_stream)), ctx)

    for _ in range(max(1, args.warmup)):
        step()
    stats = []
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        stats.append(_native.last_stats(local))
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, f"cuda:{local}")
    if rank != 0:
        return
    med = lambda k: float(np.median([s_[k] for s_ in stats]))  # noqa: E731
    line = {
        "metric": "dense linking stress: locate+link frames/s at 2048^2 x 200 u16, 20000 spots/frame",
        "value": aggregate_rate(T, world, ms), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(1, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16 in / f32 compute", "data": "synthetic (device renderer)",
        "config": {"workload": f"dense linking stress: {T} frames x {H}x{W} u16, {spec.spots} spots/frame, "
                               "step 2.5 px", "params": params},
        "stages_ms": {k: med(k) for k in ["ms_locate", "ms_finalize", "ms_link", "ms_assemble", "ms_total"]},
        "link_iterations": stats[-1]["link_iterations"],
        "link_phase_ms": {k: float(np.median([s_["link_phase_ms"][i] for s_ in stats]))
                          for i, k in enumerate(["first", "roots", "memory", "relink"])},
        "rows": int(nrows.value),
    }
    print(json.dumps(line), flush=True)


def run_postprocess(args, rank, world, local):
    """--workload postprocess: the lab pipeline's steps after linking
    (all_cleaned_up/hatzakis_lab_tracking.py:216-232: filter_stubs,
    step_tracker, durations, per-particle MSD with max_lagtime = the longest
    duration) on the linked table of the throughput movie, through
    trajectories.postprocess (host DataFrame in, DataFrames out: uploads,
    kernels and downloads inside the timed region).  Lab defaults:
    duration_filter 20, pixel_size 0.18333, tracking_time 0.036.  Particles
    that the reference's memory dedupe gave two rows in one frame are dropped
    first (trackpy's msd refuses them)."""
    import pandas as pd
    import torch

    from tracking_optimizations_b200 import _native, batch_rust, synth, trajectories

    torch.cuda.set_device(local)
    spec, params = workload()
    rspec = synth.scaled(spec, frames=args.frames or spec.frames, seed=spec.seed + rank)
    tab, cols = batch_rust(synth.make_movie(rspec), device=local, **params)
    names = [c[0] for c in cols]
    df = pd.DataFrame({k: tab[:, names.index(k)] for k in ("frame", "y", "x", "particle")})
    ids = df["particle"].to_numpy().astype(np.int64)
    key = ids * 1000003 + df["frame"].to_numpy().astype(np.int64)
    _, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    branching = np.unique(ids[cnt[inv] > 1])
    df = df[~np.isin(ids, branching)].reset_index(drop=True)

    class Params:
        duration_filter = 20
        pixel_size = 0.18333
        tracking_time = 0.036

    for _ in range(max(3, args.warmup)):
        full, msd_df = trajectories.postprocess(df, Params)
    ms_msd = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        full, msd_df = trajectories.postprocess(df, Params)
        ms_msd.append(_native.last_stats(local)["ms_msd"])
    dt = (time.perf_counter() - t0) / args.steps
    dt_max = max_over_ranks(dt, world, f"cuda:{local}")
    if rank != 0:
        return
    n = len(df)
    line = {
        "metric": "linked-table rows/s through the lab post-processing (filter_stubs, step_tracker, imsd)",
        "value": aggregate_rate(n, world, dt_max * 1e3), "unit": "rows/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": dt_max * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 positions / f64 sums",
        "data": "synthetic: the linked table of the throughput movie",
        "config": dict(config_dict(spec, params, world), workload=f"post-processing of {n} linked rows "
                       f"({len(branching)} branching particles dropped): duration_filter 20, pixel_size 0.18333, "
                       "tracking_time 0.036"),
        "rows_kept": int(len(full)), "particles": int(full["particle"].nunique()),
        "msd_entries": int(len(msd_df)), "max_lagtime": int(full["duration"].max()),
        "msd_kernel_ms": float(np.median(ms_msd)),
        "e2e": {"value": aggregate_rate(n, world, dt_max * 1e3), "unit": "rows/s",
                "h2d_bytes_per_step": int(len(df) * (8 + 4 + 4) * 3),
                "d2h_bytes_per_step": int(len(df) * (1 + 4 * 2 + 8 * 4) + len(msd_df) * 12),
                "timing": "host clock around trajectories.postprocess"},
    }
    if not args.no_cpu_baseline:
        from oracle import traj_ref
        ids_k = full["particle"].to_numpy()
        pids = np.unique(ids_k)
        t0 = time.perf_counter()
        done = 0
        for i in range(0, len(pids), 64):
            sel = np.isin(ids_k, pids[i:i + 64])
            traj_ref.imsd(ids_k[sel], full["frame"].to_numpy()[sel], full["x"].to_numpy()[sel],
                          full["y"].to_numpy()[sel], Params.pixel_size, int(full["duration"].max()))
            done += int(sel.sum())
            if time.perf_counter() - t0 > 12.0:
                break
        cdt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": done / cdt, "unit": "rows/s", "cores": 1, "kind": "port",
                                "sample": f"MSD of the first {done} kept rows (numpy restatement, one core)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="locate-link", choices=["locate-link", "adjoint", "batched", "file",
                                                                     "postprocess", "dense-link"])
    ap.add_argument("--frames", type=int, default=None,
                    help="smaller movie of the same spot model (profiling captures only)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "adjoint":
        run_adjoint(args, rank, world, local)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "file":
        run_file(args, rank, world, local)
        return
    if args.workload == "dense-link":
        run_dense(args, rank, world, local)
        return
    if args.workload == "postprocess":
        run_postprocess(args, rank, world, local)
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
    ms_max = max_over_ranks(ms, world, f"cuda:{local}")
    value = aggregate_rate(T, world, ms_max)

    # end to end through the public API: pinned host frames in, table out
    e2e_value, tab, pinned = None, None, None
    if not args.no_e2e:
        pinned = torch.from_numpy(movie).pin_memory()
        host_in = pinned.numpy()
        # warm-up in the loop's own pattern (the previous table is alive
        # while the next call runs), so that the library's page-locked
        # table blocks are allocated before the timed calls
        for _ in range(max(2, min(args.warmup, 3))):
            tab, cols = batch_rust(host_in, **params)
        if world > 1:
            dist.barrier()
        e2e_steps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            tab, cols = batch_rust(host_in, **params)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        e2e_value = aggregate_rate(T, world, max_over_ranks(e2e_s, world, f"cuda:{local}") * 1e3)

    if rank == 0:
        loc_ms = float(np.median([s["ms_locate"] for s in stats]))
        cands = stats[-1]["candidates"]
        rows = stats[-1]["particles"]
        # algorithmic bytes of the path per step: frames read once (u16) +
        # the output table (rows x columns x 4 B) + the previous frame's
        # table re-read by the linker (y, x, id: 12 B per particle)
        loc_bytes = T * H * W * 2 + rows * ncols * 4 + rows * 12
        peak, kind = peaks()
        achieved = loc_bytes / (loc_ms / 1e3) / 1e9
        traffic = locate_traffic(T)
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16 in / f32 compute", "data": "synthetic",
            "config": config_dict(spec, params, world),
            "roofline": {"bound": "hbm", "kernel": LOCATE_KERNELS.get(stats[-1]["locate_kernel"], "?"),
                         "achieved": achieved, "peak": peak,
                         "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": loc_bytes, "launch_ms": loc_ms},
            "stages_ms": {k: float(np.median([s[k] for s in stats]))
                          for k in ["ms_locate", "ms_finalize", "ms_link", "ms_assemble", "ms_total"]},
            "link_iterations": stats[-1]["link_iterations"], "fallback_walks": stats[-1]["fallback_walks"],
            "link_phase_ms": {k: float(np.median([s["link_phase_ms"][i] for s in stats]))
                              for i, k in enumerate(["first", "roots", "memory", "relink"])},
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
