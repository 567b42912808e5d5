"""ctypes binding of libgt.so (include/gt.h).

The CUDA library is the only implementation: if libgt.so is missing or no
CUDA device is present, every entry point raises instead of falling back.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgt.so")

GT_OK = 0
GT_ERR_ARG = 1
GT_ERR_CUDA = 2
GT_ERR_OOM = 3
GT_ERR_SUBNET_BUDGET = 4
GT_ERR_DEVICE_TIMEOUT = 5
GT_ERR_UNSUPPORTED = 6
GT_ERR_CAPACITY = 7
GT_U16 = 0
GT_F32 = 1
GT_MAX_COLS = 16

_FIELDS = [
    ("diameter", ctypes.c_uint32),
    ("has_minmass", ctypes.c_int32), ("minmass", ctypes.c_float),
    ("has_maxsize", ctypes.c_int32), ("maxsize", ctypes.c_float),
    ("has_separation", ctypes.c_int32), ("separation", ctypes.c_uint32),
    ("has_noise_size", ctypes.c_int32), ("noise_size", ctypes.c_float),
    ("has_smoothing_size", ctypes.c_int32), ("smoothing_size", ctypes.c_uint32),
    ("has_threshold", ctypes.c_int32), ("threshold", ctypes.c_float),
    ("has_invert", ctypes.c_int32), ("invert", ctypes.c_int32),
    ("has_percentile", ctypes.c_int32), ("percentile", ctypes.c_float),
    ("has_topn", ctypes.c_int32), ("topn", ctypes.c_uint32),
    ("has_preprocess", ctypes.c_int32), ("preprocess", ctypes.c_int32),
    ("has_max_iterations", ctypes.c_int32), ("max_iterations", ctypes.c_uint32),
    ("has_characterize", ctypes.c_int32), ("characterize", ctypes.c_int32),
    ("has_filter_close", ctypes.c_int32), ("filter_close", ctypes.c_int32),
    ("has_search_range", ctypes.c_int32), ("search_range", ctypes.c_float),
    ("has_memory", ctypes.c_int32), ("memory", ctypes.c_uint32),
    ("has_cpu_processed", ctypes.c_int32), ("cpu_processed", ctypes.c_int32),
    ("has_sig_radius", ctypes.c_int32), ("sig_radius", ctypes.c_float),
    ("has_bg_radius", ctypes.c_int32), ("bg_radius", ctypes.c_float),
    ("has_gap_radius", ctypes.c_int32), ("gap_radius", ctypes.c_float),
]


class GtParams(ctypes.Structure):
    _fields_ = _FIELDS


class GtTable(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.POINTER(ctypes.c_float)),
        ("nrows", ctypes.c_int64),
        ("ncols", ctypes.c_int32),
        ("names", (ctypes.c_char * 24) * GT_MAX_COLS),
        ("types", (ctypes.c_char * 8) * GT_MAX_COLS),
    ]


class GtStats(ctypes.Structure):
    _fields_ = [
        ("link_iterations", ctypes.c_int32),
        ("fallback_walks", ctypes.c_int32),
        ("candidates", ctypes.c_int64),
        ("particles", ctypes.c_int64),
        ("retries", ctypes.c_int32),
        ("launches", ctypes.c_int32),
        ("ms_locate", ctypes.c_float),
        ("ms_finalize", ctypes.c_float),
        ("ms_link", ctypes.c_float),
        ("ms_assemble", ctypes.c_float),
        ("ms_total", ctypes.c_float),
        ("locate_kernel", ctypes.c_int32),
        ("link_phase_ms", ctypes.c_float * 4),
        ("link_dirty", ctypes.c_int32 * 8),
        ("ms_adjoint_particles", ctypes.c_float),
        ("ms_adjoint_dense", ctypes.c_float),
        ("batch_graph", ctypes.c_int32),
        ("batch_fallbacks", ctypes.c_int32),
        ("ms_msd", ctypes.c_float),
    ]


class GtMovie(ctypes.Structure):
    _fields_ = [
        ("frames", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("H", ctypes.c_int32),
        ("W", ctypes.c_int32),
        ("params", GtParams),
        ("out", ctypes.c_void_p),
        ("out_rows", ctypes.c_int64),
        ("nrows", ctypes.c_int64),
    ]


# (name, restype, argtypes) of every symbol include/gt.h declares
SIGNATURES = [
    ("gt_version", ctypes.c_char_p, []),
    ("gt_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("gt_ctx_destroy", None, [ctypes.c_void_p]),
    ("gt_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("gt_column_names", ctypes.c_int, [ctypes.POINTER(GtParams), ctypes.c_char_p, ctypes.c_size_t]),
    ("gt_batch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.POINTER(GtParams), ctypes.POINTER(GtTable)]),
    ("gt_batch_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(GtParams), ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    ("gt_filter_stubs", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    ("gt_steps", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p]),
    ("gt_imsd", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int64, ctypes.c_double, ctypes.c_int64, ctypes.POINTER(GtTable)]),
    ("gt_link", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float,
                               ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p]),
    ("gt_table_free", None, [ctypes.POINTER(GtTable)]),
    ("gt_last_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GtStats)]),
    ("gt_ctx_set_option", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]),
    ("gt_locate_frame_static", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(GtParams), ctypes.c_void_p, ctypes.c_int64,
                                              ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    ("gt_batch_device_walk", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.POINTER(GtParams), ctypes.c_void_p,
                                            ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
                                            ctypes.c_void_p]),
    ("gt_batch_file", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32,
                                     ctypes.POINTER(GtParams), ctypes.POINTER(GtTable)]),
    ("gt_file_info", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    ("gt_file_read", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.c_int64]),
    ("gt_ets_channels", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int32)]),
    ("gt_batch_many_device", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GtMovie), ctypes.c_int,
                                            ctypes.c_void_p]),
    ("gt_synth_render", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("gt_adjoint_forward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.POINTER(GtParams), ctypes.c_void_p, ctypes.c_int64,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    ("gt_adjoint_backward", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(GtParams), ctypes.c_void_p, ctypes.c_int64,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("gt_adjoint_uncertainty", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.POINTER(GtParams), ctypes.c_void_p,
                                              ctypes.c_int64, ctypes.c_float, ctypes.c_float, ctypes.c_void_p,
                                              ctypes.c_void_p]),
]

_lib = None
_lock = threading.Lock()
_ctxs = {}


class GtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"libgt status {status}: {message}")
        self.status = status


def load():
    """Load libgt.so (raises OSError when it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"libgt.so not built at {LIB_PATH}; run "
                              "`python -m tracking_optimizations_b200.build`")
            lib = ctypes.CDLL(LIB_PATH)
            for name, res, args in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def context(device=0):
    """Per-device context, created on first use."""
    lib = load()
    with _lock:
        ctx = _ctxs.get(device)
        if ctx is None:
            h = ctypes.c_void_p()
            st = lib.gt_ctx_create(device, ctypes.byref(h))
            if st != GT_OK:
                raise GtError(st, f"cannot create a CUDA context on device {device}")
            ctx = h
            _ctxs[device] = ctx
        return ctx


def check(status, ctx):
    if status == GT_OK:
        return
    msg = load().gt_last_error(ctx).decode()
    if status == GT_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == GT_ERR_ARG:
        raise ValueError(msg)
    raise GtError(status, msg)


def set_option(key, value, device=0):
    """Tuning knob of the device's context (gt_ctx_set_option)."""
    ctx = context(device)
    check(load().gt_ctx_set_option(ctx, key.encode(), int(value)), ctx)


def last_stats(device=0):
    s = GtStats()
    load().gt_last_stats(context(device), ctypes.byref(s))
    out = {k: getattr(s, k) for k, _ in GtStats._fields_}
    out["link_phase_ms"] = list(out["link_phase_ms"])
    out["link_dirty"] = list(out["link_dirty"])
    return out


def make_params(diameter, **kw):
    """gt_params from gpu_tracking.batch keyword arguments (None = unset)."""
    p = GtParams()
    p.diameter = int(diameter)
    for key, val in kw.items():
        if val is None:
            continue
        if not hasattr(p, "has_" + key):
            raise TypeError(f"unexpected parameter {key!r}")
        setattr(p, "has_" + key, 1)
        setattr(p, key, type(getattr(p, key))(val) if not isinstance(val, bool) else int(val))
    return p
