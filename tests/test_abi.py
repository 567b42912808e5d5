"""CPU checks of the C-ABI library: it loads, exports every symbol that
include/gt.h declares, and its host-only logic (defaults, column list,
rejected options) matches the reference's.  No device compute is called."""
import ctypes
import os
import re
import subprocess

import pytest

from tracking_optimizations_b200 import _native, build as gtbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    inc = os.path.join(ROOT, "include")
    src = "".join(open(os.path.join(inc, h)).read() for h in sorted(os.listdir(inc)) if h.endswith(".h"))
    return sorted(set(re.findall(r"GT_API\s+[\w\s\*]*?\b(gt_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    gtbuild.build()
    return _native.load()


def test_header_declares_entry_points():
    names = declared()
    for n in ["gt_batch", "gt_batch_device", "gt_link", "gt_ctx_create", "gt_ctx_destroy", "gt_last_error",
              "gt_table_free", "gt_column_names", "gt_version", "gt_last_stats", "gt_ctx_set_option"]:
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    for n in declared():
        assert hasattr(lib, n), n
    assert sorted(s[0] for s in _native.SIGNATURES) == declared()


def test_version(lib):
    assert b"sm_100a" in lib.gt_version()


def test_no_device_is_an_error_not_a_crash(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    h = ctypes.c_void_p()
    assert lib.gt_ctx_create(0, ctypes.byref(h)) == _native.GT_ERR_CUDA


def cols(**kw):
    from tracking_optimizations_b200 import column_names
    return [c[0] for c in column_names(**kw)]


def test_column_names_follow_reference(lib):
    assert cols(diameter=9) == ["frame", "mass", "y", "x"]
    assert cols(diameter=9, search_range=5.0) == ["frame", "mass", "y", "x", "particle"]
    assert cols(diameter=9, search_range=5.0, cpu_processed=True, sig_radius=3.0, bg_radius=8.0,
                characterize=True) == [
        "frame", "mass", "y", "x", "particle", "Rg", "ecc", "signal", "raw_mass", "raw_bg_median",
        "raw_mass_corrected", "Rg_gpu", "raw_mass_gpu", "signal_gpu", "ecc_gpu"]


def test_column_names_match_oracle(lib):
    from oracle import oracle
    for kw in [dict(), dict(search_range=3.0), dict(cpu_processed=True), dict(sig_radius=2.0),
               dict(sig_radius=2.0, bg_radius=5.0, characterize=True, search_range=2.0)]:
        from tracking_optimizations_b200 import column_names
        assert column_names(7, **kw) == oracle.columns(oracle.resolve(7, **kw))


@pytest.mark.parametrize("name", ["maxsize", "threshold", "invert", "percentile", "topn", "preprocess"])
def test_unimplemented_options_are_rejected(lib, name):
    from tracking_optimizations_b200 import column_names
    with pytest.raises(NotImplementedError, match=name):
        column_names(9, **{name: 1})


def test_bg_without_sig_is_rejected(lib):
    from tracking_optimizations_b200 import column_names
    with pytest.raises(ValueError):
        column_names(9, bg_radius=5.0)


def test_struct_layouts_match_header(tmp_path):
    # compile a probe against include/gt.h and compare with the ctypes mirror
    src = tmp_path / "probe.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "gt.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gt_params), sizeof(gt_table), sizeof(gt_stats),
         offsetof(gt_params, gap_radius), offsetof(gt_table, names), offsetof(gt_stats, ms_total),
         sizeof(gt_movie), offsetof(gt_movie, params), offsetof(gt_movie, out), offsetof(gt_stats, batch_fallbacks),
         offsetof(gt_stats, ms_msd));
  return 0;
}
""")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_native.GtParams), ctypes.sizeof(_native.GtTable), ctypes.sizeof(_native.GtStats),
            _native.GtParams.gap_radius.offset, _native.GtTable.names.offset, _native.GtStats.ms_total.offset,
            ctypes.sizeof(_native.GtMovie), _native.GtMovie.params.offset, _native.GtMovie.out.offset,
            _native.GtStats.batch_fallbacks.offset, _native.GtStats.ms_msd.offset]
    assert got == want


def test_python_surface_mirrors_reference():
    import inspect
    import tracking_optimizations_b200 as gt
    sig = list(inspect.signature(gt.batch).parameters)
    assert sig == ["video", "diameter", "minmass", "maxsize", "separation", "noise_size", "smoothing_size",
                   "threshold", "invert", "percentile", "topn", "preprocess", "max_iterations", "characterize",
                   "filter_close", "search_range", "memory", "cpu_processed", "sig_radius", "bg_radius",
                   "gap_radius"]
    assert list(inspect.signature(gt.link_rust).parameters)[:3] == ["pyarr", "search_range", "memory"]
