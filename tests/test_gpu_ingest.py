"""batch_file_rust on the GPU: a movie read from a TIFF or ETS file gives
exactly the table batch_rust gives for the same frames in memory
(execute_gpu.rs:510-542 hands the decoded frames to the same pipeline)."""
import struct

import numpy as np
import pytest

from tracking_optimizations_b200 import batch_rust, gpu_tracking, synth

pytestmark = pytest.mark.gpu

PIL = pytest.importorskip("PIL.Image")
PARAMS = dict(diameter=7, separation=8, minmass=300.0, search_range=5.0, memory=2, cpu_processed=True)


def tiff(path, frames, compression=None):
    imgs = [PIL.frombytes("I;16", f.shape[::-1], f.tobytes()) for f in frames]
    kw = {} if compression is None else {"compression": compression}
    imgs[0].save(path, save_all=True, append_images=imgs[1:], **kw)


@pytest.mark.parametrize("compression", [None, "tiff_lzw"])
def test_tiff_file_equals_in_memory(tmp_path, gpu, compression):
    spec = synth.scaled(synth.PLAIN_1000, frames=40, height=192, width=256, seed=51)
    mv = synth.make_movie(spec)
    p = tmp_path / "movie.tif"
    tiff(str(p), mv, compression)
    got = gpu_tracking.batch_file_rust(str(p), **PARAMS)
    want = batch_rust(mv, **PARAMS)
    assert got[1] == want[1]
    assert got[0].shape[0] > 40 * 50
    np.testing.assert_array_equal(got[0], want[0])


def test_8bit_tiff_file(tmp_path, gpu):
    spec = synth.scaled(synth.PLAIN_1000, frames=6, height=128, width=128, seed=52)
    mv = np.clip(synth.make_movie(spec) // 4, 0, 255).astype(np.uint8)
    p = tmp_path / "movie8.tif"
    imgs = [PIL.fromarray(f) for f in mv]
    imgs[0].save(str(p), save_all=True, append_images=imgs[1:])
    params = dict(PARAMS, minmass=80.0)
    np.testing.assert_array_equal(gpu_tracking.batch_file_rust(str(p), **params)[0],
                                  batch_rust(mv.astype(np.uint16), **params)[0])


def test_ets_file_channel(tmp_path, gpu):
    # dims (d0, d1) = (160, 224): frames are dims[0] rows of dims[1] values
    d0, d1 = 160, 224
    spec = synth.scaled(synth.PLAIN_1000, frames=12, height=d0, width=d1, seed=53)
    mv = synth.make_movie(spec)
    ndim, data_off, add_off = 6, 256, 64
    body = b"".join(f.astype("<u2").tobytes() for f in mv)
    hdr = bytearray(256)
    hdr[0:4] = b"SIS\0"
    struct.pack_into("<IQ", hdr, 12, ndim, add_off)
    struct.pack_into("<QI", hdr, 32, data_off + len(body), len(mv))
    hdr[add_off:add_off + 4] = b"ETS\0"
    struct.pack_into("<I", hdr, add_off + 8, 4)
    struct.pack_into("<II", hdr, add_off + 28, d0, d1)
    table = b"".join(b"\0" * 4 + struct.pack("<6I", 0, 0, t, 0, 2, 0) + struct.pack("<Q", data_off + t * d0 * d1 * 2)
                     + b"\0" * 8 for t in range(len(mv)))
    p = tmp_path / "movie.ets"
    p.write_bytes(bytes(hdr) + body + table)
    got = gpu_tracking.batch_file_rust(str(p), channel=2, **PARAMS)
    np.testing.assert_array_equal(got[0], batch_rust(mv, **PARAMS)[0])
    with pytest.raises(ValueError, match="no channel 0"):
        gpu_tracking.batch_file_rust(str(p), **PARAMS)
