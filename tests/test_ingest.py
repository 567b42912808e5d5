"""File ingest on the host (no GPU): multi-page TIFF and ETS decoding by
libgt (gt_file_info / gt_file_read / gt_ets_channels), checked against the
pixels that were written.

TIFF files come from PIL (compression none, LZW, Deflate, PackBits; 8- and
16-bit pages) and from a small writer below for the layouts PIL does not
produce (BigTIFF, big-endian, tiles, horizontal predictor).  ETS files are
written in the layout that gpu-tracking/src/decoderiter.rs:133-183 parses:
"SIS" header, "ETS" header with data type and dimensions, and the
used-chunk table (coordinate 2 = frame, coordinate 4 = channel).
"""
import struct
import zlib

import numpy as np
import pytest

from tracking_optimizations_b200 import gpu_tracking

PIL = pytest.importorskip("PIL.Image")


def movie(T=5, H=37, W=53, seed=0, hi=65535):
    return np.random.default_rng(seed).integers(0, hi + 1, (T, H, W)).astype(np.uint16)


def pil_tiff(path, frames, compression=None, mode="I;16"):
    imgs = [PIL.fromarray(f.astype(np.uint8)) if mode == "L" else PIL.frombytes("I;16", f.shape[::-1], f.tobytes())
            for f in frames]
    kw = {} if compression is None else {"compression": compression}
    imgs[0].save(path, save_all=True, append_images=imgs[1:], **kw)


@pytest.mark.parametrize("compression", [None, "tiff_lzw", "tiff_adobe_deflate", "packbits"])
def test_pil_tiff_16bit(tmp_path, compression):
    m = movie(seed=1)
    # smooth rows compress well: exercise long LZW tables too
    m[2] = np.cumsum(np.ones_like(m[2]), axis=1).astype(np.uint16) * 7
    p = tmp_path / "m.tif"
    pil_tiff(str(p), m, compression)
    np.testing.assert_array_equal(gpu_tracking.read_file(str(p)), m)


@pytest.mark.parametrize("compression", [None, "tiff_lzw", "packbits"])
def test_pil_tiff_8bit_widened(tmp_path, compression):
    m = movie(seed=2, hi=255)
    p = tmp_path / "m.tiff"
    pil_tiff(str(p), m, compression, mode="L")
    np.testing.assert_array_equal(gpu_tracking.read_file(str(p)), m)


def write_tiff(path, frames, big=False, endian="<", tile=None, predictor=1, compression=1, rows_per_strip=None):
    """Minimal TIFF writer: one IFD per frame, 16-bit samples."""
    T, H, W = frames.shape
    u16, u32, u64 = endian + "H", endian + "I", endian + "Q"
    out = bytearray(b"II" if endian == "<" else b"MM")
    if big:
        out += struct.pack(u16, 43) + struct.pack(u16, 8) + struct.pack(u16, 0) + struct.pack(u64, 0)
        first_ptr = 8
    else:
        out += struct.pack(u16, 42) + struct.pack(u32, 0)
        first_ptr = 4
    prev_ptr = first_ptr

    def encode(block):
        b = block.astype(endian + "u2")
        if predictor == 2:
            d = b.astype(np.int64)
            d[:, 1:] = d[:, 1:] - d[:, :-1]
            b = (d % 65536).astype(endian + "u2")
        raw = b.tobytes()
        return zlib.compress(raw) if compression == 8 else raw

    for f in frames:
        blocks = []
        if tile:
            tw, tl = tile
            for ty in range(0, H, tl):
                for tx in range(0, W, tw):
                    blk = np.zeros((tl, tw), np.uint16)
                    part = f[ty:ty + tl, tx:tx + tw]
                    blk[:part.shape[0], :part.shape[1]] = part
                    blocks.append(encode(blk))
        else:
            rps = rows_per_strip or H
            for r0 in range(0, H, rps):
                blocks.append(encode(f[r0:r0 + rps]))
        offs = []
        for bl in blocks:
            offs.append(len(out))
            out += bl
        if len(out) % 2:
            out += b"\0"
        arr_off = len(out)
        fmt = u64 if big else u32
        out += b"".join(struct.pack(fmt, o) for o in offs)
        cnt_off = len(out)
        out += b"".join(struct.pack(fmt, len(bl)) for bl in blocks)
        tags = [(256, 4, 1, W), (257, 4, 1, H), (258, 3, 1, 16), (259, 3, 1, compression), (277, 3, 1, 1),
                (317, 3, 1, predictor)]
        ltype = 16 if big else 4
        # a one-element array is stored in the entry itself
        ov = offs[0] if len(blocks) == 1 else arr_off
        cv = len(blocks[0]) if len(blocks) == 1 else cnt_off
        if tile:
            tags += [(322, 4, 1, tile[0]), (323, 4, 1, tile[1]), (324, ltype, len(blocks), ov),
                     (325, ltype, len(blocks), cv)]
        else:
            tags += [(273, ltype, len(blocks), ov), (278, 4, 1, rows_per_strip or H),
                     (279, ltype, len(blocks), cv)]
        tags.sort()
        ifd_off = len(out)
        struct.pack_into(fmt, out, prev_ptr, ifd_off)
        out += struct.pack(u64 if big else u16, len(tags))
        for tag, typ, count, val in tags:
            out += struct.pack(u16, tag) + struct.pack(u16, typ)
            if big:
                out += struct.pack(u64, count)
                if count == 1 and typ == 3:
                    out += struct.pack(u16, val) + b"\0" * 6
                elif count == 1 and typ == 4:
                    out += struct.pack(u32, val) + b"\0" * 4
                else:
                    out += struct.pack(u64, val)
            else:
                out += struct.pack(u32, count)
                if count == 1 and typ == 3:
                    out += struct.pack(u16, val) + b"\0" * 2
                else:
                    out += struct.pack(u32, val)
        prev_ptr = len(out)
        out += struct.pack(u64 if big else u32, 0)
    with open(path, "wb") as fh:
        fh.write(bytes(out))


@pytest.mark.parametrize("kw", [dict(), dict(big=True), dict(endian=">"), dict(tile=(16, 16)),
                                dict(tile=(32, 16), big=True), dict(predictor=2, compression=8),
                                dict(rows_per_strip=5, compression=8), dict(rows_per_strip=7, endian=">")])
def test_written_tiff_layouts(tmp_path, kw):
    m = movie(seed=3)
    p = tmp_path / "m.tif"
    write_tiff(str(p), m, **kw)
    np.testing.assert_array_equal(gpu_tracking.read_file(str(p)), m)


def test_tiff_wrong_bit_depth(tmp_path):
    p = tmp_path / "f.tif"
    PIL.fromarray(np.zeros((8, 8), np.float32), mode="F").save(str(p))
    with pytest.raises(NotImplementedError, match="Wrong bit depth"):
        gpu_tracking.read_file(str(p))


def write_ets(path, channels, dims, frames_of, ndim=6, repeat_last=None):
    """ETS per decoderiter.rs:133-183.  frames_of(channel) -> list of
    (frame index, u16 array) chunks; repeat_last = (channel, array) appends a
    chunk that repeats the last frame index of that channel."""
    chunks = []
    body = bytearray()
    data_off = 256
    for ch in channels:
        for idx, arr in frames_of(ch):
            chunks.append((ch, idx, data_off + len(body)))
            body += arr.astype("<u2").tobytes()
    if repeat_last is not None:
        ch, arr = repeat_last
        last = max(idx for c, idx, _ in chunks if c == ch)
        chunks.append((ch, last, data_off + len(body)))
        body += arr.astype("<u2").tobytes()
    add_off = 64
    used_off = data_off + len(body)
    hdr = bytearray(256)
    hdr[0:4] = b"SIS\0"
    struct.pack_into("<I", hdr, 12, ndim)
    struct.pack_into("<Q", hdr, 16, add_off)
    struct.pack_into("<Q", hdr, 32, used_off)
    struct.pack_into("<I", hdr, 40, len(chunks))
    hdr[add_off:add_off + 4] = b"ETS\0"
    struct.pack_into("<I", hdr, add_off + 8, 4)  # u16
    struct.pack_into("<II", hdr, add_off + 28, dims[0], dims[1])
    table = bytearray()
    for ch, idx, off in chunks:
        coord = [0] * ndim
        coord[2] = idx
        coord[4] = ch
        table += b"\0" * 4 + struct.pack("<%dI" % ndim, *coord) + struct.pack("<Q", off) + b"\0" * 8
    with open(path, "wb") as fh:
        fh.write(bytes(hdr) + bytes(body) + bytes(table))


def test_ets_channels_frames_and_parse(tmp_path):
    d0, d1 = 40, 24
    rng = np.random.default_rng(4)
    fr = {ch: [rng.integers(0, 65536, d0 * d1).astype(np.uint16) for _ in range(4)] for ch in (0, 3)}
    extra = rng.integers(0, 65536, d0 * d1).astype(np.uint16)

    def frames_of(ch):
        # channel 3 lacks frame 2; chunks out of order
        items = [(i, fr[ch][i]) for i in range(4) if not (ch == 3 and i == 2)]
        return items[::-1] if ch == 0 else items

    p = tmp_path / "m.ets"
    write_ets(str(p), [0, 3], (d0, d1), frames_of, repeat_last=(0, extra))
    got = gpu_tracking.read_file(str(p))  # channel 0: frames 0..3, then the repeated last index
    assert got.shape == (5, d0, d1)
    np.testing.assert_array_equal(got.reshape(5, -1), np.stack(fr[0] + [extra]))
    got3 = gpu_tracking.read_file(str(p), channel=3)
    np.testing.assert_array_equal(got3.reshape(3, -1), np.stack([fr[3][0], fr[3][1], fr[3][3]]))
    parsed = gpu_tracking.parse_ets(str(p))
    assert sorted(parsed) == [0, 3]
    assert parsed[0].shape == (5, d1, d0) and parsed[3].shape == (3, d1, d0)
    np.testing.assert_array_equal(parsed[0].reshape(5, -1), got.reshape(5, -1))
    with pytest.raises(ValueError, match="no channel 1"):
        gpu_tracking.read_file(str(p), channel=1)


def test_unknown_extension_and_missing_file(tmp_path):
    p = tmp_path / "m.png"
    p.write_bytes(b"x")
    with pytest.raises(ValueError, match="not supported"):
        gpu_tracking.read_file(str(p))
    with pytest.raises(ValueError, match="Could not open"):
        gpu_tracking.read_file(str(tmp_path / "absent.tif"))
