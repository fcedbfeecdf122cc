"""The library's texture decoder (crt_image_decode, host only) against images
written here: every PNG colour type (grey, RGB, palette, grey+alpha, RGBA),
bit depths 1-16, all five row filters, stored and compressed deflate
blocks, palette transparency, binary PPM; malformed files are refused."""
import ctypes as C
import struct
import zlib

import numpy as np
import pytest

from cudaraytracer_b200 import _lib, scenes


def decode(path):
    w, h = C.c_int32(), C.c_int32()
    st = _lib.lib().crt_image_decode(str(path).encode(), C.byref(w), C.byref(h), None)
    if st:
        raise ValueError(_lib.lib().crt_last_error().decode())
    out = np.empty((h.value, w.value, 4), np.uint8)
    assert _lib.lib().crt_image_decode(str(path).encode(), C.byref(w), C.byref(h), out.ctypes.data) == 0
    return out


def chunk(tag, body):
    return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)


def png_bytes(w, h, depth, ctype, rows, extra=b"", level=6):
    """rows: filtered scanlines (filter byte + data) joined."""
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0)) + extra +
            chunk(b"IDAT", zlib.compress(rows, level)) + chunk(b"IEND", b""))


def pack_rows(samples, depth):
    """(h, n) integer samples -> unfiltered scanlines (filter 0)."""
    out = b""
    for row in samples:
        if depth == 16:
            data = b"".join(struct.pack(">H", int(v)) for v in row)
        elif depth == 8:
            data = bytes(int(v) for v in row)
        else:
            per = 8 // depth
            data = bytearray()
            for i in range(0, len(row), per):
                byte = 0
                for k in range(per):
                    v = int(row[i + k]) if i + k < len(row) else 0
                    byte |= v << ((per - 1 - k) * depth)
                data.append(byte)
            data = bytes(data)
        out += b"\x00" + data
    return out


def test_rgba_all_filters_roundtrip(tmp_path):
    img = scenes.checker_texture(53, 31, seed=5)
    img[..., 3] = np.arange(53, dtype=np.uint8)[None, :] * 4
    p = tmp_path / "a.png"
    scenes.write_png(p, img)  # filters cycle None, Sub, Up, Average, Paeth
    np.testing.assert_array_equal(decode(p), img)


def test_stored_deflate_blocks(tmp_path):
    rng = np.random.default_rng(1)
    px = rng.integers(0, 256, size=(9, 7 * 3))
    p = tmp_path / "s.png"
    p.write_bytes(png_bytes(7, 9, 8, 2, pack_rows(px, 8), level=0))  # level 0: stored blocks
    got = decode(p)
    np.testing.assert_array_equal(got[..., :3], px.reshape(9, 7, 3))
    assert (got[..., 3] == 255).all()


@pytest.mark.parametrize("depth", [1, 2, 4, 8, 16])
def test_grey_depths(tmp_path, depth):
    rng = np.random.default_rng(depth)
    px = rng.integers(0, 1 << depth, size=(5, 11))
    p = tmp_path / f"g{depth}.png"
    p.write_bytes(png_bytes(11, 5, depth, 0, pack_rows(px, depth)))
    got = decode(p)
    scale = {1: 255, 2: 85, 4: 17, 8: 1}
    want = (px >> 8) if depth == 16 else px * scale[depth]
    for k in range(3):
        np.testing.assert_array_equal(got[..., k], want)
    assert (got[..., 3] == 255).all()


def test_rgb16_and_grey_alpha(tmp_path):
    rng = np.random.default_rng(3)
    px = rng.integers(0, 65536, size=(4, 6 * 3))
    p = tmp_path / "c16.png"
    p.write_bytes(png_bytes(6, 4, 16, 2, pack_rows(px, 16)))
    np.testing.assert_array_equal(decode(p)[..., :3], (px >> 8).reshape(4, 6, 3))
    ga = rng.integers(0, 256, size=(3, 5 * 2))
    p = tmp_path / "ga.png"
    p.write_bytes(png_bytes(5, 3, 8, 4, pack_rows(ga, 8)))
    got = decode(p)
    g = ga.reshape(3, 5, 2)
    np.testing.assert_array_equal(got[..., 0], g[..., 0])
    np.testing.assert_array_equal(got[..., 3], g[..., 1])


@pytest.mark.parametrize("depth", [2, 8])
def test_palette_with_transparency(tmp_path, depth):
    rng = np.random.default_rng(7)
    n = 1 << min(depth, 4)
    pal = rng.integers(0, 256, size=(n, 3)).astype(np.uint8)
    trns = bytes(rng.integers(0, 256, size=n // 2).astype(np.uint8))
    idx = rng.integers(0, n, size=(6, 10))
    p = tmp_path / f"p{depth}.png"
    p.write_bytes(png_bytes(10, 6, depth, 3, pack_rows(idx, depth),
                            extra=chunk(b"PLTE", pal.tobytes()) + chunk(b"tRNS", trns)))
    got = decode(p)
    np.testing.assert_array_equal(got[..., :3], pal[idx])
    alpha = np.array(list(trns) + [255] * (n - len(trns)), np.uint8)
    np.testing.assert_array_equal(got[..., 3], alpha[idx])


def test_ppm(tmp_path):
    rng = np.random.default_rng(9)
    px = rng.integers(0, 256, size=(4, 5, 3)).astype(np.uint8)
    p = tmp_path / "a.ppm"
    p.write_bytes(b"P6\n# comment\n5 4\n255\n" + px.tobytes())
    got = decode(p)
    np.testing.assert_array_equal(got[..., :3], px)


@pytest.mark.parametrize("payload", [b"not an image at all", b"\x89PNG\r\n\x1a\n\x00\x00\x00\x0dIHDR"])
def test_bad_files_are_refused(tmp_path, payload):
    p = tmp_path / "bad.png"
    p.write_bytes(payload)
    with pytest.raises(ValueError):
        decode(p)
    img = scenes.checker_texture(8, 8)
    good = tmp_path / "g.png"
    scenes.write_png(good, img)
    data = good.read_bytes()
    cut = tmp_path / "cut.png"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(ValueError):
        decode(cut)
