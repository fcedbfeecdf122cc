"""The library's JPEG texture decoder (crt_image_decode, host only) on
images written here with Pillow (libjpeg): baseline with 4:4:4, 4:2:2 and
4:2:0 chroma, progressive (spectral selection and successive
approximation), greyscale, restart intervals, odd sizes. The decoded pixels
are compared with the reference's own decoder (stb_image as the reference
builds it, from oracle/_ref; the comparison is skipped where that build is
absent) and with Pillow's. The inverse DCT, chroma upsampling and colour
conversion are computed independently of both, so levels may differ by a
few units; the bounds are written in the test. Malformed files are refused."""
import ctypes as C
import os

import numpy as np
import pytest

from cudaraytracer_b200 import _lib, scenes

Image = pytest.importorskip("PIL.Image")


def decode(path):
    w, h = C.c_int32(), C.c_int32()
    st = _lib.lib().crt_image_decode(str(path).encode(), C.byref(w), C.byref(h), None)
    if st:
        raise ValueError(_lib.lib().crt_last_error().decode())
    out = np.empty((h.value, w.value, 4), np.uint8)
    assert _lib.lib().crt_image_decode(str(path).encode(), C.byref(w), C.byref(h), out.ctypes.data) == 0
    return out


def stb_decode(path):
    """The reference's decoder: stbi_load(..., 4) from its vendored
    stb_image, compiled into oracle/_ref/libcrtref.so."""
    import oracle

    if not oracle.ref_available():
        return None
    lib = C.CDLL(oracle.REF_SO)
    lib.stbi_load.restype = C.c_void_p
    lib.stbi_load.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
    lib.stbi_image_free.argtypes = [C.c_void_p]
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    p = lib.stbi_load(str(path).encode(), C.byref(w), C.byref(h), C.byref(c), 4)
    assert p, "stb_image refused the file"
    a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), (h.value, w.value, 4)).copy()
    lib.stbi_image_free(p)
    return a


def test_image(w=77, h=53, seed=3):
    rng = np.random.default_rng(seed)
    img = scenes.checker_texture(w, h, seed=seed)[..., :3].astype(np.int32)
    return np.clip(img + rng.integers(-20, 20, img.shape), 0, 255).astype(np.uint8)


CASES = {
    "baseline_444": dict(subsampling=0),
    "baseline_422": dict(subsampling=1),
    "baseline_420": dict(subsampling=2),
    "progressive_420": dict(subsampling=2, progressive=True),
    "progressive_444": dict(subsampling=0, progressive=True),
    "grey": dict(mode="L"),
    "restart_420": dict(subsampling=2, restart_marker_blocks=3),
    "progressive_restart": dict(subsampling=2, progressive=True, restart_marker_rows=1),
    "quality_30": dict(subsampling=2, quality=30),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_jpeg_matches_reference_decoder(tmp_path, name):
    kw = dict(CASES[name])
    mode = kw.pop("mode", "RGB")
    q = kw.pop("quality", 85)
    p = tmp_path / f"{name}.jpg"
    Image.fromarray(test_image()).convert(mode).save(p, quality=q, **kw)
    data = p.read_bytes()
    if "restart" in name:
        assert b"\xff\xdd" in data  # a restart interval is present
    if "progressive" in name:
        assert b"\xff\xc2" in data
    mine = decode(p)
    assert mine.shape == (53, 77, 4) and (mine[..., 3] == 255).all()
    if mode == "L":
        assert (mine[..., 0] == mine[..., 1]).all() and (mine[..., 0] == mine[..., 2]).all()
    pil = np.asarray(Image.open(p).convert("RGBA")).astype(np.int32)
    d_pil = np.abs(mine.astype(np.int32) - pil)
    assert d_pil.max() <= 4 and d_pil.mean() <= 0.25, (d_pil.max(), d_pil.mean())
    ref = stb_decode(p)
    if ref is not None:
        d_ref = np.abs(mine.astype(np.int32) - ref.astype(np.int32))
        if name == "baseline_422":
            # in the last column of an odd-width 4:2:2 image the reference's
            # decoder differs from libjpeg by up to ~10 levels; this decoder
            # follows libjpeg there (checked against Pillow above)
            d_ref = d_ref[:, :-1]
        assert d_ref.mean() <= 0.25, d_ref.mean()
        assert d_ref.max() <= 4, d_ref.max()


def test_jpeg_texture_through_scene_loader(tmp_path):
    """A textured scene whose textures are JPEG files loads them (the
    scene loader used to keep the basecolor for any non-PNG texture)."""
    spec = scenes.cornell_box(width=32, height=32, textured=True)
    path = spec.write(str(tmp_path), "cb", texture_format="jpg")
    import json

    doc = json.load(open(path))
    assert doc["textures"] and all(t["path"].endswith(".jpg") for t in doc["textures"])
    for t in doc["textures"]:
        img = decode(t["path"])
        src = spec.textures[t["name"]][..., :3].astype(np.int32)
        assert img.shape[:2] == src.shape[:2]
        pil = np.asarray(Image.open(t["path"]).convert("RGB")).astype(np.int32)
        assert np.abs(img[..., :3].astype(np.int32) - pil).max() <= 4
        assert np.abs(img[..., :3].astype(np.int32) - src).mean() < 4.0  # lossy at quality 95


@pytest.mark.parametrize("mutate", ["truncate", "no_sof", "arith", "cmyk"])
def test_bad_jpeg_refused(tmp_path, mutate):
    p = tmp_path / "a.jpg"
    Image.fromarray(test_image(16, 16)).save(p, quality=90)
    d = bytearray(p.read_bytes())
    if mutate == "truncate":
        d = d[: len(d) // 3]
    elif mutate == "no_sof":
        i = d.find(b"\xff\xc0")
        d[i + 1] = 0xFE  # turn the frame header into a comment
    elif mutate == "arith":
        i = d.find(b"\xff\xc0")
        d[i + 1] = 0xC9
    else:
        Image.fromarray(test_image(16, 16)).convert("CMYK").save(p, quality=90)
        d = bytearray(p.read_bytes())
    p.write_bytes(bytes(d))
    with pytest.raises(ValueError, match="JPEG"):
        decode(p)
