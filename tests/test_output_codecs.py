"""Image output (output/image.cpp, output/raster.cpp tone mapping) and the image codecs
(codecs.py): round trips through every format, the tone-mapping curves and auto exposure, and the
decoders on hand-built files (PNG row filters, Radiance run-length scanlines, OpenEXR ZIP blocks)."""
import math
import struct
import zlib

import numpy as np
import pytest

from liar_b200 import codecs, output
from liar_b200.recovery import RgbSpace, sRGB


def _film(rng, h=6, w=7, lo=0.05, hi=2.0):
    """XYZA of colours with positive linear sRGB, alpha in (0, 1]."""
    rgb = rng.uniform(lo, hi, size=(h, w, 3)).astype(np.float32)
    xyz = sRGB.linearSpace().toXYZlinear(rgb)
    a = rng.uniform(0.2, 1.0, size=(h, w, 1)).astype(np.float32)
    return np.concatenate([xyz, a], axis=-1), rgb


def _save(tmp_path, name, xyza, **settings):
    img = output.Image(str(tmp_path / name), (xyza.shape[1], xyza.shape[0]))
    img.exposureStops = 0.0
    for k, v in settings.items():
        setattr(img, k, v)
    img.write(xyza, np.zeros_like(xyza[..., :3]))
    return img


@pytest.mark.parametrize("ext,rtol", [(".pfm", 1e-5), (".exr", 2e-3), (".hdr", 1.2e-2)])
def test_linear_formats_round_trip(tmp_path, ext, rtol):
    xyza, rgb = _film(np.random.default_rng(1))
    _save(tmp_path, "x" + ext, xyza)
    back, space = codecs.read(tmp_path / ("x" + ext))
    assert space.gamma == 1.0
    lin = space.toRGBlinear(back[..., :3])
    if ext == ".hdr":
        # RGBE keeps 8 bits below the largest channel's exponent
        assert (np.abs(lin - rgb) <= rgb.max(axis=-1, keepdims=True) / 128 + 1e-6).all()
    else:
        np.testing.assert_allclose(lin, rgb, rtol=rtol, atol=1e-6)
    if ext == ".exr":
        np.testing.assert_allclose(back[..., 3], xyza[..., 3], rtol=1e-3)


def test_png_is_gamma_encoded_and_truncated(tmp_path):
    xyza, rgb = _film(np.random.default_rng(2), lo=0.0, hi=1.0)
    _save(tmp_path, "x.png", xyza)
    back, space = codecs.read(tmp_path / "x.png")
    assert space == sRGB                     # no colour chunk: the default space
    enc = np.clip(255.0 * sRGB.toGamma(rgb).astype(np.float64), 0, 255).astype(np.uint8)
    got = np.round(255.0 * sRGB.toGamma(sRGB.toRGBlinear(back[..., :3]))).astype(np.int32)
    assert np.abs(got - enc).max() <= 1
    a8 = np.clip(255.0 * xyza[..., 3].astype(np.float64), 0, 255).astype(np.uint8)
    np.testing.assert_array_equal(np.round(back[..., 3] * 255).astype(np.uint8), a8)
    linear = RgbSpace(sRGB.red, sRGB.green, sRGB.blue, sRGB.white, 1.0)
    one = np.zeros((1, 1, 4), np.float32)
    one[0, 0, :3] = linear.toXYZlinear(np.array([0.999, 0.5, 2.0], np.float32))
    one[0, 0, 3] = 1.0
    _save(tmp_path, "y.png", one, rgbSpace=linear)
    raw = codecs._read_png((tmp_path / "y.png").read_bytes())[0]
    np.testing.assert_array_equal(np.round(raw[0, 0] * 255), [254, 127, 255, 255])


def test_npy_keeps_the_film(tmp_path):
    xyza, _ = _film(np.random.default_rng(3))
    _save(tmp_path, "x.npy", xyza)
    np.testing.assert_array_equal(np.load(tmp_path / "x.npy"), xyza)


def _one_pixel(y):
    xyza = np.zeros((1, 2, 4), np.float32)
    xyza[0, 0] = (0.9 * y, y, 1.1 * y, 1.0)
    xyza[0, 1] = (0.3, 0.25, 0.2, 1.0)
    return xyza


@pytest.mark.parametrize("mode", output.TONE_MAPPINGS)
def test_tone_mappings(mode):
    img = output.Image("unused.npy", (2, 1))
    img.toneMapping = mode
    img.exposureStops = 1.0
    img.xyza = _one_pixel(0.7)
    lin = sRGB.linearSpace()
    out = img.tonemap(lin)
    xyz = 2.0 * img.xyza[0, 0, :3].astype(np.float64)          # gain 2^1
    Y = xyz[1]
    Lw = 2.0 * 0.7                                              # brightest pixel, with the gain
    rgb = lin.toRGBlinear(xyz.astype(np.float32)).astype(np.float64)
    filmic = lambda x: (lambda z: (z * (6.2 * z + .5) / (z * (6.2 * z + 1.7) + .06)) ** 2.2)(max(0.0, x - 0.004))
    expect = {
        "Linear": rgb,
        "CompressY": rgb / (1 + Y),
        "CompressRGB": rgb / (1 + rgb),
        "Reinhard2002Y": rgb * (1 + Y / Lw ** 2) / (1 + Y),
        "Reinhard2002RGB": rgb * (1 + rgb / Lw ** 2) / (1 + rgb),
        "ExponentialY": rgb * (-math.expm1(-Y) / Y),
        "ExponentialRGB": -np.expm1(-rgb),
        "DuikerY": rgb * filmic(Y) / max(Y, 0.004),
        "DuikerRGB": np.array([filmic(c) for c in rgb]),
    }[mode]
    np.testing.assert_allclose(out[0, 0, :3], expect, rtol=2e-5, atol=1e-7)


def test_auto_exposure_in_thirds_of_a_stop():
    img = output.Image("unused.npy", (2, 1))
    assert img.autoExposure
    xyza = np.zeros((1, 2, 4), np.float32)
    xyza[..., 1] = [0.5, 0.5]
    img.xyza = xyza
    # log-average 0.5: gain 0.184 / 0.5, log2 = -1.44 stops -> -4/3
    assert img.exposureStops == pytest.approx(-4.0 / 3.0)
    img.toneMapping = "ExponentialY"
    assert img.exposureStops == pytest.approx(round(3 * math.log2(-math.log1p(-0.184) / 0.5)) / 3)
    img.exposureStops = 0.5
    assert not img.autoExposure and img.exposureStops == 0.5
    img.xyza = np.full((1, 1, 4), np.nan, np.float32)
    img.exposureStops = 0.0
    np.testing.assert_array_equal(img.tonemap(sRGB)[0, 0], [1, 0, 1, 1])      # NaN: pink


def _png_bytes(rows: np.ndarray, ctype: int, filters) -> bytes:
    """A PNG with the given row filters (forward filters of the PNG specification, section 9)."""
    h, stride = rows.shape
    bpp = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    out, prev = b"", np.zeros(stride, np.int32)
    for y in range(h):
        cur = rows[y].astype(np.int32)
        f = filters[y % len(filters)]
        left = np.concatenate([np.zeros(bpp, np.int32), cur[:-bpp]])
        upleft = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        if f == 0:
            d = cur
        elif f == 1:
            d = cur - left
        elif f == 2:
            d = cur - prev
        elif f == 3:
            d = cur - ((left + prev) >> 1)
        else:
            p = left + prev - upleft
            pa, pb, pc = abs(p - left), abs(p - prev), abs(p - upleft)
            d = cur - np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
        out += bytes([f]) + (d & 0xFF).astype(np.uint8).tobytes()
        prev = cur
    w = stride // bpp
    ch = codecs._png_chunk
    return (b"\x89PNG\r\n\x1a\n" + ch(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0))
            + ch(b"gAMA", struct.pack(">I", 100000)) + ch(b"cHRM", struct.pack(">8I", 31270, 32900, 64000, 33000,
                                                                            30000, 60000, 15000, 6000))
            + ch(b"IDAT", zlib.compress(out)) + ch(b"IEND", b""))


@pytest.mark.parametrize("ctype", [0, 2, 4, 6])
def test_png_decoder_undoes_every_row_filter(ctype):
    rng = np.random.default_rng(ctype)
    bpp = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    rows = rng.integers(0, 256, size=(10, 9 * bpp), dtype=np.uint8)
    rgba, space = codecs._read_png(_png_bytes(rows, ctype, [0, 1, 2, 3, 4]))
    px = rows.reshape(10, 9, bpp).astype(np.float32) / 255
    if ctype in (0, 4):
        np.testing.assert_allclose(rgba[..., 0], px[..., 0])
        np.testing.assert_allclose(rgba[..., 2], px[..., 0])
    else:
        np.testing.assert_allclose(rgba[..., :3], px[..., :3])
    if ctype in (4, 6):
        np.testing.assert_allclose(rgba[..., 3], px[..., -1])
    # cHRM with gAMA 1.0: the file's own primaries, linear
    assert space.gamma == pytest.approx(1.0) and space.red == pytest.approx((0.64, 0.33))


def test_hdr_run_length_scanlines():
    w = 9
    head = f"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X {w}\n".encode()
    line = bytes([2, 2, 0, w])
    line += bytes([128 + w, 130])                   # R: one run
    line += bytes([4, 10, 20, 30, 40, 128 + 5, 50])  # G: literals then a run
    line += bytes([128 + w, 0])                      # B: zeros
    line += bytes([128 + w, 129])                    # E: exponent 1
    flat = bytes([128, 64, 32, 130]) * w             # an old-style flat scanline
    px = codecs._read_hdr(head + line + flat)
    f = 2.0 ** (129 - 136)
    np.testing.assert_allclose(px[0, :, 0], (130 + 0.5) * f)
    np.testing.assert_allclose(px[0, :5, 1], (np.array([10, 20, 30, 40, 50]) + 0.5) * f)
    np.testing.assert_allclose(px[0, 4:, 1], 50.5 * f)
    np.testing.assert_allclose(px[1, 0, :3], (np.array([128, 64, 32]) + 0.5) * 2.0 ** (130 - 136))


def test_exr_zip_blocks(tmp_path):
    """A ZIP-compressed (16-line blocks) float RGB file built by the OpenEXR spec's encoder:
    channels interleaved per line, bytes split into even and odd halves, delta-predicted, deflated."""
    rng = np.random.default_rng(5)
    h, w = 20, 5
    planes = {c: (np.round(rng.uniform(-1, 4, size=(h, w)) * 4) / 4).astype(np.float32) for c in "BGR"}
    attr = codecs._exr_attr
    chlist = b"".join(c.encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for c in "BGR") + b"\0"
    header = (b"\x76\x2f\x31\x01" + struct.pack("<i", 2) + attr("channels", "chlist", chlist)
              + attr("compression", "compression", b"\x03")
              + attr("dataWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
              + attr("displayWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
              + attr("lineOrder", "lineOrder", b"\0") + b"\0")
    blocks = []
    for y0 in range(0, h, 16):
        raw = b"".join(planes[c][y].astype("<f4").tobytes() for y in range(y0, min(h, y0 + 16)) for c in "BGR")
        b = np.frombuffer(raw, np.uint8)
        t = np.concatenate([b[0::2], b[1::2]]).astype(np.int32)
        d = np.concatenate([t[:1], (t[1:] - t[:-1] + 128) & 0xFF]).astype(np.uint8)
        z = zlib.compress(d.tobytes())
        assert len(z) < len(raw)             # else the block is stored as it is
        blocks.append((y0, z))
    off = len(header) + 8 * len(blocks)
    table, body = b"", b""
    for y0, z in blocks:
        table += struct.pack("<Q", off + len(body))
        body += struct.pack("<ii", y0, len(z)) + z
    rgba, space = codecs._read_exr(header + table + body)
    for k, c in enumerate("RGB"):
        np.testing.assert_array_equal(rgba[..., k], planes[c])
    np.testing.assert_array_equal(rgba[..., 3], 1.0)
    assert space == sRGB


def test_unknown_extension_fails_loudly(tmp_path):
    xyza, _ = _film(np.random.default_rng(4))
    with pytest.raises(ValueError):
        _save(tmp_path, "x.bmp", xyza)


@pytest.mark.parametrize("fname", ["colors-srgb.png", "colors-adobergb.png"])
def test_png_decoder_meets_the_references_codec_test(fname):
    """The reference's own known answers (test/test_codecs.cpp, lodepng_srgb and lodepng_adobergb,
    extracted to tests/golden/codec_colors.json): the space each test image reports and the XYZ
    (illuminant E) at the centres of its 24 colour patches within the test's tolerance. The images
    are read from a reference checkout (LIAR_REFERENCE_DIR, or a `reference` folder beside this
    repository); without one the test is skipped."""
    import json
    import os
    from pathlib import Path
    here = Path(__file__).resolve().parent
    ref = Path(os.environ.get("LIAR_REFERENCE_DIR", here.parents[1] / "reference"))
    path = ref / "test" / fname
    if not path.exists():
        pytest.skip("no reference checkout")
    gold = json.loads((here / "golden" / "codec_colors.json").read_text())
    xyza, space = codecs.read(path)
    assert xyza.shape == (400, 600, 4)
    want = gold["files"][fname]
    for name in ("red", "green", "blue", "white"):
        assert np.allclose(getattr(space, name), want["chromaticities"][name], atol=gold["chromaticity_tolerance"])
    assert abs(space.gamma - want["gamma"]) < gold["gamma_tolerance"]
    for y in range(4):
        for x in range(6):
            px = xyza[100 * y + 50, 100 * x + 50]
            assert np.all(np.abs(px[:3] - np.asarray(gold["xyz"][y][x])) < gold["xyz_tolerance"]), (y, x, px)
            assert abs(px[3] - 1.0) < 1e-3
