"""Image files (the reference's image codecs: kernel/image_codec.cpp, codecs/lodepng.cpp,
codecs/openexr.cpp): readers that return XYZA pixels and writers of tone-mapped RGBA, restated
from the file formats' published specifications.

Each format has the reference's colour space rule:
  .png   8 or 16 bit; read in the file's space (an sRGB chunk: sRGB; cHRM [+ gAMA]: those
         primaries, gamma 100000 / gAMA or 2.2; else the default space); written as 8-bit RGBA in
         the raster's space, each channel truncated from clamp(255 x, 0, 255) (lodepng.cpp:229-261)
  .hdr   Radiance RGBE (flat or run-length scanlines), .pfm portable float map: the given space
         (default sRGB) made linear (ImageCodecLass(false), image_codec.cpp:160-230)
  .exr   OpenEXR scanline file, half RGBA (Imf::RgbaOutputFile, WRITE_RGBA) with the space's
         chromaticities, linear (openexr.cpp:60-130); read: uncompressed, ZIPS or ZIP blocks of
         half or float channels, in the file's chromaticities or sRGB's
Writers write uncompressed scanlines (.hdr flat RGBE, .exr NO_COMPRESSION): the same pixels as
the reference's run-length / ZIP output, in larger files.
"""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

from .recovery import RgbSpace, sRGB

_default_space = sRGB


def default_space() -> RgbSpace:
    """RgbSpace.defaultSpace() (rgb_space.cpp): sRGB unless set otherwise."""
    return _default_space


def set_default_space(space: RgbSpace) -> None:
    global _default_space
    _default_space = space


def writer_space(path, raster_space: RgbSpace | None) -> RgbSpace:
    """The colour space a writer for `path` converts into (ImageWriter::rgbSpace)."""
    ext = Path(path).suffix.lower()
    space = raster_space or default_space()
    if ext in (".hdr", ".pic", ".rgbe", ".pfm", ".exr"):
        return space.linearSpace()
    if ext == ".png":
        return space
    raise ValueError(f"No image codec registered for the extension '{ext}'")


# ---- writing (rgba: (H, W, 4) float32, row 0 at the top)


def write(path, rgba: np.ndarray, space: RgbSpace) -> None:
    ext = Path(path).suffix.lower()
    rgba = np.asarray(rgba, dtype=np.float32)
    if ext == ".png":
        _write_png(path, rgba)
    elif ext in (".hdr", ".pic", ".rgbe"):
        _write_hdr(path, rgba)
    elif ext == ".pfm":
        _write_pfm(path, rgba)
    elif ext == ".exr":
        _write_exr(path, rgba, space)
    else:
        raise ValueError(f"No image codec registered for the extension '{ext}'")


def _png_chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def _write_png(path, rgba):
    h, w = rgba.shape[:2]
    q = np.clip(255.0 * rgba.astype(np.float64), 0, 255).astype(np.uint8)   # truncation, as static_cast
    raw = b"".join(b"\x00" + q[i].tobytes() for i in range(h))
    data = (b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
            + _png_chunk(b"IDAT", zlib.compress(raw, 6)) + _png_chunk(b"IEND", b""))
    Path(path).write_bytes(data)


def _rgbe(rgb: np.ndarray) -> np.ndarray:
    """Ward's RGBE: the largest channel's exponent shared by all three (Graphics Gems II, 1991)."""
    rgb = np.maximum(rgb.astype(np.float64), 0.0)
    v = rgb.max(axis=-1)
    m, e = np.frexp(v)
    out = np.zeros(rgb.shape[:-1] + (4,), dtype=np.uint8)
    ok = v >= 1e-32
    scale = np.where(ok, m * 256.0 / np.where(ok, v, 1.0), 0.0)
    out[..., :3] = np.where(ok[..., None], np.floor(rgb * scale[..., None]), 0).astype(np.uint8)
    out[..., 3] = np.where(ok, e + 128, 0).astype(np.uint8)
    return out


def _write_hdr(path, rgba):
    h, w = rgba.shape[:2]
    head = f"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y {h} +X {w}\n".encode()
    Path(path).write_bytes(head + _rgbe(rgba[..., :3]).tobytes())


def _write_pfm(path, rgba):
    h, w = rgba.shape[:2]
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(rgba[::-1, :, :3], dtype="<f4").tobytes())


def _exr_attr(name: str, kind: str, data: bytes) -> bytes:
    return name.encode() + b"\0" + kind.encode() + b"\0" + struct.pack("<i", len(data)) + data


def _write_exr(path, rgba, space: RgbSpace):
    h, w = rgba.shape[:2]
    names = ["A", "B", "G", "R"]                      # channel list in alphabetical order
    chlist = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", 1, 0, 1, 1) for n in names) + b"\0"
    chroma = struct.pack("<8f", *space.red, *space.green, *space.blue, *space.white)
    header = (b"\x76\x2f\x31\x01" + struct.pack("<i", 2)
              + _exr_attr("channels", "chlist", chlist)
              + _exr_attr("chromaticities", "chromaticities", chroma)
              + _exr_attr("comments", "string", b"rendered by liar_b200")
              + _exr_attr("compression", "compression", b"\x00")
              + _exr_attr("dataWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
              + _exr_attr("displayWindow", "box2i", struct.pack("<4i", 0, 0, w - 1, h - 1))
              + _exr_attr("lineOrder", "lineOrder", b"\x00")
              + _exr_attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _exr_attr("screenWindowCenter", "v2f", struct.pack("<2f", 0.0, 0.0))
              + _exr_attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0")
    planes = rgba[..., [3, 2, 1, 0]].astype(np.float16)       # A, B, G, R
    line_bytes = 4 * 2 * w
    first = len(header) + 8 * h
    offsets = first + np.arange(h, dtype=np.uint64) * np.uint64(8 + line_bytes)
    body = bytearray()
    for y in range(h):
        body += struct.pack("<ii", y, line_bytes)
        body += np.ascontiguousarray(planes[y].T).astype("<f2").tobytes()
    Path(path).write_bytes(header + offsets.astype("<u8").tobytes() + bytes(body))


# ---- reading: (XYZA pixels (H, W, 4) float32, row 0 at the top; the file's RgbSpace)


def read(path, space: RgbSpace | None = None) -> tuple[np.ndarray, RgbSpace]:
    """ImageReader(path, rgbSpace): the pixels as XYZA and the space they were read in."""
    p = Path(path)
    ext = p.suffix.lower()
    if ext == ".png":
        rgba, file_space = _read_png(p.read_bytes())
        sp = space or file_space
    elif ext in (".hdr", ".pic", ".rgbe"):
        rgba = _read_hdr(p.read_bytes())
        sp = (space or default_space()).linearSpace()
    elif ext == ".pfm":
        rgba = _read_pfm(p.read_bytes())
        sp = (space or default_space()).linearSpace()
    elif ext == ".exr":
        rgba, file_space = _read_exr(p.read_bytes())
        sp = (space or file_space).linearSpace()
    else:
        raise ValueError(f"No image codec registered for the extension '{ext}'")
    xyz = sp.toXYZarray(rgba[..., :3])
    return np.concatenate([xyz, rgba[..., 3:4]], axis=-1).astype(np.float32), sp


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def _read_png(data: bytes):
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, info = 8, b"", {}
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if tag == b"IHDR":
            info["w"], info["h"], info["depth"], info["ctype"], _, _, info["interlace"] = struct.unpack(">IIBBBBB", body)
        elif tag == b"PLTE":
            info["plte"] = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif tag == b"tRNS":
            info["trns"] = body
        elif tag == b"IDAT":
            idat += body
        elif tag == b"sRGB":
            info["srgb"] = True
        elif tag == b"gAMA":
            info["gama"] = struct.unpack(">I", body)[0]
        elif tag == b"cHRM":
            info["chrm"] = struct.unpack(">8I", body)
        elif tag == b"IEND":
            break
    w, h, depth, ctype = info["w"], info["h"], info["depth"], info["ctype"]
    if info["interlace"]:
        raise NotImplementedError("interlaced PNG files are not supported")
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    if depth not in (8, 16) and ctype != 3:
        raise NotImplementedError(f"PNG bit depth {depth} is not supported")
    if ctype == 3 and depth != 8:
        raise NotImplementedError("palette PNG files need 8 bits per index")
    bpp = max(1, channels * depth // 8)
    stride = w * channels * depth // 8
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, stride + 1)
    out = np.zeros((h, stride), np.int32)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        if f == 0:
            cur = line
        elif f == 2:
            cur = (line + prev) & 0xFF
        else:
            cur = np.zeros(stride, np.int32)
            for x in range(stride):       # Sub, Average and Paeth depend on the bytes just decoded
                a = cur[x - bpp] if x >= bpp else 0
                c = prev[x - bpp] if x >= bpp else 0
                if f == 1:
                    pred = a
                elif f == 3:
                    pred = (a + prev[x]) >> 1
                else:
                    pred = int(_paeth(np.int32(a), np.int32(prev[x]), np.int32(c)))
                cur[x] = (line[x] + pred) & 0xFF
        out[y] = cur
        prev = cur
    if depth == 16:
        vals = (out[:, 0::2] << 8 | out[:, 1::2]).astype(np.float32) / 65535.0
    else:
        vals = out.astype(np.float32) / 255.0
    vals = vals.reshape(h, w, channels)
    if ctype == 3:
        idx = out.reshape(h, w)
        rgb = info["plte"][idx].astype(np.float32) / 255.0
        alpha = np.ones((h, w, 1), np.float32)
        if "trns" in info:
            t = np.ones(256, np.float32)
            tr = np.frombuffer(info["trns"], np.uint8)
            t[:len(tr)] = tr / 255.0
            alpha = t[idx][..., None]
        rgba = np.concatenate([rgb, alpha], axis=-1)
    elif channels in (1, 2):
        g = vals[..., :1]
        a = vals[..., 1:2] if channels == 2 else np.ones_like(g)
        rgba = np.concatenate([g, g, g, a], axis=-1)
    else:
        rgba = vals if channels == 4 else np.concatenate([vals, np.ones((h, w, 1), np.float32)], axis=-1)
    if info.get("srgb"):
        space = sRGB
    elif "chrm" in info:
        c = [v / 100000.0 for v in info["chrm"]]
        gamma = 100000.0 / info["gama"] if "gama" in info else 2.2
        space = RgbSpace((c[2], c[3]), (c[4], c[5]), (c[6], c[7]), (c[0], c[1]), gamma)
    else:
        space = default_space()
    return rgba.astype(np.float32), space


def _read_hdr(data: bytes) -> np.ndarray:
    pos = data.index(b"\n\n") + 2
    end = data.index(b"\n", pos)
    dims = data[pos:end].split()
    pos = end + 1
    if dims[0] != b"-Y" or dims[2] != b"+X":
        raise NotImplementedError("only -Y H +X W Radiance files are supported")
    h, w = int(dims[1]), int(dims[3])
    buf = np.frombuffer(data, np.uint8)
    px = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        if 8 <= w < 0x8000 and buf[pos] == 2 and buf[pos + 1] == 2 and not (buf[pos + 2] & 0x80):
            pos += 4                      # new run-length scanline: four planes of runs
            for c in range(4):
                x = 0
                while x < w:
                    n = int(buf[pos])
                    pos += 1
                    if n > 128:
                        n -= 128
                        px[y, x:x + n, c] = buf[pos]
                        pos += 1
                    else:
                        px[y, x:x + n, c] = buf[pos:pos + n]
                        pos += n
                    x += n
        else:
            px[y] = buf[pos:pos + 4 * w].reshape(w, 4)
            pos += 4 * w
    e = px[..., 3].astype(np.int32)
    f = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    rgb = (px[..., :3].astype(np.float64) + 0.5) * f[..., None]
    rgb = np.where(e[..., None] > 0, rgb, 0.0)
    return np.concatenate([rgb, np.ones((h, w, 1))], axis=-1).astype(np.float32)


def _read_pfm(data: bytes) -> np.ndarray:
    parts = data.split(b"\n", 3)
    kind = parts[0].strip()
    w, h = (int(v) for v in parts[1].split())
    scale = float(parts[2])
    ch = 3 if kind == b"PF" else 1
    a = np.frombuffer(parts[3][:4 * w * h * ch], dtype="<f4" if scale < 0 else ">f4").reshape(h, w, ch)[::-1]
    if ch == 1:
        a = np.repeat(a, 3, axis=-1)
    return np.concatenate([a, np.ones((h, w, 1), np.float32)], axis=-1).astype(np.float32)


def _read_exr(data: bytes):
    if data[:4] != b"\x76\x2f\x31\x01":
        raise ValueError("not an OpenEXR file")
    flags = struct.unpack("<i", data[4:8])[0]
    if flags & 0x200:
        raise NotImplementedError("tiled OpenEXR files are not supported")
    pos, attrs = 8, {}
    while data[pos] != 0:
        e1 = data.index(b"\0", pos)
        e2 = data.index(b"\0", e1 + 1)
        name, kind = data[pos:e1].decode(), data[e1 + 1:e2].decode()
        n = struct.unpack("<i", data[e2 + 1:e2 + 5])[0]
        attrs[name] = (kind, data[e2 + 5:e2 + 5 + n])
        pos = e2 + 5 + n
    pos += 1
    chans, cd = [], attrs["channels"][1]
    q = 0
    while cd[q] != 0:
        e = cd.index(b"\0", q)
        ptype = struct.unpack("<i", cd[e + 1:e + 5])[0]
        chans.append((cd[q:e].decode(), ptype))
        q = e + 17
    comp = attrs["compression"][1][0]
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    lines = {0: 1, 2: 1, 3: 16}.get(comp)
    if lines is None:
        raise NotImplementedError(f"OpenEXR compression {comp} is not supported")
    nblocks = (h + lines - 1) // lines
    offsets = np.frombuffer(data[pos:pos + 8 * nblocks], "<u8")
    size = {0: 4, 1: 2, 2: 4}
    planes = {c: np.zeros((h, w), np.float32) for c, _ in chans}
    for b in range(nblocks):
        o = int(offsets[b])
        y, n = struct.unpack("<ii", data[o:o + 8])
        block = data[o + 8:o + 8 + n]
        rows = min(lines, y1 + 1 - y)
        expect = rows * w * sum(size[t] for _, t in chans)
        if comp != 0 and n < expect:
            t = np.frombuffer(zlib.decompress(block), np.uint8).astype(np.int32)
            t = np.cumsum(np.concatenate([t[:1], t[1:] - 128])) & 0xFF    # the predictor undone
            half = (len(t) + 1) // 2
            inter = np.empty(len(t), np.uint8)
            inter[0::2], inter[1::2] = t[:half], t[half:]
            block = inter.tobytes()
        q = 0
        for r in range(rows):
            for c, t in chans:
                nb = size[t] * w
                dt = {0: "<u4", 1: "<f2", 2: "<f4"}[t]
                planes[c][y - y0 + r] = np.frombuffer(block[q:q + nb], dt).astype(np.float32)
                q += nb
    ones = np.ones((h, w), np.float32)
    rgba = np.stack([planes.get("R", planes.get("Y", ones)), planes.get("G", planes.get("Y", ones)),
                     planes.get("B", planes.get("Y", ones)), planes.get("A", ones)], axis=-1)
    space = sRGB
    if "chromaticities" in attrs:
        c = struct.unpack("<8f", attrs["chromaticities"][1])
        space = RgbSpace((c[0], c[1]), (c[2], c[3]), (c[4], c[5]), (c[6], c[7]), 1.0)
    return rgba, space
