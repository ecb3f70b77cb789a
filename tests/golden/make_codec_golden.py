"""Writes tests/golden/codec_colors.json from the reference's own codec test (test/test_codecs.cpp):
the CIE XYZ (illuminant E) values expected at the centres of the 4 x 6 colour patches of
test/colors-srgb.png and test/colors-adobergb.png, the tolerance the test allows, and the RGB
spaces (primaries, white, gamma) each file must report. Read from the test source as text.

Usage: python tests/golden/make_codec_golden.py REFERENCE_CHECKOUT
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref: Path) -> None:
    src = (ref / "test" / "test_codecs.cpp").read_text()
    table = src.split("const XYZ colors[4][6] =", 1)[1].split("};", 1)[0]
    rows = []
    for line in table.splitlines():
        vals = re.findall(r"XYZ\(([^)]*)\)", line)
        if vals:
            rows.append([[float(v.strip().rstrip("f")) for v in t.split(",")] for t in vals])
    assert len(rows) == 4 and all(len(r) == 6 for r in rows), rows
    tol = float(re.search(r"constexpr XYZ::TValue tol = ([0-9.e-]+)f;", src).group(1))
    spaces = {}
    for name, fname in (("lodepng_srgb", "colors-srgb.png"), ("lodepng_adobergb", "colors-adobergb.png")):
        body = src.split(f"TEST(Codecs, {name})", 1)[1].split("testImage", 1)[0]
        chroma = {k: [float(a), float(b)] for k, a, b in
                  re.findall(r"EXPECT_CHROMATICITY\(rgbSpace->(\w+)\(\),\s*([0-9.]+),\s*([0-9.]+)\)", body)}
        gamma = float(re.search(r"EXPECT_DOUBLE\(rgbSpace->gamma\(\), ([0-9.]+)\)", body).group(1))
        spaces[fname] = {"chromaticities": chroma, "gamma": gamma}
    out = {"patch_centres": "pixel (100 x + 50, 100 y + 50) of the 600 x 400 image", "xyz": rows,
           "xyz_tolerance": tol, "chromaticity_tolerance": 1e-3, "gamma_tolerance": 1e-3, "files": spaces}
    (HERE / "codec_colors.json").write_text(json.dumps(out, indent=1))
    print(HERE / "codec_colors.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} REFERENCE_CHECKOUT")
    main(Path(sys.argv[1]))
