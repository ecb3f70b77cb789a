"""Named RGB spaces (the reference's liar.tools.rgb_spaces): white points as xy chromaticities and
RgbSpace(red, green, blue, white, gamma) for the common spaces, from their published primaries."""
from __future__ import annotations

from liar_b200.recovery import CIEXYZ, RgbSpace, sRGB  # noqa: F401

A = (0.44757, 0.40745)
B = (0.34842, 0.35161)
C = (0.31006, 0.31616)
D50 = (0.34567, 0.35850)
D55 = (0.33242, 0.34743)
D65 = (0.31271, 0.32902)
D75 = (0.29902, 0.31485)
E = (1.0 / 3, 1.0 / 3)

AdobeRGB = RgbSpace((0.64, 0.33), (0.21, 0.71), (0.15, 0.06), D65, 2.2)
AppleRGB = RgbSpace((0.625, 0.34), (0.28, 0.595), (0.155, 0.07), D65, 1.8)
BestRGB = RgbSpace((0.7347, 0.2653), (0.215, 0.775), (0.13, 0.035), D50, 2.2)
BetaRGB = RgbSpace((0.6888, 0.3112), (0.1986, 0.7551), (0.1265, 0.0352), D50, 2.2)
BruceRGB = RgbSpace((0.64, 0.33), (0.28, 0.65), (0.15, 0.06), D65, 2.2)
CIERGB = RgbSpace((0.735, 0.265), (0.274, 0.717), (0.167, 0.009), E, 2.2)
ColorMatchRGB = RgbSpace((0.63, 0.34), (0.295, 0.605), (0.15, 0.075), D50, 1.8)
HDTV_RGB = sRGB
NTSC_RGB = RgbSpace((0.67, 0.33), (0.21, 0.71), (0.14, 0.08), C, 2.2)
PAL_SECAM_RGB = RgbSpace((0.64, 0.33), (0.29, 0.6), (0.15, 0.06), D65, 2.2)
ProPhotoRGB = RgbSpace((0.7347, 0.2653), (0.1596, 0.8404), (0.0366, 0.0001), D50, 1.8)
SMPTE_C_RGB = RgbSpace((0.63, 0.34), (0.31, 0.595), (0.155, 0.07), D65, 2.2)
WideGamutRGB = RgbSpace((0.735, 0.265), (0.115, 0.826), (0.157, 0.018), D50, 2.2)
