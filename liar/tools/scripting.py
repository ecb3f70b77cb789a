"""Script helpers (the reference's liar.tools.scripting, src/liar/tools/scripting.py).

renderOptions(**defaults) turns each keyword into a command-line option (``--super-sampling`` for
``super_sampling``; int, float or string by the default's type) and returns the parsed options, so
that a script's sizes can be set from the command line. makeRenderTarget(width, height, filename,
title, ...) builds the image file target and, where the output module has a Display, a display
window scaled to fit 1500 x 1000; with both it returns a Splitter of the two.
"""
from __future__ import annotations

import optparse

_MAX_DISPLAY_WIDTH, _MAX_DISPLAY_HEIGHT = 1500, 1000


def makeRenderTarget(width, height, filename=None, title=None, display=True, fStops=None, rgbSpace=None,
                     toneMapping=None):
    from liar_b200 import output
    from liar_b200.recovery import sRGB

    targets = []
    if filename:
        image = output.Image(filename, (width, height))
        if fStops is not None:
            image.exposureStops = fStops
            image.autoExposure = False
        image.toneMapping = toneMapping or output.Image.ToneMapping.Linear
        image.rgbSpace = rgbSpace or sRGB
        targets.append(image)
    if display and hasattr(output, "Display"):
        scale = min(float(_MAX_DISPLAY_WIDTH) / width, float(_MAX_DISPLAY_HEIGHT) / height)
        resolution = (int(scale * width), int(scale * height)) if scale < 1 else (width, height)
        win = output.Display(title or filename or "", resolution)
        win.rgbSpace = rgbSpace or sRGB
        if fStops is not None:
            win.exposureStops = fStops
            win.autoExposure = False
        win.toneMapping = toneMapping or output.Display.ToneMapping.Linear
        targets.append(win)
    if not targets:
        raise AssertionError("Failed to create any kind of render target")
    return targets[0] if len(targets) == 1 else output.Splitter(targets)


def renderOptions(**kwargs):
    parser = optparse.OptionParser()
    for switch, default in kwargs.items():
        kind = "int" if isinstance(default, int) else "float" if isinstance(default, float) else "string"
        parser.add_option("", "--" + switch.replace("_", "-"), action="store", type=kind, default=default,
                          help="[default=%default]")
    options, _ = parser.parse_args()
    return options
