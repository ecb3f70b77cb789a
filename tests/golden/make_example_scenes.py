"""Runs the reference's Cornell box example scripts, unchanged, through this repository's ``liar``
package and stores what each asks the engine to render as a fixture (tests/golden/example_*.npz).

Usage: python tests/golden/make_example_scenes.py REFERENCE_CHECKOUT

Each script (examples/cornell_box/<name>.py of the reference) runs with runpy as ``__main__``, with
small image sizes given through its own command-line options (scripting.renderOptions). The GPU
render is replaced by a capture of the flattened scene and the render description, so the scripts
need no GPU here. tests/test_examples.py re-runs the capture when the reference is present and
checks it against the fixtures; tests/test_examples_gpu.py renders the fixtures on the GPU and
compares them with the oracle.
"""
from __future__ import annotations

import contextlib
import os
import runpy
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
for p in (str(ROOT), str(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

# example script -> its own command-line options for a small render
EXAMPLES = {
    "direct_lighting": ["--width", "48", "--height", "48", "--super-sampling", "4"],
    "photon_mapper_classic": ["--size", "40", "--super-sampling", "4", "--global-size", "20000",
                              "--gather-rays", "16"],
}


class _CaptureContext:
    def set_cancel_flag(self, flag):
        pass


class _CaptureScene:
    """Stands in for liar_b200.render.GpuScene: records the scene and the description."""

    log: list = []

    def __init__(self, ctx, flat):
        self.ctx = _CaptureContext()
        self.flat = flat

    def render(self, desc):
        _CaptureScene.log.append((self.flat, desc))
        return np.zeros((desc.height, desc.width, 8), np.float32)


def capture(script: Path, argv: list[str]):
    """(FlatScene, CRenderDesc) of the one engine.render() of the script."""
    from liar_b200 import kernel, render as R

    _CaptureScene.log = []
    saved = (R.GpuScene, sys.argv, os.getcwd(), kernel.default_context)
    R.GpuScene = _CaptureScene
    kernel.default_context = lambda: None
    try:
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)  # the script's image file lands here
            sys.argv = [str(script), *argv]
            with contextlib.redirect_stdout(sys.stderr):
                runpy.run_path(str(script), run_name="__main__")
    finally:
        R.GpuScene, sys.argv, kernel.default_context = saved[0], saved[1], saved[3]
        os.chdir(saved[2])
    if len(_CaptureScene.log) != 1:
        raise RuntimeError(f"{script.name}: expected one render, got {len(_CaptureScene.log)}")
    return _CaptureScene.log[0]


def main(ref: Path) -> None:
    import scene_io

    for name, argv in EXAMPLES.items():
        script = ref / "examples" / "cornell_box" / f"{name}.py"
        flat, desc = capture(script, argv)
        out = HERE / f"example_{name}.npz"
        scene_io.save(out, flat, desc, argv=np.array(argv))
        print(out, flat.triangles.shape[0], "triangles", desc.width, "x", desc.height, desc.spp, "spp")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} REFERENCE_CHECKOUT")
    main(Path(sys.argv[1]))
