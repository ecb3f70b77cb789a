"""The reference's scene-script surface on the host: ``from liar import *`` and ``liar.tools``
(src/liar/__init__.py:37-79, src/liar/tools/), the samplers' settings, and the reference's Cornell
box example scripts, run unchanged through this package with the render captured.

The capture test reads the example scripts from a reference checkout (LIAR_REFERENCE_DIR, or a
``reference`` folder beside this repository) and is skipped without one; its result must equal
the committed fixtures that tests/test_examples_gpu.py renders on the GPU."""
import io
import os
import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

import make_example_scenes  # noqa: E402
import scene_io  # noqa: E402

REF = Path(os.environ.get("LIAR_REFERENCE_DIR", HERE.parents[1] / "reference"))


def test_star_import_has_the_reference_names():
    ns = {}
    exec("from liar import *", ns)
    for name in ("cameras", "mediums", "output", "samplers", "scenery", "shaders", "spectra", "textures",
                 "tracers", "RenderEngine", "rgb", "sRGB", "CIEXYZ", "RgbSpace", "tolerance", "setTolerance"):
        assert name in ns, name
    import liar
    import liar.scenery
    assert liar.scenery.Parallelogram is ns["scenery"].Parallelogram
    assert ns["tolerance"]() == 1e-6


def test_spd_round_trip_and_builtin_metals():
    from liar.tools import spd
    a, b = spd.loads("# comment\n; other\n400 0.1 1\n500 0.2 2\n600 0.3 3\n")
    assert a.wavelengths == pytest.approx((400e-9, 500e-9, 600e-9)) and b.values == (1.0, 2.0, 3.0)
    buf = io.StringIO()
    spd.dump([a, b], buf)
    a2, b2 = spd.loads(buf.getvalue())
    assert a2.values == a.values and b2.wavelengths == pytest.approx(b.wavelengths)
    n, k = spd.load_builtin_refractive_index("Cu")
    assert len(n.values) == len(k.values) > 10
    with pytest.raises(ValueError):
        spd.load_builtin_refractive_index("Unobtainium")


def test_cornell_box_tool_scene():
    from liar.tools import cornell_box
    from liar_b200 import render as R
    flat = R.flatten(cornell_box.scene())
    # 5 walls and the light as 2 triangles each, 2 blocks of 12
    assert flat.triangles.shape == (36, 3)
    assert len(flat.lights) == 1 and flat.lights[0].emission_samples == 16
    cam = cornell_box.camera()
    assert cam.position == pytest.approx((2.78, 2.73, -8.0))


def test_scripting_options_and_targets(monkeypatch, tmp_path):
    from liar.tools import scripting
    from liar_b200 import output
    monkeypatch.setattr(sys, "argv", ["x.py", "--super-sampling", "9", "--global-size", "123"])
    o = scripting.renderOptions(width=800, super_sampling=4, global_size=200000, caustics_quality=1.0)
    assert (o.width, o.super_sampling, o.global_size, o.caustics_quality) == (800, 9, 123, 1.0)
    t = scripting.makeRenderTarget(3000, 200, str(tmp_path / "a.hdr"), "title")
    assert isinstance(t, output.Splitter)
    img, win = t.children
    assert isinstance(img, output.Image) and img.toneMapping == "Linear"
    assert win.resolution == (1500, 100) and win.title == "title"
    assert t.resolution == (3000, 200)


def test_samplers_follow_the_reference_settings(capsys):
    from liar_b200 import samplers
    s = samplers.Stratifier((64, 32), 8)
    assert s.samplesPerPixel == 9 and "using size 9 instead of 8" in capsys.readouterr().out
    assert s.mode == samplers.LIAR_SAMPLER_STRATIFIER
    s.jittered = False
    assert s.mode == samplers.LIAR_SAMPLER_NOT_JITTERED
    lh = samplers.LatinHypercube((8, 8), 8)
    assert lh.samplesPerPixel == 8 and lh.mode == samplers.LIAR_SAMPLER_LATIN_HYPERCUBE


def test_unsupported_settings_are_refused():
    from liar.tools import cornell_box
    from liar_b200 import RenderEngine, kernel, mediums, samplers, tracers
    e = RenderEngine()
    e.scene, e.camera, e.tracer = cornell_box.scene(), cornell_box.camera(), tracers.DirectLighting()
    e.sampler = samplers.Halton()
    with pytest.raises(NotImplementedError, match="progressive"):
        e.render()
    e.sampler = samplers.Stratifier((8, 8), 1)
    kernel.setTolerance(kernel.tolerance() * 1000)
    try:
        with pytest.raises(NotImplementedError, match="tolerance"):
            e.render()
    finally:
        kernel.setTolerance(1e-6)
    e.scene.children[-1].interior = mediums.Beer()
    from liar_b200 import render as R
    with pytest.raises(NotImplementedError, match="media"):
        R.flatten(e.scene)


@pytest.mark.parametrize("name", sorted(make_example_scenes.EXAMPLES))
def test_reference_example_runs_unchanged_and_matches_its_fixture(name):
    script = REF / "examples" / "cornell_box" / f"{name}.py"
    if not script.exists():
        pytest.skip("no reference checkout")
    flat, desc = make_example_scenes.capture(script, make_example_scenes.EXAMPLES[name])
    fflat, fdesc, extra = scene_io.load(HERE / "golden" / f"example_{name}.npz")
    assert scene_io.equal(flat, fflat)
    assert bytes(desc) == bytes(fdesc)
    assert list(extra["argv"]) == make_example_scenes.EXAMPLES[name]


def test_fixtures_load():
    for name in make_example_scenes.EXAMPLES:
        flat, desc, _ = scene_io.load(HERE / "golden" / f"example_{name}.npz")
        assert flat.triangles.shape == (36, 3) and desc.spp == 4
        assert np.isfinite(flat.pool).all()
