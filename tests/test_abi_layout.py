"""The ctypes mirrors of the C-ABI structs (render.py, photons.py, batch.py, guiding.py,
_native.py) have the header's layout: a C program compiled against include/liar_gpu.h prints every
struct's size and every field's offset, which must equal what ctypes computes."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from liar_b200 import _native, batch, guiding, photons, render

ROOT = Path(__file__).resolve().parent.parent

MIRRORS = {
    "liar_ray": _native.Ray, "liar_hit": _native.Hit, "liar_build_opts": _native.BuildOpts,
    "liar_trace_config": _native.TraceConfig, "liar_mesh_stats": _native.MeshStats,
    "liar_spectrum": render.CSpectrum, "liar_material": render.CMaterial, "liar_texture": render.CTexture,
    "liar_light": render.CLight, "liar_scene_desc": render.CSceneDesc, "liar_camera": render.CCamera,
    "liar_photon_mapper_desc": render.CPhotonMapperDesc, "liar_render_desc": render.CRenderDesc,
    "liar_batch_item": batch.BatchItem, "liar_batch_config": batch.BatchConfig,
    "liar_guide_config": guiding.GuideConfig,
    "liar_photon_desc": photons.PhotonDesc, "liar_photon_buffers": photons.PhotonBuffers,
    "liar_photon_counts": photons.PhotonCounts,
}
RENAMED = {"global_": "global"}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "liar_gpu.h"', "int main(void) {"]
    expected = []
    for cname, cls in MIRRORS.items():
        lines.append(f'    printf("{cname} %zu\\n", sizeof({cname}));')
        expected.append(f"{cname} {ctypes.sizeof(cls)}")
        for fname, *_ in cls._fields_:
            c_field = RENAMED.get(fname, fname)
            lines.append(f'    printf("{cname}.{c_field} %zu\\n", offsetof({cname}, {c_field}));')
            expected.append(f"{cname}.{c_field} {getattr(cls, fname).offset}")
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = [g for g in got if g]
    mismatched = [(e, g) for e, g in zip(expected, got) if e != g]
    assert not mismatched, f"ctypes (left) and the header (right) disagree: {mismatched[:8]}"
    assert len(got) == len(expected)
