"""GPU photon tracing (PhotonMapper::fillPhotonMaps) against the CPU restatement, and the
trace -> map -> gather pipeline. Both sides draw the same per-photon random numbers, so the stored
photons coincide except where the two machines' libm rounding sends a path another way."""
import numpy as np
import pytest

import oracle
from liar_b200 import photons, render as R, scenes_render
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu


def _both(global_target, rt_direct, wave=8192, max_emitted=400_000, quality=1.0):
    scene, _ = scenes_render.photon_scene()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    d = photons.photon_desc(global_target, max_emitted=max_emitted, wave=wave, ray_traced_direct=rt_direct, seed=4,
                            caustics_quality=quality)
    g, gc = photons.trace_photons(gs, d, capacity=400_000)
    c, cc = oracle.photon_trace(oracle.RenderScene(flat), d, 400_000)
    g = {k: v.cpu().numpy() for k, v in g.items()}
    return g, gc, c, cc


@pytest.mark.parametrize("rt_direct,quality", [(True, 1.0), (False, 1.0), (False, 4.0), (True, 0.0)])
def test_photon_trace_matches_oracle(rt_direct, quality):
    """quality: causticsQuality, whose storage probabilities (1 / 4 global, 1 caustic at 4; no
    caustic photons at 0) decide by Russian roulette which diffuse hits are stored."""
    g, gc, c, cc = _both(3000, rt_direct, quality=quality)
    if quality == 0.0:
        assert gc["caustic"] == 0 and cc["caustic"] == 0
    assert gc["emitted"] == cc["emitted"]
    for k in ("stored", "global", "caustic"):
        assert abs(gc[k] - cc[k]) <= max(3, 0.01 * cc[k]), (k, gc, cc)
    # match photons by (path, bounce)
    gkey = (g["path"].astype(np.int64) << 8) | ((g["tag"] >> 8) & 0xFF)
    ckey = (c["path"].astype(np.int64) << 8) | ((c["tag"] >> 8) & 0xFF)
    common, gi, ci = np.intersect1d(gkey, ckey, return_indices=True)
    assert len(common) >= 0.98 * len(ckey)
    np.testing.assert_allclose(g["position"][gi], c["pos"][ci], atol=2e-4)
    np.testing.assert_allclose(g["omega_in"][gi], c["omega"][ci], atol=2e-4)
    np.testing.assert_allclose(g["power"][gi], c["power"][ci], rtol=2e-3, atol=1e-3)
    np.testing.assert_array_equal(g["tag"][gi] & 3, c["tag"][ci] & 3)


def test_trace_build_gather_pipeline():
    ctx = default_context()
    scene, _ = scenes_render.photon_scene()
    flat = R.flatten(scene)
    gs = R.GpuScene(ctx, flat)
    d = photons.photon_desc(50_000, max_emitted=2_000_000, wave=65536, ray_traced_direct=False)
    g, gc = photons.trace_photons(gs, d, capacity=500_000)
    assert gc["global"] >= 50_000
    glob = (g["tag"] & photons.GLOBAL) != 0
    pos = g["position"][glob].contiguous()
    r = photons.automatic_radius(g["power"][glob].cpu().numpy(), gc["emitted"], 64)
    m = photons.PhotonMap(ctx, device_ptr=pos.data_ptr(), n=pos.shape[0], r_max=r)
    q = pos[::37].cpu().numpy() + np.float32(1e-3)
    gi, gd, gn = m.gather(q, 64)
    ci, cd, cn = oracle.knn(pos.cpu().numpy(), q, 64, r)
    np.testing.assert_array_equal(gi, ci)
    np.testing.assert_array_equal(gn, cn)
    assert (gn == 64).mean() > 0.5
