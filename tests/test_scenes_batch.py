"""The batched workload's scene generator: seeded, uneven sizes in range, closed outward meshes."""
import numpy as np

from liar_b200 import render as R, scenes_batch as SB


def test_cube_sphere_is_closed_and_outward():
    rng = np.random.default_rng(0)
    v, t = SB.cube_sphere(6, (1.0, 2.0, 3.0), 0.5, rng)
    assert t.shape == (12 * 36, 3)
    # every directed edge appears once and its reverse once once duplicate vertices are merged
    key = {tuple(p): i for i, p in enumerate(v.tolist())}
    idx = np.array([key[tuple(p)] for p in v.tolist()])
    tt = idx[t]
    edges = np.concatenate([tt[:, [0, 1]], tt[:, [1, 2]], tt[:, [2, 0]]])
    fwd = {tuple(e) for e in edges.tolist()}
    assert len(fwd) == edges.shape[0]
    assert all((b, a) in fwd for a, b in fwd)
    c = v[t].mean(axis=1) - np.array([1.0, 2.0, 3.0])
    n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    assert (np.einsum("ij,ij->i", n, c) > 0).all()


def test_workload_sizes_seeded_and_in_range():
    w1 = SB.batch_workload(6, seed=5, tris=(10_000, 60_000), side=(16, 64), spp=(4, 64))
    w2 = SB.batch_workload(6, seed=5, tris=(10_000, 60_000), side=(16, 64), spp=(4, 64))
    for a, b in zip(w1, w2):
        assert (a.n_triangles, a.width, a.spp, a.materials) == (b.n_triangles, b.width, b.spp, b.materials)
        assert 9_000 <= a.n_triangles <= 66_000 and 16 <= a.width <= 64 and 4 <= a.spp <= 64
        flat = R.flatten(a.scene)
        assert flat.triangles.shape[0] == a.n_triangles + 2      # + the light's parallelogram
        assert len(flat.lights) == 2                              # sky + area light
