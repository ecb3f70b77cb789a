"""GPU parity of closest hit / any hit through the C ABI against the CPU oracle.

Bar: the hit triangle index and the bit pattern of t are identical to the oracle's for every
ray (the triangle test is evaluated with the same IEEE roundings on both sides and equal t
resolves to the lower index), which is stricter than the 1e-6 tie / 1e-5 relative-t tolerance
the workload states."""
import numpy as np
import pytest

import oracle
from liar_b200 import scenes
from liar_b200._native import LiarGpuError
from liar_b200.trace import Mesh

pytestmark = pytest.mark.gpu


def assert_same(p_gpu, t_gpu, p_ref, t_ref):
    bad = np.nonzero(p_gpu != p_ref)[0]
    assert bad.size == 0, f"{bad.size} index mismatches, first {bad[:5]}: gpu {p_gpu[bad[:5]]} ref {p_ref[bad[:5]]}"
    hit = p_ref >= 0
    np.testing.assert_array_equal(t_gpu[hit].view(np.int32), t_ref[hit].view(np.int32))
    assert np.all(np.isinf(t_gpu[~hit]))


def edge_rays(v, f, n_extra=2000, seed=0):
    """Rays from inside the mesh aimed at vertices and edge midpoints, plus random ones."""
    targets = np.concatenate([v, 0.5 * (v[f[:, 0]] + v[f[:, 1]])])
    c = v.mean(axis=0)
    o = np.broadcast_to(c, targets.shape)
    r = np.concatenate([o, np.zeros((len(o), 1)), targets - o, np.full((len(o), 1), np.inf)], axis=1)
    return np.concatenate([r.astype(np.float32), scenes.random_rays(v, n_extra, seed=seed)])


@pytest.mark.parametrize("leaf", [1, 4, 8])
def test_matches_bruteforce_small(gpu_ctx, leaf):
    v, f = scenes.displaced_icosphere(levels=3, seed=2)
    r = np.concatenate([scenes.random_rays(v, 40000, seed=1), edge_rays(v, f)])
    r[::11, 3] = 0.05
    r[::13, 7] = 0.8
    mesh = Mesh(gpu_ctx, v, f, max_leaf_size=leaf)
    p, t = mesh.intersect(r)
    pr, tr = oracle.trace_bruteforce(v, f, r)
    assert (pr >= 0).mean() > 0.2
    assert_same(p, t, pr, tr)
    pa, _ = mesh.intersect(r, any_hit=True)
    par, _ = oracle.trace_bruteforce(v, f, r, any_hit=True)
    np.testing.assert_array_equal(pa >= 0, par >= 0)


def test_matches_oracle_on_workload_mesh(gpu_ctx):
    """The 1,310,720-triangle displaced icosphere, 1M rays of the workload distribution."""
    v, f = scenes.displaced_icosphere(levels=8, seed=0)
    mesh = Mesh(gpu_ctx, v, f)
    st = mesh.stats
    assert st["n_triangles"] == 1310720 and st["stack_needed"] <= 64
    r = scenes.random_rays(v, 1 << 20, seed=7)
    p, t = mesh.intersect(r)
    tree = oracle.Tree(v, f)
    pr, tr = tree.trace(r)
    assert_same(p, t, pr, tr)
    ra = r.copy()
    ra[:, 7] = 0.5
    pa, _ = mesh.intersect(ra, any_hit=True)
    par, _ = tree.trace(ra, any_hit=True)
    np.testing.assert_array_equal(pa >= 0, par >= 0)


def test_edge_cases(gpu_ctx):
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    v = np.array([a, b, c, a, c, b, a, b, c, (0, 0, 0), (0, 0, 0), (1, 1, 0)], dtype=np.float32)
    f = np.arange(12, dtype=np.uint32).reshape(4, 3)  # tri 3 is degenerate (zero area)
    mesh = Mesh(gpu_ctx, v, f)
    # empty batch
    p, t = mesh.intersect(np.zeros((0, 8), np.float32))
    assert p.shape == (0,)
    # ties resolve to the lower index; near/far limits; NaN rays miss
    r = np.array([
        [0.25, 0.25, 1, 0, 0, 0, -1, np.inf],
        [0.25, 0.25, 1, 1.0, 0, 0, -1, np.inf],
        [0.25, 0.25, 1, 0, 0, 0, -1, 1.0],
        [0.25, 0.25, 1, 0, 0, 0, -1, 1.00001],
        [np.nan, 0.25, 1, 0, 0, 0, -1, np.inf],
        [0.25, 0.25, 1, 0, 0, 0, 0, np.inf],          # zero direction
        [0.25, 0.25, -3, 0, 0, 0, 2, np.inf],         # from below, unnormalised
    ], dtype=np.float32)
    p, t = mesh.intersect(r)
    np.testing.assert_array_equal(p, [0, -1, -1, 0, -1, -1, 0])
    assert t[0] == 1.0 and t[6] == 1.5
    pr, tr = oracle.trace_bruteforce(v, f, r)
    np.testing.assert_array_equal(p, pr)
    # ragged batch sizes around the warp width
    rr = scenes.random_rays(v, 97, seed=3)
    for n in (1, 31, 32, 33, 97):
        p, _ = mesh.intersect(rr[:n])
        pr, _ = oracle.trace_bruteforce(v, f, rr[:n])
        np.testing.assert_array_equal(p, pr)


def test_invalid_meshes_raise(gpu_ctx):
    v = np.zeros((3, 3), np.float32)
    with pytest.raises(LiarGpuError, match="INVALID"):
        Mesh(gpu_ctx, v, np.array([[0, 1, 5]], np.uint32))
    with pytest.raises(LiarGpuError, match="INVALID"):
        Mesh(gpu_ctx, np.array([[0, 0, np.nan], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    with pytest.raises(LiarGpuError, match="INVALID"):
        Mesh(gpu_ctx, v, np.zeros((0, 3), np.uint32))


def test_device_entry_point_matches_host(gpu_ctx):
    import torch
    v, f = scenes.displaced_icosphere(levels=5, seed=4)
    mesh = Mesh(gpu_ctx, v, f)
    r = scenes.random_rays(v, 100003, seed=9)
    p, t = mesh.intersect(r)
    rd = torch.from_numpy(r).cuda()
    hd = torch.empty((len(r), 2), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    mesh.trace_into(rd.data_ptr(), len(r), hd.data_ptr(), stream=s.cuda_stream, counters_ptr=cnt.data_ptr())
    s.synchronize()
    gpu_ctx.synchronize()
    h = hd.cpu().numpy()
    np.testing.assert_array_equal(h[:, 0], p)
    np.testing.assert_array_equal(h[:, 1].view(np.float32)[p >= 0], t[p >= 0])
    nodes, tris = cnt.cpu().tolist()
    assert nodes >= len(r) and tris > 0


def test_full_size_properties(gpu_ctx):
    """16,777,216 rays on the workload mesh: properties that do not need a full CPU trace."""
    v, f = scenes.displaced_icosphere(levels=8, seed=0)
    mesh = Mesh(gpu_ctx, v, f)
    r = scenes.random_rays(v, 1 << 24, seed=0)
    p, t = mesh.intersect(r)
    p2, t2 = mesh.intersect(r)
    np.testing.assert_array_equal(p, p2)                         # deterministic
    hit = p >= 0
    assert 0.15 < hit.mean() < 0.6
    assert np.all(t[hit] > 0) and np.all(np.isfinite(t[hit]))
    ra = r.copy()
    ra[:, 7] = 0.5
    pa, _ = mesh.intersect(ra, any_hit=True)
    # closest hit below the shrunk far limit implies an occluder in (0, 0.5), and an occluder
    # in (0, 0.5) implies a closest hit no farther than 0.5
    assert np.all(pa[hit & (t < 0.5 * (1 - 1e-6))] >= 0)
    assert np.all(hit[pa >= 0]) and np.all(t[pa >= 0] < 0.5)
    # the hit point lies on the reported triangle's plane
    idx = np.nonzero(hit)[0][:: max(1, hit.sum() // 200000)]
    o, d = r[idx, :3].astype(np.float64), r[idx, 4:7].astype(np.float64)
    x = o + t[idx, None] * d
    tri = v[f[p[idx]]].astype(np.float64)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    assert np.max(np.abs(np.einsum("ij,ij->i", x - tri[:, 0], n))) < 1e-5
    # a 1M-ray sample of the same call agrees with the oracle exactly
    s = np.random.default_rng(1).choice(len(r), 1 << 20, replace=False)
    pr, tr = oracle.Tree(v, f).trace(r[s])
    assert_same(p[s], t[s], pr, tr)


@pytest.mark.parametrize("cfg", [(128, 8), (128, 16), (128, 24), (256, 8), (256, 16)])
def test_every_launch_shape_matches_oracle(gpu_ctx, cfg):
    """All trace kernel variants give identical results; the 8-entry shared stack makes deep rays
    spill to local memory on the 1.3M-triangle mesh."""
    v, f = scenes.displaced_icosphere(levels=8, seed=0)
    mesh = Mesh(gpu_ctx, v, f)
    r = scenes.random_rays(v, 1 << 18, seed=21)
    # rays from the centre cross the whole sphere's subtree: deep stacks
    r[::2, 0:3] = 0.0
    old = gpu_ctx.trace_config
    try:
        gpu_ctx.trace_config = cfg
        assert gpu_ctx.trace_config == cfg
        p, t = mesh.intersect(r)
        pa, _ = mesh.intersect(r, any_hit=True)
    finally:
        gpu_ctx.trace_config = old
    pr, tr = oracle.Tree(v, f).trace(r)
    assert_same(p, t, pr, tr)
    np.testing.assert_array_equal(pa >= 0, oracle.Tree(v, f).trace(r, any_hit=True)[0] >= 0)


def test_unsupported_launch_shape_is_rejected(gpu_ctx):
    with pytest.raises(LiarGpuError, match="INVALID"):
        gpu_ctx.trace_config = (96, 16)
    assert gpu_ctx.trace_config == (128, 16)
