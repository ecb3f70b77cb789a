"""Photon-map gather on the GPU against the brute-force restatement of KdTree::rangeSearch
(src/liar/tracers/photon_mapper.cpp:1257, 1312, 1352): identical neighbour indices, identical
squared distances (same IEEE operations), identical counts."""
import numpy as np
import pytest

import oracle
from liar_b200.kernel import default_context
from liar_b200.photons import PhotonMap

pytestmark = pytest.mark.gpu


def surface_photons(n, seed):
    """Photons on a few planes and a sphere, like photons stored on diffuse surfaces."""
    rng = np.random.default_rng(seed)
    a = rng.random((n // 2, 2))
    plane = np.stack([a[:, 0] * 4 - 2, np.zeros(len(a)), a[:, 1] * 4 - 2], axis=1)
    v = rng.normal(size=(n - n // 2, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    sphere = v * 0.6 + np.array([0, 0.6, 0])
    return np.concatenate([plane, sphere]).astype(np.float32)


@pytest.mark.parametrize("k,r", [(64, 0.05), (64, 0.2), (16, 0.1), (1, 0.3)])
def test_gather_matches_bruteforce(k, r):
    ctx = default_context()
    P = surface_photons(60000, seed=1)
    rng = np.random.default_rng(2)
    Q = np.concatenate([P[rng.choice(len(P), 3000, replace=False)] + rng.normal(scale=0.01, size=(3000, 3)),
                        rng.uniform(-2.5, 2.5, size=(1000, 3))]).astype(np.float32)
    m = PhotonMap(ctx, P, r_max=r)
    gi, gd, gc = m.gather(Q, k)
    ci, cd, cc = oracle.knn(P, Q, k, r)
    np.testing.assert_array_equal(gc, cc)
    np.testing.assert_array_equal(gi, ci)
    np.testing.assert_array_equal(gd.view(np.int32), cd.view(np.int32))
    assert (gc == k).mean() > 0.2 or r < 0.1


def test_gather_ties_and_duplicates():
    ctx = default_context()
    # many photons at exactly the same spot: ties in distance resolve to the lower index
    P = np.concatenate([np.zeros((100, 3)), np.full((50, 3), 0.01), np.random.default_rng(3).random((500, 3))])
    P = P.astype(np.float32)
    Q = np.array([[0, 0, 0], [0.005, 0.005, 0.005], [10, 10, 10]], np.float32)
    m = PhotonMap(ctx, P, r_max=0.5)
    gi, gd, gc = m.gather(Q, 64)
    ci, cd, cc = oracle.knn(P, Q, 64, 0.5)
    np.testing.assert_array_equal(gi, ci)
    np.testing.assert_array_equal(gc, cc)
    assert gc[2] == 0 and (gi[2] == -1).all() and np.isinf(gd[2]).all()
    np.testing.assert_array_equal(gi[0, :64], np.arange(64))


def test_gather_empty_map_and_queries():
    ctx = default_context()
    m = PhotonMap(ctx, np.zeros((0, 3), np.float32), r_max=0.1)
    gi, gd, gc = m.gather(np.zeros((5, 3), np.float32), 8)
    assert (gc == 0).all() and (gi == -1).all()
    m2 = PhotonMap(ctx, np.ones((10, 3), np.float32), r_max=0.1)
    gi, gd, gc = m2.gather(np.zeros((0, 3), np.float32), 8)
    assert gi.shape == (0, 8)


def test_gather_rejects_bad_arguments():
    from liar_b200._native import LiarGpuError
    ctx = default_context()
    with pytest.raises(LiarGpuError, match="INVALID"):
        PhotonMap(ctx, np.ones((3, 3), np.float32), r_max=0.0)
    m = PhotonMap(ctx, np.ones((3, 3), np.float32), r_max=1.0)
    with pytest.raises(LiarGpuError, match="INVALID"):
        m.gather(np.zeros((2, 3), np.float32), 65)


def test_rebuild_in_place_matches_a_fresh_map():
    """A map rebuilt over other photons (fewer, then more than its buffers hold, and another
    radius) answers exactly like a map built fresh over them."""
    import torch
    ctx = default_context()
    rng = np.random.default_rng(9)
    Q = rng.uniform(-2, 2, size=(2000, 3)).astype(np.float32)
    first = torch.from_numpy(surface_photons(40000, seed=3)).cuda()
    m = PhotonMap(ctx, device_ptr=first.data_ptr(), n=40000, r_max=0.1)
    for n, r, seed in ((20000, 0.1, 4), (80000, 0.15, 5)):
        P = surface_photons(n, seed=seed)
        d = torch.from_numpy(P).cuda()
        m.rebuild(d.data_ptr(), n, r)
        torch.cuda.synchronize()
        gi, gd, gc = m.gather(Q, 32)
        ci, cd, cc = oracle.knn(P, Q, 32, r)
        np.testing.assert_array_equal(gc, cc)
        np.testing.assert_array_equal(gi, ci)
        np.testing.assert_array_equal(gd.view(np.int32), cd.view(np.int32))


def test_many_queries_take_the_spatially_ordered_path():
    """From 32,768 queries on, the gather orders them along a Morton curve first; the answers stay
    those of each query, in the caller's order."""
    ctx = default_context()
    P = surface_photons(100000, seed=11)
    rng = np.random.default_rng(12)
    Q = np.concatenate([P[rng.choice(len(P), 30000, replace=False)] + rng.normal(scale=0.02, size=(30000, 3)),
                        rng.uniform(-2.5, 2.5, size=(10000, 3))]).astype(np.float32)
    rng.shuffle(Q)
    m = PhotonMap(ctx, P, r_max=0.08)
    gi, gd, gc = m.gather(Q, 48)
    ci, cd, cc = oracle.knn_grid(P, Q, 48, 0.08)
    np.testing.assert_array_equal(gc, cc)
    np.testing.assert_array_equal(gi, ci)
    np.testing.assert_array_equal(gd.view(np.int32), cd.view(np.int32))
