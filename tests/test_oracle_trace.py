"""CPU checks of the traversal oracle: analytic known answers of the triangle test, the
BoundedRay::inRange rule (src/liar/kernel/bounded_ray.h:69-77), ties, and agreement of the
oracle's tree with its brute-force definition."""
import numpy as np
import pytest

import oracle
from liar_b200 import scenes

A, B, C = (0, 0, 0), (1, 0, 0), (0, 1, 0)


def ray(o, d, tmin=0.0, tmax=np.inf):
    return np.array([[*o, tmin, *d, tmax]], dtype=np.float32)


def test_triangle_known_answers():
    assert oracle.tri_intersect((0.25, 0.25, 1), (0, 0, -1), A, B, C) == (1.0, 0.25, 0.25)
    # two-sided: from below
    assert oracle.tri_intersect((0.25, 0.25, -2), (0, 0, 1), A, B, C) == (2.0, 0.25, 0.25)
    # unnormalised direction: t in units of |d|
    assert oracle.tri_intersect((0.5, 0.25, 4), (0, 0, -2), A, B, C) == (2.0, 0.5, 0.25)
    assert oracle.tri_intersect((1, 1, 1), (0, 0, -1), A, B, C) is None       # outside
    assert oracle.tri_intersect((0.2, 0.2, 1), (1, 0, 0), A, B, C) is None     # parallel, det == 0
    # on the edges and corners: barycentrics exactly 0 or u + v == 1 are inside
    assert oracle.tri_intersect((0, 0, 1), (0, 0, -1), A, B, C) == (1.0, 0.0, 0.0)
    assert oracle.tri_intersect((0.5, 0.5, 1), (0, 0, -1), A, B, C) == (1.0, 0.5, 0.5)
    # behind the origin: the test itself reports negative t, the range check rejects it
    assert oracle.tri_intersect((0.25, 0.25, 1), (0, 0, 1), A, B, C) == (-1.0, 0.25, 0.25)


def tri_mesh(*tris):
    v = np.array([p for t in tris for p in t], dtype=np.float32)
    f = np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3)
    return v, f


@pytest.mark.parametrize("trace", ["brute", "tree"])
def test_in_range_rule(trace):
    v, f = tri_mesh((A, B, C))

    def run(r, any_hit=False):
        if trace == "brute":
            return oracle.trace_bruteforce(v, f, r, any_hit)
        return oracle.Tree(v, f).trace(r, any_hit)

    o, d = (0.25, 0.25, 1.0), (0.0, 0.0, -1.0)
    assert run(ray(o, d))[0][0] == 0
    assert run(ray(o, d, tmin=1.0))[0][0] == -1                # t must exceed the near limit
    assert run(ray(o, d, tmin=0.9999995))[0][0] == -1          # ... by the relative tolerance
    assert run(ray(o, d, tmin=0.999))[0][0] == 0
    assert run(ray(o, d, tmax=1.0))[0][0] == -1                # t < far * (1 - 1e-6)
    assert run(ray(o, d, tmax=1.0000005))[0][0] == -1
    assert run(ray(o, d, tmax=1.00001))[0][0] == 0
    # any hit: the plain open interval
    assert run(ray(o, d, tmax=1.0), True)[0][0] == -1
    assert run(ray(o, d, tmax=1.0000005), True)[0][0] == 0
    assert run(ray(o, d, tmin=1.0), True)[0][0] == -1


def test_ties_resolve_to_lower_index():
    t0 = (A, B, C)
    v, f = tri_mesh(t0, ((0, 0, 0), (0, 1, 0), (1, 0, 0)), t0)  # same plane, same t three times
    r = ray((0.25, 0.25, 1.0), (0, 0, -1))
    assert oracle.trace_bruteforce(v, f, r)[0][0] == 0
    assert oracle.Tree(v, f).trace(r)[0][0] == 0
    v2, f2 = tri_mesh(((0, 0, 0.5), (1, 0, 0.5), (0, 1, 0.5)), t0)
    assert oracle.trace_bruteforce(v2, f2, r)[0][0] == 0  # nearer plane wins


def test_tree_matches_bruteforce_random():
    v, f = scenes.displaced_icosphere(levels=4, seed=3)
    r = scenes.random_rays(v, 20000, seed=5)
    r[::7, 3] = 0.01                     # some near limits
    r[::5, 7] = 0.75                     # some far limits
    p1, t1 = oracle.trace_bruteforce(v, f, r)
    p2, t2 = oracle.Tree(v, f).trace(r)
    assert (p1 >= 0).mean() > 0.1
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(t1.view(np.int32), t2.view(np.int32))
    a1, _ = oracle.trace_bruteforce(v, f, r, True)
    a2, _ = oracle.Tree(v, f).trace(r, True)
    np.testing.assert_array_equal(a1 >= 0, a2 >= 0)
    # any hit <=> there is a triangle strictly inside (tmin, tmax); the closest hit lies in the
    # shrunk interval, so a closest hit implies an any hit
    assert np.all(a1[p1 >= 0] >= 0)


def test_vertex_rays_hit_consistently():
    """Rays aimed exactly at shared vertices and edge midpoints (several triangles tie). The
    Moller-Trumbore test is not watertight, so a few of these slip between triangles; what
    matters is that every traversal decides each of them identically."""
    v, f = scenes.displaced_icosphere(levels=2, seed=1)
    targets = np.concatenate([v, 0.5 * (v[f[:, 0]] + v[f[:, 1]])])
    o = np.zeros_like(targets)
    d = targets - o
    r = np.concatenate([o, np.zeros((len(o), 1)), d, np.full((len(o), 1), np.inf)], axis=1).astype(np.float32)
    p1, t1 = oracle.trace_bruteforce(v, f, r)
    p2, t2 = oracle.Tree(v, f).trace(r)
    assert (p1 >= 0).mean() > 0.5
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(t1, t2)


def test_icosphere_counts():
    v, f = scenes.displaced_icosphere(levels=3)
    assert v.shape == (10 * 4 ** 3 + 2, 3) and f.shape == (20 * 4 ** 3, 3)
    # closed, consistently connected mesh: every edge is shared by exactly two triangles
    e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    assert (counts == 2).all()
