"""Scene API flattening: Box (scenery/box.cpp), Transformation (scenery/transformation.cpp) and
Translation (scenery/translation.cpp). The flattened triangle soup is what the GPU traces, so these
checks are on the host; the render tests cover the soup on the GPU."""
import math

import numpy as np
import pytest

from liar_b200 import render as R, scenery, shaders, spectra, textures


def _normals(flat):
    v, t = flat.vertices.astype(np.float64), flat.triangles
    n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def test_box_is_closed_and_outward():
    b = scenery.Box((-1, 0, 2), (3, 1, 5))
    flat = R.flatten(b)
    v, t = flat.vertices, flat.triangles
    assert t.shape == (12, 3)
    assert np.allclose(v.min(0), (-1, 0, 2)) and np.allclose(v.max(0), (3, 1, 5))
    c = v[t].mean(axis=1) - v.mean(axis=0)
    assert (np.einsum("ij,ij->i", _normals(flat), c) > 0).all()
    edges = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]).tolist()
    fwd = {tuple(e) for e in edges}
    assert len(fwd) == 36 and all((b_, a) in fwd for a, b_ in fwd)
    # total area of the faces
    vv = v.astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(vv[t[:, 1]] - vv[t[:, 0]], vv[t[:, 2]] - vv[t[:, 0]]), axis=1).sum()
    assert area == pytest.approx(2 * (4 * 1 + 4 * 3 + 1 * 3))


def test_box_constructors_match_the_reference():
    assert scenery.Box().bounds == ((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    assert scenery.Box(((0, 0, 0), (1, 2, 3))).max == (1.0, 2.0, 3.0)
    with pytest.raises(TypeError):
        scenery.Box(1, 2, 3)


def _rot_y(a, t=(0.0, 0.0, 0.0)):
    c, s = math.cos(a), math.sin(a)
    return [[c, 0, s, t[0]], [0, 1, 0, t[1]], [-s, 0, c, t[2]], [0, 0, 0, 1]]


def test_transformation_moves_vertices_normals_and_lights():
    mesh = scenery.TriangleMesh([(0, 0, 0), (1, 0, 0), (0, 0, 1)], [(0, 1, 0)], [],
                                [((0, 0), (1, 0), (2, 0))])
    mesh.shader = shaders.Lambert()
    lamp = scenery.LightArea(scenery.Parallelogram((0, 2, 0), (1, 0, 0), (0, 0, 1)))
    lamp.radiance = spectra.Spectrum(3.0)
    point = scenery.LightPoint((1, 1, 1), spectra.Spectrum(2.0))
    m = _rot_y(math.pi / 2, (5, 0, 0))
    flat = R.flatten(scenery.List([scenery.Transformation(scenery.List([mesh, lamp, point]), m)]))
    M = np.asarray(m)
    first = flat.vertices[:3].astype(np.float64)
    expect = np.array([(0, 0, 0, 1), (1, 0, 0, 1), (0, 0, 1, 1)], dtype=np.float64) @ M.T
    np.testing.assert_allclose(first, expect[:, :3], atol=1e-6)
    # a rotation keeps the normal's relation to the triangle
    np.testing.assert_allclose(flat.normals[0], (0, 1, 0), atol=1e-6)
    L = flat.lights[0]
    np.testing.assert_allclose(tuple(L.pos), (5, 2, 0), atol=1e-6)
    np.testing.assert_allclose(tuple(L.u), (0, 0, -1), atol=1e-6)
    np.testing.assert_allclose(tuple(L.v), (1, 0, 0), atol=1e-6)
    np.testing.assert_allclose(tuple(flat.lights[1].pos), (6, 1, -1), atol=1e-6)
    assert L.power == pytest.approx(math.pi * 1.0 * 3.0)


def test_nested_translation_and_scaled_normals():
    sph = scenery.Sphere((0, 0, 0), 1.0, subdivisions=1)
    sph.shader = shaders.Lambert()
    scale = [[2, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]]
    obj = scenery.Translation(scenery.Transformation(sph, scale), (0, 3, 0))
    assert obj.worldToLocal == (0.0, -3.0, 0.0)
    flat = R.flatten(obj)
    v = flat.vertices.astype(np.float64)
    assert np.allclose(v.min(0), (-2, 2, -1), atol=1e-6) and np.allclose(v.max(0), (2, 4, 1), atol=1e-6)
    # normals of the ellipsoid: the inverse transpose of the scale, renormalised
    p = (v - (0, 3, 0)) / (2, 1, 1)  # back to the unit sphere
    n_expect = p / np.array([2.0, 1.0, 1.0])
    n_expect /= np.linalg.norm(n_expect, axis=1, keepdims=True)
    idx = flat.triangle_normals[:, 0]
    np.testing.assert_allclose(flat.normals[idx], n_expect[flat.triangles[:, 0]], atol=1e-5)


def test_mirror_transformation_keeps_outward_winding():
    box = scenery.Box((0, 0, 0), (1, 1, 1))
    mirror = [[-1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]]
    flat = R.flatten(scenery.Transformation(box, mirror))
    v, t = flat.vertices, flat.triangles
    c = v[t].mean(axis=1) - v.mean(axis=0)
    assert (np.einsum("ij,ij->i", _normals(flat), c) > 0).all()
    lamp = scenery.LightArea(scenery.Parallelogram((0, 2, 0), (1, 0, 0), (0, 0, 1)))
    fl = R.flatten(scenery.List([box, scenery.Transformation(lamp, mirror)]))
    L = fl.lights[0]
    n_light = np.cross(tuple(L.u), tuple(L.v))
    tri = fl.triangles[-2:]
    vv = fl.vertices.astype(np.float64)
    n_tri = np.cross(vv[tri[0, 1]] - vv[tri[0, 0]], vv[tri[0, 2]] - vv[tri[0, 0]])
    assert np.dot(n_light, n_tri) > 0


def test_bad_transformations_are_refused():
    with pytest.raises(ValueError):
        scenery.Transformation(scenery.Box(), [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [1, 0, 0, 1]])
    with pytest.raises(ValueError):
        scenery.Transformation(scenery.Box(), np.zeros((4, 4)) + np.diag([0, 0, 0, 1]))
    with pytest.raises(ValueError):
        scenery.Transformation(scenery.Box(), [1, 2, 3])
    # a 3 x 4 matrix is accepted
    t = scenery.Transformation(scenery.Box(), [[1, 0, 0, 1], [0, 1, 0, 2], [0, 0, 1, 3]])
    assert t.localToWorld[3, 3] == 1.0
    assert np.allclose(t.worldToLocal[:3, 3], (-1, -2, -3))


def test_textured_constants_pass_through():
    """Shaders inside transformed subtrees keep their materials."""
    red = shaders.Lambert(textures.Constant(0.5))
    b = scenery.Box()
    b.shader = red
    flat = R.flatten(scenery.List([scenery.Translation(b, (1, 0, 0))]))
    assert flat.object_material.tolist() == [0]
