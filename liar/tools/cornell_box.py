"""The Cornell box (the reference's liar.tools.cornell_box, src/liar/tools/cornell_box.py:19-136).

scene() = lights() + walls() + blocks(); camera() looks into the open side. Geometry is the
Cornell University Program of Computer Graphics' Cornell box in millimetres, scaled to metres;
the walls, blocks and light use its measured spectra (white, red and green reflectances and the
light's emission, 400-700 nm). The light is a 130 x 105 mm LightArea just below the ceiling with
16 emission samples and a shader that both emits its radiance and reflects as Lambert 0.78.
"""
from __future__ import annotations

import math

from liar_b200 import _tables, cameras, scenery, shaders, textures
from liar_b200.spectra import Sampled


def _measured():
    t = _tables.cornell_box()
    ws = t["wavelengths"]
    return tuple(Sampled(ws, t[k]) for k in ("white", "red", "green", "light"))


_WHITE, _RED, _GREEN, _LIGHT = _measured()


def _mm(x, y, z):
    return (0.01 * x, 0.01 * y, 0.01 * z)


def scene():
    return scenery.List(lights() + walls() + blocks())


def camera():
    cam = cameras.PerspectiveCamera()
    cam.aspectRatio = 1
    # a 35 mm lens in front of a 25 mm film
    cam.fovAngle = 2 * math.atan((0.025 / 0.035) / 2)
    cam.position = _mm(278, 273, -800)
    cam.sky = (0, 1, 0)
    cam.direction = (0, 0, 1)
    return cam


def lights():
    surface = scenery.Parallelogram(_mm(213, 548.79, 227), _mm(343 - 213, 0, 0), _mm(0, 0, 332 - 227))
    light = scenery.LightArea(surface)
    light.radiance = _LIGHT
    light.numberOfEmissionSamples = 16
    light.shader = shaders.Sum([shaders.Unshaded(textures.Constant(light.radiance)),
                                shaders.Lambert(textures.Constant(0.78))])
    return [light]


def walls():
    white = shaders.Lambert(textures.Constant(_WHITE))
    red = shaders.Lambert(textures.Constant(_RED))
    green = shaders.Lambert(textures.Constant(_GREEN))
    # (support, first side, second side) in mm; the sides' cross product faces into the box
    quads = [
        ((0, 0, 559.2), (552.8, 0, 0), (0, 0, -559.2), white),      # floor
        ((0.0, 548.8, 0), (556.0, 0, 0), (0, 0, 559.2), white),     # ceiling
        ((556, 0, 559.2), (-556.0, 0, 0), (0, 548.8, 0), white),    # back wall
        ((0, 0, 559.2), (0, 0, -559.2), (0, 548.8, 0), green),      # right wall
        ((552.8, 0, 0), (0, 0, 559.2), (0, 548.8, 0), red),         # left wall
    ]
    out = []
    for support, u, v, shader in quads:
        wall = scenery.Parallelogram(_mm(*support), _mm(*u), _mm(*v))
        wall.shader = shader
        out.append(wall)
    return out


def blocks():
    white = shaders.Lambert(textures.Constant(_WHITE))
    short = _block([(130.0, 65.0), (82.0, 225.0), (240.0, 272.0), (290.0, 114.0)], [0.05, 165.0])
    tall = _block([(423.0, 247.0), (265.0, 296.0), (314.0, 456.0), (472.0, 406.0)], [0.05, 330.0])
    short.shader = white
    tall.shader = white
    return [short, tall]


def _block(footprint, heights):
    """A prism over a quadrilateral footprint (x, z in mm) between two heights: 8 corners (the
    footprint at the lower height, then at the upper one), 6 faces of 2 triangles each, every face
    with its own flat normal."""
    verts = [_mm(x, h, z) for h in heights for (x, z) in footprint]

    def face_normal(a, b, c):
        pa, pb, pc = verts[a], verts[b], verts[c]
        u = [pb[k] - pa[k] for k in range(3)]
        v = [pc[k] - pa[k] for k in range(3)]
        n = (u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0])
        length = math.sqrt(sum(x * x for x in n))
        return tuple(x / length for x in n)

    # per face: the corners that span its normal, and its two triangles
    faces = [
        ((0, 3, 1), [(0, 2, 1), (0, 3, 2)]),  # bottom
        ((4, 5, 7), [(4, 6, 7), (4, 5, 6)]),  # top
        ((0, 1, 4), [(0, 5, 4), (0, 1, 5)]),
        ((1, 2, 5), [(1, 6, 5), (1, 2, 6)]),
        ((2, 3, 6), [(2, 7, 6), (2, 3, 7)]),
        ((3, 0, 7), [(3, 4, 7), (3, 0, 4)]),
    ]
    normals = [face_normal(*span) for span, _ in faces]
    triangles = [tuple((corner, n) for corner in tri) for n, (_, tris) in enumerate(faces) for tri in tris]
    return scenery.TriangleMesh(verts, normals, [], triangles)
