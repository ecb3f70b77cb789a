"""uv textures of the scene API (src/liar/textures/checker_board.cpp, grid_board.cpp,
transformation_uv.cpp): their flattening into liar_texture trees, the surface coordinates of the
shapes, and the oracle's renders of a checker board lit by a uniform sky, whose quadrants show the
board's reflectances."""
import numpy as np
import pytest

import oracle
from liar_b200 import cameras, output, render as R, scenery, shaders, spectra, textures as tx, tracers


def test_checker_tree_is_flattened_once_per_node():
    white, black = tx.Constant(0.8), tx.Constant(0.2)
    board = tx.CheckerBoard(white, black)
    board.split = (0.25, 0.75)
    board.antiAliasing = tx.CheckerBoard.AA_NONE
    moved = tx.TransformationUv(board, [[4, 0, 0.5], [0, 4, 0], [0, 0, 1]])
    grid = tx.GridBoard(moved, black)
    grid.thickness = (0.2, 0.4)
    a = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    a.shader = shaders.Lambert(grid)
    b = scenery.Parallelogram((0, 0, 1), (1, 0, 0), (0, 1, 0))
    b.shader = shaders.Lambert(board)   # shares the board's nodes
    flat = R.flatten(scenery.List([a, b]))
    T = list(flat.textures)
    kinds = [t.type for t in T]
    assert kinds.count(R.TEX_CHECKER) == 1 and kinds.count(R.TEX_GRID) == 1 and kinds.count(R.TEX_UV_TRANSFORM) == 1
    assert kinds.count(R.TEX_CONSTANT) == 2
    m0, m1 = flat.materials[0], flat.materials[1]
    assert m0.spec[0] == -1 and m1.spec[0] == -1
    g = T[m0.tex[0]]
    assert g.type == R.TEX_GRID and tuple(g.p[:2]) == pytest.approx((0.1, 0.2))   # half thickness
    tr = T[g.a]
    assert tr.type == R.TEX_UV_TRANSFORM and list(tr.p) == pytest.approx([4, 0, 0.5, 0, 4, 0])
    assert tr.a == m1.tex[0] and T[tr.a].type == R.TEX_CHECKER and tuple(T[tr.a].p[:2]) == (0.25, 0.75)
    assert T[T[tr.a].b].spectrum == T[g.b].spectrum
    # parallelogram uvs: (u, v) of support + u sizeU + v sizeV at the corners
    np.testing.assert_array_equal(flat.triangle_uvs[:2].reshape(2, 3, 2), a.corner_uvs())


def test_constant_only_scenes_carry_no_uvs_and_constants_stay_spectra():
    p = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    p.shader = shaders.Lambert(tx.Constant(0.5))
    flat = R.flatten(p)
    assert flat.triangle_uvs is None and flat.textures is None
    assert flat.materials[0].tex[0] == -1 and flat.materials[0].spec[0] >= 0


def test_shape_uvs():
    box = scenery.Box((0, 0, 0), (2, 1, 4))
    v, t, _, _ = box.triangles()
    uv = box.corner_uvs()
    for k in range(12):
        axis, positive = k // 4, (k // 2) % 2 == 1
        i, j = (axis + 1) % 3, (axis + 2) % 3
        for c in range(3):
            p = v[t[k][c]]
            expect_v = p[j] / (2, 1, 4)[j]
            assert uv[k, c, 0] == pytest.approx(p[i] / (2, 1, 4)[i])
            assert uv[k, c, 1] == pytest.approx(expect_v if positive else 1 - expect_v)
    sphere = scenery.Sphere((1, 2, 3), 2.0, subdivisions=2)
    sv, st, _, _ = sphere.triangles()
    suv = sphere.corner_uvs()
    n = (sv.astype(np.float64) - (1, 2, 3)) / 2.0
    theta = np.arccos(np.clip(n[:, 2], -1, 1)) / np.pi
    np.testing.assert_allclose(suv[..., 1], theta[st], atol=1e-6)
    assert (np.ptp(suv[..., 0], axis=1) < 0.3).all()      # unwrapped across the seam
    mesh = scenery.TriangleMesh([(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)], (), [(0.1, 0.2), (0.3, 0.4), (0.5, 0.6)],
                                [((0, None, 0), (1, None, 1), (2, None, 2)), (1, 3, 2)])
    muv = mesh.corner_uvs()
    np.testing.assert_allclose(muv[0], [[0.1, 0.2], [0.3, 0.4], [0.5, 0.6]])
    np.testing.assert_allclose(muv[1], [[0, 0], [1, 0], [0, 1]])   # no uvs: the barycentrics


def test_mirroring_transformation_rewinds_uvs_with_the_triangles():
    p = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    p.shader = shaders.Lambert(tx.CheckerBoard(0.1, 0.9))
    m = scenery.Transformation(p, [[-1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])
    flat = R.flatten(m)
    uv = flat.triangle_uvs.reshape(-1, 3, 2)
    np.testing.assert_array_equal(uv, p.corner_uvs()[:, [0, 2, 1]])
    assert (flat.triangles == np.array([[0, 2, 1], [0, 3, 2]])).all()


def test_bad_texture_uses_fail_loudly():
    with pytest.raises(NotImplementedError):
        tx.TransformationUv(tx.Constant(1), [[1, 0, 0], [0, 1, 0], [0.5, 0, 1]])
    with pytest.raises(KeyError):
        tx.CheckerBoard(0, 1).antiAliasing = "trilinear"
    light = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    light.shader = shaders.Unshaded(tx.CheckerBoard(0, 1))
    with pytest.raises(TypeError):
        R.flatten(light)


def _board_scene(texture):
    """A unit checker plane z = 0 (uv = (x, y)) under a uniform sky of radiance 1, seen from above
    with x to the right of the image and y up: the view covers x in [0.1, 0.9], y in [0.2, 0.8]."""
    plane = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    plane.shader = shaders.Lambert(texture)
    sky = scenery.LightSky(tx.Constant(1.0))
    cam = cameras.PerspectiveCamera()
    cam.position = (0.5, 0.5, 0.4)
    cam.sky = (0, 1, 0)
    cam.lookAt((0.5, 0.5, 0.0))
    return scenery.List([plane, sky]), cam


def _quadrants(img, w, h, band=3):
    """Mean luminance of the image's top-left, top-right, bottom-left and bottom-right quadrants,
    leaving out a band around the middle lines."""
    Y = img[..., 1]
    cx, cy = w // 2, h // 2
    return (Y[:cy - band, :cx - band].mean(), Y[:cy - band, cx + band:].mean(),
            Y[cy + band:, :cx - band].mean(), Y[cy + band:, cx + band:].mean())


@pytest.mark.parametrize("shift", [False, True])
def test_oracle_checker_board_quadrants(shift):
    a, b = 0.8, 0.2
    board = tx.CheckerBoard(tx.Constant(a), tx.Constant(b))
    board.antiAliasing = "none"
    tex = tx.TransformationUv(board, [[1, 0, 0.5], [0, 1, 0], [0, 0, 1]]) if shift else board
    scene, cam = _board_scene(tex)
    t = tracers.DirectLighting()
    t.maxRayGeneration = 1
    w, h = 40, 30
    flat = R.flatten(scene)
    img, _ = R.resolve(oracle.RenderScene(flat).render(R.render_desc(cam, w, h, 16, t, seed=1)))
    tl, tr, bl, br = _quadrants(img, w, h)
    # A where u and v lie on the same side of the split: (u > 0.5, v > 0.5) is the top right
    expect = (b, a, a, b) if not shift else (a, b, b, a)
    np.testing.assert_allclose((tl, tr, bl, br), expect, rtol=0.05)


def test_oracle_grid_board_lines():
    grid = tx.GridBoard(tx.Constant(0.9), tx.Constant(0.1))
    grid.thickness = (0.2, 0.2)
    # 2 cells per unit: lines (0.1 wide in uv) at x = 0.5 and y = 0.5 cross the image's middle
    scene, cam = _board_scene(tx.TransformationUv(grid, [[2, 0, 0], [0, 2, 0], [0, 0, 1]]))
    t = tracers.DirectLighting()
    t.maxRayGeneration = 1
    w, h = 40, 30
    img, _ = R.resolve(oracle.RenderScene(R.flatten(scene)).render(R.render_desc(cam, w, h, 8, t, seed=2)))
    Y = img[..., 1]
    assert Y[h // 2 - 1:h // 2 + 1, :].mean() == pytest.approx(0.9, rel=0.05)    # the line y = 0.5
    assert Y[:, w // 2 - 1:w // 2 + 1].mean() == pytest.approx(0.9, rel=0.05)    # the line x = 0.5
    assert Y[4:10, 6:12].mean() == pytest.approx(0.1, rel=0.1)                    # inside a cell


def _grey_xyz(levels):
    """XYZ of equal-energy greys (x = y = 1/3) of the given luminances."""
    lv = np.asarray(levels, dtype=np.float32)
    return np.stack([lv, lv, lv], axis=-1)


def test_image_texture_is_flattened_into_the_pixel_pool(tmp_path):
    a = tx.Image.from_xyz(_grey_xyz([[0.2, 0.4, 0.3], [0.6, 0.8, 0.5]]), antiAliasing="none")
    b = tx.Image.from_xyz(_grey_xyz([[0.1], [0.9]]))
    p = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    p.shader = shaders.Lambert(a)
    q = scenery.Parallelogram((0, 0, 1), (1, 0, 0), (0, 1, 0))
    q.shader = shaders.Lambert(tx.TransformationUv(b, [[2, 0, 0], [0, 1, 0], [0, 0, 1]]))
    flat = R.flatten(scenery.List([p, q]))
    T = list(flat.textures)
    ia = T[flat.materials[0].tex[0]]
    ib = T[T[flat.materials[1].tex[0]].a]
    # each image: its mip table (a header and one entry per level; from_xyz has no mip levels),
    # then the pixels
    assert (ia.type, ia.a, ia.b, ia.pixels, ia.p[0]) == (R.TEX_IMAGE, 3, 2, 0, 0.0)
    assert (ib.type, ib.a, ib.b, ib.pixels, ib.p[0]) == (R.TEX_IMAGE, 1, 2, 8, 1.0)
    assert flat.texture_pixels.shape == (12, 4)
    head = flat.texture_pixels[:2].view(np.int32)
    assert list(head[0]) == [1, 1, 0, 0] and list(head[1]) == [2, 0, 3, 2]
    np.testing.assert_array_equal(flat.texture_pixels[2:8, 1], np.float32([0.2, 0.4, 0.3, 0.6, 0.8, 0.5]))
    # a file is read in its codec's colour space
    img = output.Image(str(tmp_path / "t.pfm"), (3, 2))
    img.exposureStops = 0.0
    xyza = np.concatenate([_grey_xyz([[0.2, 0.4, 0.3], [0.6, 0.8, 0.5]]), np.ones((2, 3, 1), np.float32)], -1)
    img.write(xyza, None)
    t = tx.Image(str(tmp_path / "t.pfm"))
    assert t.resolution == (3, 2) and t.antiAliasing == "trilinear" and t.mipMapping == "anisotropic"
    assert t.rgbSpace.gamma == 1.0
    np.testing.assert_allclose(t.xyz, xyza[..., :3], rtol=1e-5, atol=1e-6)
    p.shader = shaders.Lambert(t)
    f2 = R.flatten(p)
    # anisotropic levels of a 3 x 2 image: 2 along u (3, 1 wide) x 2 along v (2, 1 high)
    assert f2.textures[f2.materials[0].tex[0]].p[0] == 2.0
    assert list(f2.texture_pixels[:1].view(np.int32)[0]) == [2, 2, 2, 0]


@pytest.mark.parametrize("filter", ["none", "bilinear"])
def test_oracle_image_quadrants(filter):
    levels = np.array([[0.2, 0.7], [0.45, 0.1]], np.float32)
    tex = tx.Image.from_xyz(_grey_xyz(levels), antiAliasing=filter)
    scene, cam = _board_scene(tex)
    t = tracers.DirectLighting()
    t.maxRayGeneration = 1
    w, h = 40, 30
    img, _ = R.resolve(oracle.RenderScene(R.flatten(scene)).render(R.render_desc(cam, w, h, 16, t, seed=3)))
    tl, tr, bl, br = _quadrants(img, w, h, band=5 if filter == "none" else 1)
    if filter == "none":
        # the image's top row at the top of the plane (v up), its pixels filling the quadrants
        np.testing.assert_allclose((tl, tr, bl, br), levels.ravel(), rtol=0.05)
    else:
        # bilinear between pixel centres (u, v = 0.25, 0.75) with wrap-around: at the view's
        # corners the nearest pixel dominates, in the middle all four blend equally
        Y = img[..., 1]
        assert Y[h // 2 - 1:h // 2 + 1, w // 2 - 1:w // 2 + 1].mean() == pytest.approx(levels.mean(), rel=0.05)
        assert list(np.argsort([tl, tr, bl, br])) == list(np.argsort(levels.ravel()))


def _noise(tables, p):
    """Improved Perlin noise as perlin.cpp:60-90, 170-205 states it, in numpy (float64)."""
    G = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
                  [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1], [1, 1, 0], [-1, 1, 0], [0, -1, 1], [0, -1, -1]])
    q = np.mod(p, 256.0)
    i = np.floor(q).astype(int)
    d = q - i
    fade = lambda t: (6 * t ** 3 - 15 * t ** 2 + 10 * t) * t ** 2
    s = fade(d)
    g = {}
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                h = tables[0][i[..., 0] + a] ^ tables[1][i[..., 1] + b] ^ tables[2][i[..., 2] + c]
                grad = G[h % 16]
                g[a, b, c] = (grad * (d - (a, b, c))).sum(-1)
    lerp = lambda x, y, t: x + t * (y - x)
    return lerp(lerp(lerp(g[0, 0, 0], g[1, 0, 0], s[..., 0]), lerp(g[0, 1, 0], g[1, 1, 0], s[..., 0]), s[..., 1]),
                lerp(lerp(g[0, 0, 1], g[1, 0, 1], s[..., 0]), lerp(g[0, 1, 1], g[1, 1, 1], s[..., 0]), s[..., 1]), s[..., 2])


def test_noise_tables_and_flattening():
    p = tx.Perlin(7)
    assert p.tables.shape == (3, 257) and (p.tables[:, 256] == p.tables[:, 0]).all()
    assert all(sorted(t[:256]) == list(range(256)) for t in p.tables)
    assert (tx.Perlin(7).tables == p.tables).all() and not (tx.Perlin(8).tables == p.tables).all()
    f = tx.FBm(5, 0.6)
    tex = tx.Sum([tx.Constant(0.25), 0.25, tx.Product(tx.Constant(0.5), tx.Abs(f))])
    plane = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    plane.shader = shaders.Lambert(tex)
    flat = R.flatten(plane)
    T = list(flat.textures)
    s = T[flat.materials[0].tex[0]]
    assert s.type == R.TEX_AFFINE and tuple(s.p[:2]) == (1.0, 0.5)
    m = T[s.a]
    assert m.type == R.TEX_AFFINE and tuple(m.p[:2]) == (0.5, 0.0)
    a = T[m.a]
    n = T[a.a]
    assert a.type == R.TEX_ABS and n.type == R.TEX_NOISE and tuple(n.p[:2]) == pytest.approx((5.0, 0.6))
    np.testing.assert_array_equal(flat.noise_tables[n.pixels:n.pixels + 771], f.tables.reshape(-1))
    with pytest.raises(NotImplementedError):
        plane.shader = shaders.Lambert(tx.Product(tx.Perlin(), tx.Perlin(1)))
        R.flatten(plane)


@pytest.mark.parametrize("octaves", [0, 3])
def test_oracle_noise_follows_the_hit_point(octaves):
    """A plane shaded with 0.5 + 0.4 noise(x) under a uniform sky shows that reflectance at every
    pixel: the oracle's noise against the numpy statement above, at the pixel centres' hits."""
    noise = tx.FBm(octaves, 0.5) if octaves else tx.Perlin(3)
    scene, cam = _board_scene(tx.Sum(0.5, tx.Product(0.4, noise)))
    t = tracers.DirectLighting()
    t.maxRayGeneration = 1
    w, h = 40, 30
    img, var = R.resolve(oracle.RenderScene(R.flatten(scene)).render(R.render_desc(cam, w, h, 64, t, seed=4)))
    # pixel centres on the plane: x right over [0.1, 0.9], y up over [0.2, 0.8]
    xs = 0.5 + 0.4 * (2 * (np.arange(w) + 0.5) / w - 1)
    ys = 0.5 - 0.3 * (2 * (np.arange(h) + 0.5) / h - 1)
    P = np.stack(list(np.meshgrid(xs, ys)) + [np.zeros((h, w))], axis=-1)
    n = np.zeros((h, w))
    for k in range(max(octaves, 1)):
        n += 0.5 ** k * _noise(noise.tables, P * 2.0 ** k)
    expect = 0.5 + 0.4 * n
    err = np.abs(img[..., 1] - expect)
    # within the sky estimate's noise (and the noise's change across a pixel)
    assert (err <= 4 * np.sqrt(var[..., 1]) + 0.01).mean() > 0.99 and np.ptp(expect) > 0.1
    assert np.corrcoef(img[..., 1].ravel(), expect.ravel())[0, 1] > 0.95


def test_perlin_tables_are_the_references_for_the_seed():
    """pcg32_k2_fast and std::shuffle as restated in textures.py against the vectors of
    tests/golden/make_perlin_golden.py (pcg-cpp's generator and libstdc++'s std::shuffle, compiled):
    the generator's first outputs, the three lattice tables of Perlin(seed) (perlin.cpp:137-152),
    and shuffles of both parities."""
    import json
    from pathlib import Path
    gold = json.loads((Path(__file__).resolve().parent / "golden" / "perlin_tables.json").read_text())
    for seed, v in gold["seeds"].items():
        g = tx.Pcg32K2Fast(int(seed))
        assert [g() for _ in range(20)] == v["outputs"]
        t = tx.Perlin(int(seed)).tables
        assert (t[:, :256] == np.asarray(v["tables"])).all()
        assert (t[:, 256] == t[:, 0]).all()
        for n, ref in v["shuffles"].items():
            vals = list(range(int(n)))
            tx.std_shuffle(vals, tx.Pcg32K2Fast(int(seed)))
            assert vals == ref


def test_pcg_extension_table_advances_like_an_inside_out_generator():
    """The table step (taken when the state's low 32 bits are zero) inverts the RXS M XS output,
    steps the 32-bit LCG with increment + 2(i + 1) and outputs again."""
    g = tx.Pcg32K2Fast(0)
    for v in (0, 1, 0xDEADBEEF, 0xFFFFFFFF):
        assert tx._rxs_m_xs_32_inverse(tx._rxs_m_xs_32(v)) == v
    before = list(g.table)
    g._advance_table()
    st = (tx._rxs_m_xs_32_inverse(before[0]) * tx._PCG_MUL32 + tx._PCG_INC32 + 2) & 0xFFFFFFFF
    assert g.table[0] == tx._rxs_m_xs_32(st)


def test_mip_levels_follow_the_references_construction():
    """Image::makeMipMaps (image.cpp:365-560): even sizes average pairs; odd sizes 2n+1 weigh three
    neighbours by (n - k, n, k + 1) / (2n + 1), except that the vectorised build (the reference's
    default) multiplies the middle pixel along x by itself; anisotropic tables halve y per row and x
    per column, isotropic levels halve both."""
    rng = np.random.default_rng(4)
    img = rng.uniform(0.1, 0.9, size=(6, 5, 4)).astype(np.float32)
    nu, nv, lv = tx.mip_levels(img, "anisotropic")
    assert (nu, nv, len(lv)) == (3, 3, 9)
    assert [x.shape[:2] for x in lv[:3]] == [(6, 5), (6, 2), (6, 1)]
    assert [x.shape[:2] for x in lv[3::3]] == [(3, 5), (1, 5)]
    # x: 5 -> 2 (odd): w0 = (2 - k) / 5, middle squared, w2 = (k + 1) / 5
    w = np.float32(1) / np.float32(5)
    k0 = (w * np.float32(2)) * img[:, 0] + img[:, 1] * img[:, 1] + (w * np.float32(1)) * img[:, 2]
    np.testing.assert_allclose(lv[1][:, 0], k0, rtol=1e-6)
    # y: 6 -> 3 (even): pairs averaged
    np.testing.assert_allclose(lv[3][1], (img[2] + img[3]) * np.float32(0.5), rtol=1e-6)
    # y: 3 -> 1 (odd): the middle row weighed by 1/3
    w3 = np.float32(1) / np.float32(3)
    np.testing.assert_allclose(lv[6][0], (w3 * lv[3][0] + w3 * lv[3][1]) + w3 * lv[3][2], rtol=1e-6)
    nu, nv, lv = tx.mip_levels(img, "isotropic")
    assert (nu, nv) == (3, 1) and [x.shape[:2] for x in lv] == [(6, 5), (3, 2), (1, 1)]
    assert tx.mip_levels(img, "none")[:2] == (1, 1)


def test_oracle_checker_board_anti_aliasing_averages_the_footprint():
    """A board of many checkers per pixel: with bilinear anti-aliasing each camera hit sees the
    share of A over its footprint (CheckerBoard::integrate), so the pixels are near the average of
    A and B and vary far less than with point lookups ("none")."""
    res = {}
    for aa in ("none", "bilinear"):
        board = tx.CheckerBoard(0.9, 0.1)
        board.antiAliasing = aa
        tex = tx.TransformationUv(board, [[200, 0, 0], [0, 200, 0], [0, 0, 1]])
        scene, cam = _board_scene(tex)
        t = tracers.DirectLighting()
        t.maxRayGeneration = 1
        img, _ = R.resolve(oracle.RenderScene(R.flatten(scene)).render(R.render_desc(cam, 24, 24, 16, t, seed=5)))
        res[aa] = img[..., 1]
    assert abs(res["bilinear"].mean() - 0.5) < 0.05
    assert res["bilinear"].std() < 0.5 * res["none"].std()


def test_oracle_fbm_octaves_follow_the_footprint():
    """FBm keeps every octave where the footprint is zero (past the camera vertex) and fewer at a
    camera hit whose footprint is wide: the camera image of a distant FBm plane is smoother than
    the same texture looked up without a footprint."""
    from liar_b200 import cameras
    plane = scenery.Parallelogram((-50, 0, -50), (100, 0, 0), (0, 0, 100))
    plane.shader = shaders.Lambert(tx.Sum(tx.Product(tx.FBm(8, 0.5), 0.3), 0.5))
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 30, -40)
    cam.sky = (0, 1, 0)
    cam.lookAt((0, 0, 0))
    scene = scenery.List([plane, scenery.LightSky(tx.Constant(1.0))])
    flat = R.flatten(scene)
    t = tracers.DirectLighting()
    t.maxRayGeneration = 1
    img, _ = R.resolve(oracle.RenderScene(flat).render(R.render_desc(cam, 32, 32, 1, t, seed=2)))
    assert np.isfinite(img).all() and img[..., 1].mean() > 0.1
