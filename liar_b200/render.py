"""Flattening of the scene graph into the renderer's C ABI (include/liar_gpu.h) and the render call.

RenderEngine (kernel.py) uses this to hand the whole scene to the GPU in one upload: every
geometric object becomes triangles of one soup tagged with an object index; shaders become
material records, spectra become spectrum records (their tables in one float pool), lights become
light records with the total power that drives light selection (kernel/light_context.cpp:272-333).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from . import _tables, mediums, scenery, shaders, spectra
from . import textures as tx
from .textures import as_scalar, as_spectrum

# ---- C structs (mirrors of include/liar_gpu.h)


class CSpectrum(C.Structure):
    _fields_ = [("type", C.c_int32), ("offset", C.c_int32), ("count", C.c_int32), ("p", C.c_float * 3)]


class CMaterial(C.Structure):
    _fields_ = [("type", C.c_int32), ("mdf", C.c_int32), ("spec", C.c_int32 * 4), ("emission", C.c_int32),
                ("rough_u", C.c_float), ("rough_v", C.c_float), ("samples", C.c_int32), ("tex", C.c_int32 * 4)]


class CTexture(C.Structure):
    _fields_ = [("type", C.c_int32), ("a", C.c_int32), ("b", C.c_int32), ("spectrum", C.c_int32), ("p", C.c_float * 6),
                ("pixels", C.c_int64)]


class CLight(C.Structure):
    _fields_ = [("type", C.c_int32), ("spectrum", C.c_int32), ("object", C.c_int32), ("double_sided", C.c_int32),
                ("first_tri", C.c_int32), ("n_tris", C.c_int32), ("pos", C.c_float * 3), ("u", C.c_float * 3),
                ("v", C.c_float * 3), ("power", C.c_float), ("emission_samples", C.c_int32)]


_P = C.c_void_p
_S = C.c_size_t


class CSceneDesc(C.Structure):
    _fields_ = [("vertices", _P), ("n_vertices", _S), ("triangles", _P), ("n_triangles", _S),
                ("triangle_object", _P), ("normals", _P), ("n_normals", _S), ("triangle_normals", _P),
                ("object_material", _P), ("object_light", _P), ("n_objects", _S),
                ("materials", _P), ("n_materials", _S), ("spectra", _P), ("n_spectra", _S),
                ("spectrum_pool", _P), ("pool_size", _S), ("lights", _P), ("n_lights", _S),
                ("observer", _P), ("n_observer", _S), ("scene_radius", C.c_float),
                ("textures", _P), ("n_textures", _S), ("triangle_uvs", _P),
                ("texture_pixels", _P), ("n_texture_pixels", _S), ("noise_tables", _P), ("n_noise_tables", _S),
                ("spheres", _P), ("n_spheres", _S), ("sphere_object", _P)]


class CCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("direction", C.c_float * 3), ("right", C.c_float * 3),
                ("down", C.c_float * 3), ("direction_normal", C.c_float * 3), ("right_normal", C.c_float * 3),
                ("down_normal", C.c_float * 3), ("lens_radius", C.c_float), ("focus_distance", C.c_float),
                ("near_limit", C.c_float), ("far_limit", C.c_float)]


class CPhotonMapperDesc(C.Structure):
    _fields_ = [("max_photons", C.c_uint64), ("global_map_size", C.c_uint64),
                ("estimation_radius", C.c_float * 2), ("estimation_tolerance", C.c_float * 2),
                ("estimation_size", C.c_int32 * 2), ("ray_trace_direct", C.c_int32), ("visualize", C.c_int32),
                ("final_gather_rays", C.c_int32), ("secondary_gather_rays", C.c_int32),
                ("ratio_precomputed_irradiance", C.c_float), ("caustics_quality", C.c_float)]


class CRenderDesc(C.Structure):
    _fields_ = [("camera", CCamera), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("tracer", C.c_int32), ("max_ray_generation", C.c_int32), ("max_depth", C.c_int32),
                ("seed", C.c_uint64), ("first_sample", C.c_int32), ("wave_paths", C.c_int32),
                ("secondary_light_samples", C.c_int32), ("trace_glossy", C.c_int32),
                ("filter", C.c_int32), ("filter_param", C.c_float), ("max_sample_luminance", C.c_float),
                ("photon_mapper", CPhotonMapperDesc), ("sampler", C.c_int32)]


FILTER_BOX, FILTER_TRIANGLE, FILTER_MITCHELL = 0, 1, 2


TEX_CONSTANT, TEX_CHECKER, TEX_GRID, TEX_UV_TRANSFORM, TEX_IMAGE, TEX_NOISE, TEX_ABS, TEX_AFFINE = range(8)
SPEC_CONSTANT, SPEC_SAMPLED, SPEC_BLACKBODY, SPEC_CAUCHY = 0, 1, 2, 3
MAT_NONE, MAT_LAMBERT, MAT_CONDUCTOR, MAT_COOK_TORRANCE, MAT_DIELECTRIC, MAT_WALTER, MAT_MIRROR = range(7)
LIGHT_PARA, LIGHT_MESH, LIGHT_POINT, LIGHT_SKY = 0, 1, 2, 3


@dataclass
class FlatScene:
    vertices: np.ndarray
    triangles: np.ndarray
    triangle_object: np.ndarray
    normals: np.ndarray | None
    triangle_normals: np.ndarray | None
    object_material: np.ndarray
    object_light: np.ndarray
    materials: C.Array
    spectra: C.Array
    pool: np.ndarray
    lights: C.Array
    observer: np.ndarray
    scene_radius: float
    textures: C.Array | None = None
    triangle_uvs: np.ndarray | None = None  # n_triangles x 3 x 2, when a texture needs them
    texture_pixels: np.ndarray | None = None  # image textures' pixels, n x 4 (X, Y, Z, 0)
    noise_tables: np.ndarray | None = None    # noise textures' permutation tables, bytes
    spheres: np.ndarray | None = None         # analytic spheres, n x 4 (centre, radius)
    sphere_object: np.ndarray | None = None
    keep: list = field(default_factory=list)

    def desc(self) -> CSceneDesc:
        d = CSceneDesc()
        if self.triangles.shape[0]:
            d.vertices = self.vertices.ctypes.data
            d.n_vertices = self.vertices.shape[0]
            d.triangles = self.triangles.ctypes.data
            d.n_triangles = self.triangles.shape[0]
            d.triangle_object = self.triangle_object.ctypes.data
        if self.normals is not None and self.triangle_normals is not None:
            d.normals = self.normals.ctypes.data
            d.n_normals = self.normals.shape[0]
            d.triangle_normals = self.triangle_normals.ctypes.data
        d.object_material = self.object_material.ctypes.data
        d.object_light = self.object_light.ctypes.data
        d.n_objects = self.object_material.shape[0]
        d.materials = C.addressof(self.materials) if len(self.materials) else None
        d.n_materials = len(self.materials)
        d.spectra = C.addressof(self.spectra) if len(self.spectra) else None
        d.n_spectra = len(self.spectra)
        d.spectrum_pool = self.pool.ctypes.data if self.pool.size else None
        d.pool_size = self.pool.size
        d.lights = C.addressof(self.lights) if len(self.lights) else None
        d.n_lights = len(self.lights)
        d.observer = self.observer.ctypes.data
        d.n_observer = self.observer.shape[0]
        d.scene_radius = self.scene_radius
        if self.textures is not None and len(self.textures):
            d.textures = C.addressof(self.textures)
            d.n_textures = len(self.textures)
        if self.triangle_uvs is not None:
            d.triangle_uvs = self.triangle_uvs.ctypes.data
        if self.texture_pixels is not None:
            d.texture_pixels = self.texture_pixels.ctypes.data
            d.n_texture_pixels = self.texture_pixels.shape[0]
        if self.noise_tables is not None:
            d.noise_tables = self.noise_tables.ctypes.data
            d.n_noise_tables = self.noise_tables.size
        if self.spheres is not None and len(self.spheres):
            d.spheres = self.spheres.ctypes.data
            d.n_spheres = self.spheres.shape[0]
            d.sphere_object = self.sphere_object.ctypes.data
        return d


class _Builder:
    def __init__(self):
        self.verts, self.tris, self.tri_obj, self.norms, self.tri_norms = [], [], [], [], []
        self.n_verts = self.n_tris = self.n_norms = 0
        self.has_normals = False
        self.obj_mat, self.obj_light = [], []
        self.materials, self.mat_ids = [], {}
        self.spectra, self.spec_ids, self.pool = [], {}, []
        self.lights = []
        self.textures, self.tex_ids = [], {}
        self.tex_pixels, self.n_tex_pixels = [], 0
        self.noise_tables, self.n_noise = [], 0
        self.tri_uvs = []  # per object: n x 3 x 2 corner uvs, or None for the barycentric ones
        self.spheres, self.sphere_obj = [], []
        self.M = None  # current local-to-world affine matrix (None: identity)

    # -- transformations (scenery/transformation.cpp, translation.cpp)
    def point(self, p) -> np.ndarray:
        p = np.asarray(p, dtype=np.float64)
        return p if self.M is None else p @ self.M[:3, :3].T + self.M[:3, 3]

    def vector(self, v) -> np.ndarray:
        v = np.asarray(v, dtype=np.float64)
        return v if self.M is None else v @ self.M[:3, :3].T

    # -- spectra
    def spectrum(self, x, reflectant_hint=False) -> int:
        s = as_spectrum(x)
        key = id(s)
        if key in self.spec_ids:
            return self.spec_ids[key][0]
        rec = CSpectrum()
        if isinstance(s, spectra.Sampled):
            rec.type = SPEC_SAMPLED
            rec.offset = len(self.pool)
            rec.count = len(s.wavelengths)
            self.pool.extend(s.wavelengths)
            self.pool.extend(s.values)
        elif isinstance(s, spectra.Xyz):
            # the recovered spectrum at the recovery's wavelengths, with the recovery's bound for
            # the reflectance rescale (RecoveryMengSimon::doRecover, Single mode)
            from .recovery import standard
            ws, vs, mx = standard().sampled(s.xyz)
            rec.type = SPEC_SAMPLED
            rec.offset = len(self.pool)
            rec.count = len(ws)
            rec.p[0] = mx
            self.pool.extend(float(w) for w in ws)
            self.pool.extend(float(v) for v in vs)
        elif isinstance(s, spectra.BlackBody):
            rec.type = SPEC_BLACKBODY
            rec.p[0], rec.p[1] = s.temperature, s.scale
        elif isinstance(s, spectra.Cauchy):
            rec.type = SPEC_CAUCHY
            rec.p[0], rec.p[1] = s.a, s.b
        elif type(s) is spectra.Spectrum:
            rec.type = SPEC_CONSTANT
            rec.p[0] = s.value
        else:
            raise TypeError(f"unsupported spectrum {type(s).__name__}")
        idx = len(self.spectra)
        self.spectra.append(rec)
        self.spec_ids[key] = (idx, s)
        return idx

    # -- textures (src/liar/textures/): a tree of nodes per textured material parameter
    def texture(self, t) -> int:
        key = id(t)
        if key in self.tex_ids:
            return self.tex_ids[key][0]
        rec = CTexture()
        rec.a = rec.b = rec.spectrum = -1
        if isinstance(t, tx.CheckerBoard):
            rec.type = TEX_CHECKER
            rec.p[0], rec.p[1] = t.split
            rec.p[2] = 1.0 if t.antiAliasing == tx.CheckerBoard.AA_BILINEAR else 0.0
        elif isinstance(t, tx.GridBoard):
            rec.type = TEX_GRID
            rec.p[0], rec.p[1] = t.thickness[0] / 2, t.thickness[1] / 2  # GridBoard's halfThickness
        elif isinstance(t, tx.Image):
            if t.xyz is None:
                raise ValueError("Image texture has no pixels (loadFile first)")
            h, w = t.xyz.shape[:2]
            rec.type = TEX_IMAGE
            rec.a, rec.b = w, h
            rec.p[0] = {"none": 0.0, "bilinear": 1.0, "trilinear": 2.0}[t.antiAliasing]
            rec.pixels = self.n_tex_pixels
            block = tx.image_pool_block(t)
            self.tex_pixels.append(block)
            self.n_tex_pixels += block.shape[0]
        elif isinstance(t, tx.Perlin):
            rec.type = TEX_NOISE
            rec.p[0] = float(t.numOctaves) if isinstance(t, tx.FBm) else 0.0
            rec.p[1] = float(t.falloff) if isinstance(t, tx.FBm) else 0.0
            rec.pixels = self.n_noise
            self.noise_tables.append(t.tables.reshape(-1))
            self.n_noise += t.tables.size
        elif isinstance(t, tx.Abs):
            rec.type = TEX_ABS
        elif isinstance(t, (tx.Product, tx.Sum)):
            parts = t.factors if isinstance(t, tx.Product) else t.terms
            varying = [f for f in parts if tx.flat_value(f) is None]
            consts = [tx.flat_value(f) for f in parts if tx.flat_value(f) is not None]
            if len(varying) > 1:
                raise NotImplementedError(f"{type(t).__name__} of more than one non-constant texture is not on the GPU path")
            if not varying:
                raise NotImplementedError(f"a {type(t).__name__} of constants: use a Constant")
            rec.type = TEX_AFFINE
            if isinstance(t, tx.Product):
                rec.p[0], rec.p[1] = float(np.prod(consts)) if consts else 1.0, 0.0
            else:
                rec.p[0], rec.p[1] = 1.0, float(np.sum(consts)) if consts else 0.0
        elif isinstance(t, tx.TransformationUv):
            rec.type = TEX_UV_TRANSFORM
            m = t.transformation
            rec.p[:] = [float(m[0, 0]), float(m[0, 1]), float(m[0, 2]), float(m[1, 0]), float(m[1, 1]), float(m[1, 2])]
        else:
            rec.type = TEX_CONSTANT
            rec.spectrum = self.spectrum(t)
        idx = len(self.textures)
        self.textures.append(rec)
        self.tex_ids[key] = (idx, t)
        if isinstance(t, tx.BinaryOperator):
            self.textures[idx].a = self.texture(t.textureA)
            self.textures[idx].b = self.texture(t.textureB)
        elif isinstance(t, tx.UnaryOperator):
            self.textures[idx].a = self.texture(t.texture)
        elif isinstance(t, (tx.Product, tx.Sum)):
            parts = t.factors if isinstance(t, tx.Product) else t.terms
            self.textures[idx].a = self.texture(next(f for f in parts if tx.flat_value(f) is None))
        return idx

    def param(self, m, k: int, value):
        """Material parameter k: a uv texture as a texture tree, else a constant spectrum."""
        if tx.is_uv_texture(value):
            m.tex[k] = self.texture(value)
        else:
            m.spec[k] = self.spectrum(value)

    # -- shaders
    def material(self, shader) -> int:
        if shader is None:
            return -1
        key = id(shader)
        if key in self.mat_ids:
            return self.mat_ids[key][0]
        m = CMaterial()
        m.spec[:] = [-1, -1, -1, -1]
        m.tex[:] = [-1, -1, -1, -1]
        m.emission = -1
        m.samples = 1
        bsdf = shader
        if isinstance(shader, shaders.Sum):
            emitters = [c for c in shader.children if isinstance(c, shaders.Unshaded)]
            others = [c for c in shader.children if not isinstance(c, shaders.Unshaded)]
            if len(emitters) > 1 or len(others) > 1:
                raise NotImplementedError("Sum supports one BSDF and one Unshaded component on the GPU")
            if emitters:
                m.emission = self.spectrum(emitters[0].colour)
            bsdf = others[0] if others else None
        if isinstance(bsdf, shaders.Unshaded):
            m.emission = self.spectrum(bsdf.colour)
            bsdf = None
        if bsdf is None:
            m.type = MAT_NONE
        elif isinstance(bsdf, shaders.Lambert):
            m.type = MAT_LAMBERT
            self.param(m, 0, bsdf.diffuse)
        elif isinstance(bsdf, shaders.Mirror):
            m.type = MAT_MIRROR
            self.param(m, 0, bsdf.reflectance)
        elif isinstance(bsdf, (shaders.Conductor, shaders.CookTorrance)):
            m.type = MAT_CONDUCTOR if isinstance(bsdf, shaders.Conductor) else MAT_COOK_TORRANCE
            self.param(m, 0, bsdf.refractionIndex)
            self.param(m, 1, bsdf.absorptionCoefficient)
            self.param(m, 2, bsdf.reflectance)
            if isinstance(bsdf, shaders.CookTorrance):
                m.samples = int(getattr(bsdf, "numberOfSamples", 1))
                m.rough_u = as_scalar(bsdf.roughnessU)
                m.rough_v = as_scalar(bsdf.roughnessV)
                m.mdf = bsdf.mdf.kind
        elif isinstance(bsdf, shaders.Dielectric):
            m.type = MAT_WALTER if isinstance(bsdf, shaders.Walter) else MAT_DIELECTRIC
            self.param(m, 0, bsdf.innerRefractionIndex)
            self.param(m, 1, bsdf.outerRefractionIndex)
            self.param(m, 2, bsdf.reflectance)
            self.param(m, 3, bsdf.transmittance)
            if isinstance(bsdf, shaders.Walter):
                m.samples = int(getattr(bsdf, "numberOfSamples", 1))
                m.rough_u = as_scalar(bsdf.roughnessU)
                m.rough_v = as_scalar(bsdf.roughnessV)
                m.mdf = bsdf.mdf.kind
        else:
            raise NotImplementedError(f"shader {type(bsdf).__name__} is not on the GPU path")
        idx = len(self.materials)
        self.materials.append(m)
        self.mat_ids[key] = (idx, shader)
        return idx

    # -- geometry
    def geometry(self, obj, shader, light: int) -> tuple[int, int]:
        v, t, n, tn = obj.triangles()
        uv = obj.corner_uvs() if hasattr(obj, "corner_uvs") else None
        if self.M is not None:
            v = self.point(v).astype(np.float32)
            if n is not None:
                nn = np.asarray(n, dtype=np.float64) @ np.linalg.inv(self.M[:3, :3])  # inverse transpose
                n = (nn / np.maximum(np.linalg.norm(nn, axis=1, keepdims=True), 1e-300)).astype(np.float32)
            if np.linalg.det(self.M[:3, :3]) < 0:
                # a mirroring transformation: keep the geometric normal the transformed local one,
                # as the reference transforms the local context's normal
                t = np.asarray(t)[:, [0, 2, 1]]
                if uv is not None:
                    uv = np.asarray(uv)[:, [0, 2, 1]]
                if tn is not None:
                    tn = np.asarray(tn)[:, [0, 2, 1]]
        obj_index = len(self.obj_mat)
        self.obj_mat.append(self.material(shader))
        self.obj_light.append(light)
        first = self.n_tris
        self.verts.append(np.asarray(v, dtype=np.float32))
        self.tris.append(np.asarray(t, dtype=np.int64) + self.n_verts)
        self.tri_obj.append(np.full(len(t), obj_index, dtype=np.int32))
        self.tri_uvs.append(None if uv is None else np.asarray(uv, dtype=np.float32).reshape(len(t), 3, 2))
        if n is not None and tn is not None:
            self.has_normals = True
            self.norms.append(np.asarray(n, dtype=np.float32))
            self.tri_norms.append(np.where(tn >= 0, tn + self.n_norms, -1).astype(np.int32))
            self.n_norms += len(n)
        else:
            self.tri_norms.append(np.full((len(t), 3), -1, dtype=np.int32))
        self.n_verts += len(v)
        self.n_tris += len(t)
        return first, len(t)

    def visit(self, obj, inherited=None):
        if not mediums.is_vacuum(getattr(obj, "interior", None)):
            raise NotImplementedError(f"{type(obj).__name__}.interior is a {type(obj.interior).__name__}: "
                                      "participating media are not on the GPU path")
        if isinstance(obj, scenery.List):
            for c in obj.children:
                self.visit(c, obj.shader or inherited)
        elif isinstance(obj, (scenery.Transformation, scenery.Translation)):
            saved = self.M
            local = obj.matrix()
            self.M = local if saved is None else saved @ local
            try:
                self.visit(obj.child, obj.shader or inherited)
            finally:
                self.M = saved
        elif isinstance(obj, scenery.LightArea):
            surf = obj.surface
            li = len(self.lights)
            L = CLight()
            L.spectrum = self.spectrum(obj.radiance)
            L.double_sided = int(bool(obj.isDoubleSided))
            L.emission_samples = int(obj.numberOfEmissionSamples)
            first, count = self.geometry(surf, obj.shader or surf.shader or inherited, li)
            L.object = len(self.obj_mat) - 1
            if isinstance(surf, scenery.Parallelogram):
                L.type = LIGHT_PARA
                pos, u, v = self.point(surf.support), self.vector(surf.sizeU), self.vector(surf.sizeV)
                if self.M is not None and np.linalg.det(self.M[:3, :3]) < 0:
                    u, v = v, u  # the same surface, facing like its (re-wound) triangles
                L.pos[:], L.u[:], L.v[:] = (tuple(float(x) for x in a) for a in (pos, u, v))
                area = float(np.linalg.norm(np.cross(u, v)))
            else:
                L.type = LIGHT_MESH
                L.first_tri, L.n_tris = first, count
                v = self.verts[-1].astype(np.float64)
                t = self.tris[-1] - (self.n_verts - len(self.verts[-1]))
                area = float(0.5 * np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1).sum())
            # LightArea::doTotalPower (light_area.cpp:290-294)
            L.power = math.pi * area * as_spectrum(obj.radiance).luminance * (2 if obj.isDoubleSided else 1)
            self.lights.append(L)
        elif isinstance(obj, scenery.LightPoint):
            L = CLight()
            L.type = LIGHT_POINT
            L.object = -1
            L.emission_samples = int(obj.numberOfEmissionSamples)
            L.spectrum = self.spectrum(obj.intensity)
            L.pos[:] = tuple(float(x) for x in self.point(obj.position))
            L.power = 4 * math.pi * as_spectrum(obj.intensity).luminance  # LightPoint::doTotalPower
            self.lights.append(L)
        elif isinstance(obj, scenery.LightSky):
            L = CLight()
            L.type = LIGHT_SKY
            L.object = -1
            L.emission_samples = int(obj.numberOfEmissionSamples)
            L.spectrum = self.spectrum(obj.radiance)
            self.lights.append(L)
        elif isinstance(obj, scenery.Sphere) and obj.analytic and self.similarity() is not None:
            # an analytic sphere: centre and radius through the similarity (uniform scale)
            scale = self.similarity()
            obj_index = len(self.obj_mat)
            self.obj_mat.append(self.material(obj.shader or inherited))
            self.obj_light.append(-1)
            c = self.point(obj.center)
            self.spheres.append((float(c[0]), float(c[1]), float(c[2]), obj.radius * scale))
            self.sphere_obj.append(obj_index)
        elif hasattr(obj, "triangles"):
            self.geometry(obj, obj.shader or inherited, -1)
        else:
            raise NotImplementedError(f"scene object {type(obj).__name__} is not on the GPU path")

    def similarity(self) -> float | None:
        """The uniform scale of the current transformation when it is a similarity (rotation or
        mirror times a uniform scale, plus a translation), else None."""
        if self.M is None:
            return 1.0
        A = self.M[:3, :3]
        G = A.T @ A
        s2 = G[0, 0]
        if s2 <= 0 or not np.allclose(G, s2 * np.eye(3), rtol=1e-9, atol=1e-12 * s2):
            return None
        return float(np.sqrt(s2))

    def finish(self) -> FlatScene:
        if not self.verts and not self.spheres:
            raise ValueError("the scene has no geometry")
        V = np.ascontiguousarray(np.concatenate(self.verts), dtype=np.float32) if self.verts else np.zeros((0, 3), np.float32)
        T = np.ascontiguousarray(np.concatenate(self.tris), dtype=np.uint32) if self.tris else np.zeros((0, 3), np.uint32)
        SP = np.asarray(self.spheres, dtype=np.float32).reshape(-1, 4)
        ext = [V] + ([SP[:, :3] - SP[:, 3:], SP[:, :3] + SP[:, 3:]] if len(SP) else [])
        E = np.concatenate([e for e in ext if len(e)])
        lo, hi = E.min(axis=0).astype(np.float64), E.max(axis=0).astype(np.float64)
        radius = float(0.5 * np.linalg.norm(hi - lo))
        for L in self.lights:
            if L.type == LIGHT_SKY:
                # power of a constant sky: pi * radiance * the area of the scene's bounding sphere
                L.power = math.pi * 4 * math.pi * radius ** 2 * self.spec_ids_lum(L.spectrum)
        return FlatScene(
            vertices=V, triangles=T,
            triangle_object=np.ascontiguousarray(np.concatenate(self.tri_obj), dtype=np.int32) if self.tri_obj else np.zeros(0, np.int32),
            normals=np.ascontiguousarray(np.concatenate(self.norms), dtype=np.float32) if self.has_normals else None,
            triangle_normals=np.ascontiguousarray(np.concatenate(self.tri_norms), dtype=np.int32) if self.has_normals else None,
            object_material=np.asarray(self.obj_mat, dtype=np.int32),
            object_light=np.asarray(self.obj_light, dtype=np.int32),
            materials=(CMaterial * len(self.materials))(*self.materials),
            spectra=(CSpectrum * len(self.spectra))(*self.spectra),
            pool=np.asarray(self.pool, dtype=np.float32),
            lights=(CLight * len(self.lights))(*self.lights),
            observer=np.ascontiguousarray(_tables.observer(), dtype=np.float32),
            scene_radius=radius,
            textures=(CTexture * len(self.textures))(*self.textures) if self.textures else None,
            triangle_uvs=self.triangle_uvs(),
            texture_pixels=np.ascontiguousarray(np.concatenate(self.tex_pixels)) if self.tex_pixels else None,
            noise_tables=np.ascontiguousarray(np.concatenate(self.noise_tables)) if self.noise_tables else None,
            spheres=np.ascontiguousarray(SP) if len(SP) else None,
            sphere_object=np.asarray(self.sphere_obj, dtype=np.int32) if len(SP) else None,
        )

    def triangle_uvs(self) -> np.ndarray | None:
        """Corner uvs of every triangle when a texture reads them and an object has its own; the
        others keep the barycentric ones (corners (0, 0), (1, 0), (0, 1))."""
        if not self.textures or all(u is None for u in self.tri_uvs):
            return None
        bary = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float32)
        parts = [u if u is not None else np.broadcast_to(bary, (len(o), 3, 2))
                 for u, o in zip(self.tri_uvs, self.tri_obj)]
        return np.ascontiguousarray(np.concatenate(parts).reshape(-1, 6), dtype=np.float32)

    def spec_ids_lum(self, idx: int) -> float:
        for i, s in self.spec_ids.values():
            if i == idx:
                return s.luminance
        return 1.0


def flatten(scene) -> FlatScene:
    b = _Builder()
    b.visit(scene)
    return b.finish()


def render_desc(camera, width: int, height: int, spp: int, tracer, seed: int = 0, first_sample: int = 0,
                wave_paths: int = 0, filter: int = FILTER_BOX, filter_param: float = 0.0,
                max_sample_luminance: float = 0.0, sampler: int = 0) -> CRenderDesc:
    """The C render description. filter / filter_param select the reconstruction filter (box;
    triangle of the given width, default 1; Mitchell with the given B, default 1/3);
    max_sample_luminance > 0 clamps each sample's Y (Raster.maxSampleLuminance); sampler holds
    the LIAR_SAMPLER_* bits of the sampler (samplers.Stratifier.mode)."""
    r = CRenderDesc()
    cam = camera.flatten()
    for k in ("position", "direction", "right", "down", "direction_normal", "right_normal", "down_normal"):
        getattr(r.camera, k)[:] = cam[k]
    r.camera.lens_radius = cam["lens_radius"]
    r.camera.focus_distance = min(cam["focus_distance"], 3.4028234663852886e38)
    r.camera.near_limit = cam["near_limit"]
    r.camera.far_limit = min(cam["far_limit"], 3.4028234663852886e38)
    r.width, r.height, r.spp = int(width), int(height), int(spp)
    r.tracer = getattr(tracer, "kind", 0)
    r.max_ray_generation = int(tracer.maxRayGeneration)
    r.max_depth = int(getattr(tracer, "maxDepth", 0))
    r.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    r.first_sample = int(first_sample)
    r.wave_paths = int(wave_paths)
    r.secondary_light_samples = int(getattr(tracer, "numberOfSecondaryLightSamples", 1))
    r.trace_glossy = 1 if getattr(tracer, "traceGlossy", True) else -1
    if r.tracer == 2:
        pm = r.photon_mapper
        q = max(float(getattr(tracer, "causticsQuality", 1.0)), 0.0)   # setCausticsQuality clamps at 0
        pm.caustics_quality = q if q > 0.0 else -1.0
        pm.max_photons = int(tracer.maxNumberOfPhotons)
        pm.global_map_size = int(tracer.globalMapSize)
        for m in range(2):
            pm.estimation_radius[m] = float(tracer._radius[m])
            pm.estimation_tolerance[m] = float(tracer._tolerance[m])
            pm.estimation_size[m] = int(tracer._size[m])
        pm.ray_trace_direct = 1 if tracer.isRayTracingDirect else -1
        pm.visualize = 1 if tracer.isVisualizingPhotonMap else 0
        pm.final_gather_rays = int(tracer.numFinalGatherRays)
        pm.secondary_gather_rays = int(tracer.numSecondaryGatherRays) or -1
        ratio = float(tracer.ratioPrecomputedIrradiance)
        pm.ratio_precomputed_irradiance = ratio if ratio > 0 else -1.0
    r.filter = int(filter)
    r.filter_param = float(filter_param)
    r.max_sample_luminance = float(max_sample_luminance) if math.isfinite(max_sample_luminance) else 0.0
    r.sampler = int(sampler)
    return r


def resolve(film: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(H, W, 8) sums -> mean XYZ + alpha (H, W, 4) and variance of the mean of XYZ (H, W, 3).

    The mean is the reference's pixel (Raster::weighted, output/raster.cpp:645-651): the weighted
    sums over the sum of the filter weights (the sample count for the box filter), zero where no
    weight arrived. The variance is the sample variance of the mean for the box filter and an
    estimate of it with the filter weights otherwise."""
    w = film[..., 7:8].astype(np.float64)
    ok = w > 0
    n = np.where(ok, w, 1.0)
    mean = np.where(ok, film[..., 0:4].astype(np.float64) / n, 0.0)
    ex2 = np.where(ok, film[..., 4:7].astype(np.float64) / n, 0.0)
    var = np.maximum(ex2 - mean[..., 0:3] ** 2, 0.0) / np.maximum(n - 1, 1)
    return mean, var


# ---- GPU scene handle


_RENDER_SIGS = {
    "liar_gpu_scene_upload": (C.c_int, [C.c_void_p, C.POINTER(CSceneDesc), C.POINTER(C.c_void_p)]),
    "liar_gpu_scene_destroy": (None, [C.c_void_p]),
    "liar_gpu_render": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(CRenderDesc), C.c_void_p]),
    "liar_gpu_render_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(CRenderDesc), C.c_void_p, C.c_void_p]),
    "liar_gpu_render_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong)]),
}


class GpuScene:
    """A flattened scene resident on the device (liar_gpu_scene_upload)."""

    def __init__(self, ctx, flat: FlatScene):
        self.ctx = ctx
        self.flat = flat
        lib = ctx._lib
        for name, (res, args) in _RENDER_SIGS.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        from .recovery import set_standard_on
        set_standard_on(ctx)  # Spectral::fromXYZ of image textures and of the PhotonMapper's photons
        h = C.c_void_p()
        d = flat.desc()
        ctx.check(lib.liar_gpu_scene_upload(ctx.handle, C.byref(d), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.liar_gpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, desc: CRenderDesc, film: np.ndarray | None = None) -> np.ndarray:
        """Adds desc.spp samples per pixel to film ((H, W, 8) float32 sums); returns film."""
        if film is None:
            film = np.zeros((desc.height, desc.width, 8), dtype=np.float32)
        assert film.dtype == np.float32 and film.flags.c_contiguous and film.shape == (desc.height, desc.width, 8)
        self.ctx.check(self.ctx._lib.liar_gpu_render(self.ctx.handle, self.handle, C.byref(desc), film.ctypes.data))
        return film

    def render_device(self, desc: CRenderDesc, film_ptr: int, stream: int | None = None) -> None:
        self.ctx.check(self.ctx._lib.liar_gpu_render_device(self.ctx.handle, self.handle, C.byref(desc),
                                                            C.c_void_p(film_ptr), C.c_void_p(stream or 0)))

    def stats(self) -> dict:
        out = (C.c_ulonglong * 3)()
        self.ctx.check(self.ctx._lib.liar_gpu_render_stats(self.ctx.handle, out))
        return {"paths": out[0], "segments": out[1], "hits": out[2]}


# ---- PhotonMapper maps (liar_gpu_photon_mapper_stats / _get_map)

def photon_mapper_stats(ctx) -> dict:
    """The photon maps of the last PhotonMapper render on ctx."""
    out = (C.c_ulonglong * 4)()
    radii = (C.c_float * 2)()
    fn = ctx._lib.liar_gpu_photon_mapper_stats
    fn.restype, fn.argtypes = C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]
    ctx.check(fn(ctx.handle, out, radii))
    return {"emitted": out[0], "global": out[1], "caustic": out[2], "valid": bool(out[3]),
            "radius": (radii[0], radii[1])}


def photon_mapper_map(ctx, m: int) -> dict:
    """Map m (0 global, 1 caustic) of the last PhotonMapper render as host arrays."""
    st = photon_mapper_stats(ctx)
    n = int(st["global"] if m == 0 else st["caustic"])
    a = {k: np.zeros((n, 3), np.float32) for k in ("position", "omega_in", "power", "blend_w")}
    a["blend_idx"] = np.zeros((n, 3), np.int32)
    got = C.c_size_t()
    fn = ctx._lib.liar_gpu_photon_mapper_get_map
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                   C.POINTER(C.c_size_t)]
    ctx.check(fn(ctx.handle, int(m), a["position"].ctypes.data, a["omega_in"].ctypes.data, a["power"].ctypes.data,
                 a["blend_idx"].ctypes.data, a["blend_w"].ctypes.data, n, C.byref(got)))
    a["radius"] = st["radius"][m]
    return a


def photon_mapper_irradiance(ctx) -> dict:
    """The irradiance map of the last PhotonMapper render with final gathering, as host arrays."""
    got = C.c_size_t()
    fn = ctx._lib.liar_gpu_photon_mapper_get_irradiance
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] + [C.c_void_p] * 6 + [C.c_size_t, C.POINTER(C.c_size_t)]
    # the size first (a call with capacity 0 reports it, refusing the copy when there are points)
    rc = fn(ctx.handle, None, None, None, None, None, None, 0, C.byref(got))
    n = int(got.value)
    a = {k: np.zeros((n, 3), np.float32) for k in ("position", "normal", "xyz", "blend_w")}
    a["blend_idx"] = np.zeros((n, 3), np.int32)
    a["r2"] = np.zeros(n, np.float32)
    if n:
        ctx.check(fn(ctx.handle, a["position"].ctypes.data, a["normal"].ctypes.data, a["xyz"].ctypes.data,
                     a["blend_idx"].ctypes.data, a["blend_w"].ctypes.data, a["r2"].ctypes.data, n, C.byref(got)))
    elif rc:
        ctx.check(rc)  # no maps at all
    return a
