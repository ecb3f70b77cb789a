"""CPU oracle of the hot path -- TEST INFRASTRUCTURE ONLY.

A plain C++ restatement of the reference's arithmetic (liboracle.so, built by oracle/build.py),
used by tests/, by ``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg as the
checker. The product (``liar_b200``) never imports it.

Parity status: the reference's geometry core lives in the Lass library
(lass/1.11.0-250+g078d9309, conanfile.py:39), which is not part of the reference tree and cannot
be built here. The traversal restatement is therefore pinned by construction (the nearest-t rule
with ties to the lower index is tree-independent) and by the brute-force definition, not by
golden vectors of the reference, which ships none for this path. The spectral restatement is
pinned by the known-answer test of test/test_spectrum.cpp:256-278 (tests/golden/).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            from . import build as _b
            _b.build()
        L = C.CDLL(str(path))
        vp, u64 = C.c_void_p, C.c_uint64
        L.oracle_tri_intersect.restype = C.c_int
        L.oracle_tri_intersect.argtypes = [vp] * 8
        L.oracle_trace_bruteforce.restype = C.c_int
        L.oracle_trace_bruteforce.argtypes = [vp, u64, vp, u64, vp, u64, vp, C.c_int, C.c_int]
        L.oracle_tree_build.restype = vp
        L.oracle_tree_build.argtypes = [vp, u64, vp, u64]
        L.oracle_tree_trace.restype = C.c_int
        L.oracle_tree_trace.argtypes = [vp, vp, u64, vp, C.c_int, C.c_int]
        L.oracle_tree_free.restype = None
        L.oracle_tree_free.argtypes = [vp]
        L.oracle_hardware_threads.restype = C.c_int
        _bind_extra(L)
        _LIB = L
    return _LIB


def _bind_extra(L) -> None:
    """Binds the optional restatements (spectra, shading, tracer, photons) when present."""
    from . import _sigs
    for name, (res, args) in _sigs.SIGNATURES.items():
        fn = getattr(L, name, None)
        if fn is not None:
            fn.restype = res
            fn.argtypes = args


def hardware_threads() -> int:
    return int(lib().oracle_hardware_threads())


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def tri_intersect(o, d, a, b, c):
    """Moller-Trumbore on one ray/triangle; returns (t, u, v) or None."""
    o, d, a, b, c = map(_f32, (o, d, a, b, c))
    t, u, v = C.c_float(), C.c_float(), C.c_float()
    hit = lib().oracle_tri_intersect(o.ctypes.data, d.ctypes.data, a.ctypes.data, b.ctypes.data, c.ctypes.data,
                                     C.addressof(t), C.addressof(u), C.addressof(v))
    return (t.value, u.value, v.value) if hit else None


def trace_bruteforce(vertices, triangles, rays, any_hit=False, threads=0):
    V = _f32(vertices).reshape(-1, 3)
    T = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    R = _f32(rays).reshape(-1, 8)
    H = np.empty((R.shape[0], 2), dtype=np.int32)
    lib().oracle_trace_bruteforce(V.ctypes.data, V.shape[0], T.ctypes.data, T.shape[0], R.ctypes.data, R.shape[0],
                                  H.ctypes.data, int(bool(any_hit)), int(threads))
    return H[:, 0].copy(), H[:, 1].view(np.float32).copy()


class RenderScene:
    """The path-tracer restatement (oracle_render.cpp) over a flattened scene. ``flat`` is the
    same ``liar_b200.render.FlatScene`` the GPU receives; it must outlive this object."""

    def __init__(self, flat):
        self.flat = flat
        self._desc = flat.desc()
        L = lib()
        L.oracle_scene_create.restype = C.c_void_p
        L.oracle_scene_create.argtypes = [C.c_void_p]
        L.oracle_scene_free.restype = None
        L.oracle_scene_free.argtypes = [C.c_void_p]
        L.oracle_render.restype = C.c_int
        L.oracle_render.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int]
        self.h = L.oracle_scene_create(C.addressof(self._desc))
        if getattr(flat, "texture_pixels", None) is not None:
            # image textures turn their colours into spectra with the standard recovery
            from liar_b200.recovery import device_table
            t = device_table()
            self._rec = t
            L.oracle_scene_set_recovery.restype = None
            L.oracle_scene_set_recovery.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                                    C.c_void_p, C.c_int]
            L.oracle_scene_set_recovery(self.h, t["wavelengths"].ctypes.data, t["wavelengths"].size,
                                        t["points"].ctypes.data, t["spectra"].ctypes.data, t["spectra"].shape[0],
                                        t["triangles"].ctypes.data, t["triangles"].shape[0])

    def render(self, desc, film=None, pixels=None, threads=0):
        """Adds desc.spp samples of pixels [begin, end) (all by default) to film (H, W, 8)."""
        if film is None:
            film = np.zeros((desc.height, desc.width, 8), dtype=np.float32)
        b, e = pixels if pixels is not None else (0, desc.width * desc.height)
        lib().oracle_render(self.h, C.addressof(desc), film.ctypes.data, int(b), int(e), int(threads))
        return film

    def render_pm(self, desc, maps, recovery_table, film=None, pixels=None, threads=0, irradiance=None):
        """The PhotonMapper restatement with the given maps: ``maps`` is a list of two dicts (global,
        caustic) with position, omega_in, power (n x 3 float32), blend_idx (n x 3 int32), blend_w
        (n x 3 float32), radius and k; ``recovery_table`` is liar_b200.recovery.device_table();
        ``irradiance`` the irradiance map of final gathering (position, normal, blend_idx, blend_w,
        r2) or None. Final gathering follows desc.photon_mapper."""
        if film is None:
            film = np.zeros((desc.height, desc.width, 8), dtype=np.float32)
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        pm = _PmIn()
        for m in range(2):
            d = maps[m]
            pm.position[m] = arr(d["position"], np.float32)
            pm.omega_in[m] = arr(d["omega_in"], np.float32)
            pm.power[m] = arr(d["power"], np.float32)
            pm.blend_idx[m] = arr(d["blend_idx"], np.int32)
            pm.blend_w[m] = arr(d["blend_w"], np.float32)
            pm.n[m] = int(np.asarray(d["position"]).reshape(-1, 3).shape[0])
            pm.radius[m] = float(d["radius"])
            pm.k[m] = int(d["k"])
        pm.visualize = int(bool(desc.photon_mapper.visualize))
        pm.ray_direct = 0 if desc.photon_mapper.ray_trace_direct < 0 else 1
        t = recovery_table
        pm.rec_wavelengths = arr(t["wavelengths"], np.float32)
        pm.rec_spectra = arr(t["spectra"], np.float32)
        pm.rec_points = arr(t["points"], np.float32)
        pm.rec_tris = arr(t["triangles"], np.int32)
        pm.rec_nw = int(np.asarray(t["wavelengths"]).size)
        pm.rec_ns = int(np.asarray(t["spectra"]).shape[0])
        pm.rec_nt = int(np.asarray(t["triangles"]).shape[0])
        D = desc.photon_mapper
        fg = D.ray_trace_direct >= 0 and D.final_gather_rays > 0
        pm.fg_rays = int(D.final_gather_rays) if fg else 0
        pm.fg_secondary = (1 if D.secondary_gather_rays == 0 else max(0, int(D.secondary_gather_rays))) if fg else 0
        if irradiance is not None and len(irradiance["position"]):
            pm.irr_position = arr(irradiance["position"], np.float32)
            pm.irr_normal = arr(irradiance["normal"], np.float32)
            pm.irr_blend_idx = arr(irradiance["blend_idx"], np.int32)
            pm.irr_blend_w = arr(irradiance["blend_w"], np.float32)
            pm.irr_r2 = arr(irradiance["r2"], np.float32)
            pm.n_irr = int(np.asarray(irradiance["position"]).reshape(-1, 3).shape[0])
        L = lib()
        L.oracle_render_pm.restype = C.c_int
        L.oracle_render_pm.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int]
        b, e = pixels if pixels is not None else (0, desc.width * desc.height)
        rc = L.oracle_render_pm(self.h, C.addressof(desc), C.byref(pm), film.ctypes.data, int(b), int(e), int(threads))
        if rc:
            raise RuntimeError(f"oracle_render_pm failed ({rc})")
        return film

    def __del__(self):
        try:
            if self.h:
                lib().oracle_scene_free(self.h)
                self.h = None
        except Exception:
            pass


class _PmIn(C.Structure):
    _fields_ = [("position", C.c_void_p * 2), ("omega_in", C.c_void_p * 2), ("power", C.c_void_p * 2),
                ("blend_idx", C.c_void_p * 2), ("blend_w", C.c_void_p * 2), ("n", C.c_uint64 * 2),
                ("radius", C.c_float * 2), ("k", C.c_int32 * 2), ("visualize", C.c_int32), ("ray_direct", C.c_int32),
                ("rec_wavelengths", C.c_void_p), ("rec_spectra", C.c_void_p), ("rec_points", C.c_void_p),
                ("rec_tris", C.c_void_p), ("rec_nw", C.c_int32), ("rec_ns", C.c_int32), ("rec_nt", C.c_int32),
                ("fg_rays", C.c_int32), ("fg_secondary", C.c_int32), ("irr_position", C.c_void_p),
                ("irr_normal", C.c_void_p), ("irr_blend_idx", C.c_void_p), ("irr_blend_w", C.c_void_p),
                ("irr_r2", C.c_void_p), ("n_irr", C.c_uint64)]


class Tree:
    """Median-split binary tree over the mesh (CPU only)."""

    def __init__(self, vertices, triangles):
        self.V = _f32(vertices).reshape(-1, 3)
        self.T = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        self.h = lib().oracle_tree_build(self.V.ctypes.data, self.V.shape[0], self.T.ctypes.data, self.T.shape[0])

    def trace(self, rays, any_hit=False, threads=0):
        R = _f32(rays).reshape(-1, 8)
        H = np.empty((R.shape[0], 2), dtype=np.int32)
        lib().oracle_tree_trace(self.h, R.ctypes.data, R.shape[0], H.ctypes.data, int(bool(any_hit)), int(threads))
        return H[:, 0].copy(), H[:, 1].view(np.float32).copy()

    def __del__(self):
        try:
            if self.h:
                lib().oracle_tree_free(self.h)
                self.h = None
        except Exception:
            pass


def knn(photons, queries, k, r_max, threads=0):
    """Brute-force k nearest photons within r_max: (idx, d2, count) like liar_gpu_photon_gather."""
    L = lib()
    L.oracle_knn.restype = C.c_int
    L.oracle_knn.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.c_int]
    P = _f32(photons).reshape(-1, 3)
    Q = _f32(queries).reshape(-1, 3)
    idx = np.empty((Q.shape[0], k), np.int32)
    d2 = np.empty((Q.shape[0], k), np.float32)
    cnt = np.empty(Q.shape[0], np.int32)
    L.oracle_knn(P.ctypes.data, P.shape[0], Q.ctypes.data, Q.shape[0], int(k), float(r_max), idx.ctypes.data,
                 d2.ctypes.data, cnt.ctypes.data, int(threads))
    return idx, d2, cnt


def knn_grid(photons, queries, k, r_max, threads=0):
    """Grid-accelerated version of knn (identical results), for large photon counts."""
    L = lib()
    L.oracle_knn_grid.restype = C.c_int
    L.oracle_knn_grid.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_int]
    P = _f32(photons).reshape(-1, 3)
    Q = _f32(queries).reshape(-1, 3)
    idx = np.empty((Q.shape[0], k), np.int32)
    d2 = np.empty((Q.shape[0], k), np.float32)
    cnt = np.empty(Q.shape[0], np.int32)
    L.oracle_knn_grid(P.ctypes.data, P.shape[0], Q.ctypes.data, Q.shape[0], int(k), float(r_max), idx.ctypes.data,
                      d2.ctypes.data, cnt.ctypes.data, int(threads))
    return idx, d2, cnt


def photon_trace(render_scene, desc, capacity, threads=0):
    """The photon-tracing restatement over a RenderScene; photons sorted by (path, bounce).
    Returns (records (n,) structured array, counts dict)."""
    L = lib()
    L.oracle_photon_trace.restype = C.c_int
    L.oracle_photon_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int]
    rec = np.zeros(capacity, dtype=[("pos", "<f4", 3), ("omega", "<f4", 3), ("power", "<f4", 3), ("path", "<u4"),
                                    ("tag", "<u4")])
    counts = np.zeros(4, np.uint64)
    rc = L.oracle_photon_trace(render_scene.h, C.addressof(desc), rec.ctypes.data, capacity, counts.ctypes.data,
                               int(threads))
    n = int(min(counts[0], capacity))
    return rec[:n], {"stored": int(counts[0]), "global": int(counts[1]), "caustic": int(counts[2]),
                     "emitted": int(counts[3]), "rc": rc}


# ---- path-guiding network (oracle_guide.cpp)

GUIDE_PARAMS = 256 * 64 + 4 * 64 * 64 + 64 * 48


def _guide_lib():
    L = lib()
    vp = C.c_void_p
    L.oracle_guide_forward.restype = C.c_int
    L.oracle_guide_forward.argtypes = [vp, vp, C.c_uint64, vp, vp, C.c_int, vp, vp]
    L.oracle_guide_grad.restype = C.c_int
    L.oracle_guide_grad.argtypes = [vp, vp, C.c_uint64, vp, vp, C.c_int, vp, vp]
    L.oracle_vmf_pdf.restype = C.c_int
    L.oracle_vmf_pdf.argtypes = [vp, vp, C.c_uint64, vp]
    L.oracle_vmf_sample.restype = C.c_int
    L.oracle_vmf_sample.argtypes = [vp, vp, C.c_uint64, vp, vp]
    return L


def guide_forward(params, inputs, lo, hi, emulate=True):
    """(raw outputs (n, 48), mixtures (n, 40)) of the guiding network on raw inputs (n, 9)."""
    p, x = _f32(params), _f32(inputs).reshape(-1, 9)
    lo, hi = _f32(lo), _f32(hi)
    raw = np.zeros((x.shape[0], 48), np.float32)
    mix = np.zeros((x.shape[0], 40), np.float32)
    _guide_lib().oracle_guide_forward(p.ctypes.data, x.ctypes.data, x.shape[0], lo.ctypes.data, hi.ctypes.data,
                                      int(emulate), raw.ctypes.data, mix.ctypes.data)
    return raw, mix


def guide_grad(params, records, lo, hi, emulate=True):
    """(gradient (GUIDE_PARAMS,) float64, loss) of the mean training loss over records (n, 13)."""
    p, r = _f32(params), _f32(records).reshape(-1, 13)
    lo, hi = _f32(lo), _f32(hi)
    g = np.zeros(GUIDE_PARAMS, np.float64)
    loss = C.c_double()
    _guide_lib().oracle_guide_grad(p.ctypes.data, r.ctypes.data, r.shape[0], lo.ctypes.data, hi.ctypes.data,
                                   int(emulate), g.ctypes.data, C.addressof(loss))
    return g, loss.value


def vmf_pdf(mix, dirs):
    m, d = _f32(mix).reshape(-1, 40), _f32(dirs).reshape(-1, 3)
    out = np.zeros(d.shape[0], np.float32)
    _guide_lib().oracle_vmf_pdf(m.ctypes.data, d.ctypes.data, d.shape[0], out.ctypes.data)
    return out


def vmf_sample(mix, u):
    m, uu = _f32(mix).reshape(-1, 40), _f32(u).reshape(-1, 3)
    dirs = np.zeros((uu.shape[0], 3), np.float32)
    pdf = np.zeros(uu.shape[0], np.float32)
    _guide_lib().oracle_vmf_sample(m.ctypes.data, uu.ctypes.data, uu.shape[0], dirs.ctypes.data, pdf.ctypes.data)
    return dirs, pdf
