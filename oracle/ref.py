"""ctypes wrapper of oracle/_ref/liboracle_ref.so (TEST INFRASTRUCTURE ONLY).

The library is the reference renderer itself (rainbow-core + rainbow-cpu sources
compiled by oracle/Makefile) plus oracle/harness/ref_harness.cpp. Entry points
take the same rb_scene_desc / rb_camera_desc structures as the product, or build
the seeded benchmark scenes themselves (RefScene.generated), in which case
nothing of the product is imported or loaded.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle_ref.so")

_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing (build with `make -C oracle ref` where the reference is present)")
        L = C.CDLL(LIB_PATH)
        vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
        sig = {
            "orc_scene_build": (i32, [vp, vp, C.POINTER(vp)]),
            "orc_scene_generate": (i32, [vp, C.POINTER(vp), C.POINTER(u32)]),
            "orc_scene_free": (None, [vp]),
            "orc_export_bvh": (i32, [vp, vp, vp, vp, C.POINTER(u32), C.POINTER(u32)]),
            "orc_export_mesh_bvh": (i32, [vp, u32, vp, vp, C.POINTER(u32), C.POINTER(u32)]),
            "orc_export_camera": (i32, [vp, vp, vp]),
            "orc_export_areas": (i32, [vp, vp]),
            "orc_trace": (i32, [vp, vp, u32, i32, vp, vp]),
            "orc_make_rays": (i32, [vp, u32, C.c_uint64, vp]),
            "orc_camera_rays": (i32, [vp, vp, vp, u32, u32, vp]),
            "orc_trace_samples": (i32, [vp, vp, vp, u32, u32, f32, u32, vp]),
            "orc_render": (i32, [vp, u32, u32, u32, f32, u32, i32, i32, i32, vp, vp, C.POINTER(C.c_double)]),
            "orc_render_shipped": (i32, [vp, u32, u32, f32, vp, C.POINTER(C.c_double)]),
            "orc_render_photons": (i32, [vp, u32, u32, u32, f32, vp, C.POINTER(C.c_double)]),
            "orc_pcg32": (i32, [C.c_uint64, u32, vp, vp]),
            "orc_bsdf": (i32, [vp, u32, u32, vp, vp, vp, u32, vp, vp, vp, vp, vp, vp]),
            "orc_texture_sample": (i32, [vp, u32, u32, u32, vp, vp]),
            "orc_set_volume": (None, [vp, i32]),
            "orc_set_direct": (None, [vp, C.c_uint32, C.c_uint32]),
            "orc_film_read": (i32, [vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _LIB = L
    return _LIB


def _ok(st, where):
    if st != 0:
        raise RuntimeError(f"{where} returned {st}")


class _GenParams(C.Structure):
    """rb_scene_gen_params of include/rbgpu.h."""
    _fields_ = [("kind", C.c_uint32), ("seed", C.c_uint32), ("num_spheres", C.c_uint32), ("subdivision", C.c_uint32),
                ("width", C.c_int32), ("height", C.c_int32)]


class RefScene:
    """A reference `scene` + `perspective_camera` built from a product Scene description."""

    def __init__(self, scene):
        self.scene = scene
        self.h = C.c_void_p()
        _ok(lib().orc_scene_build(C.addressof(scene.desc), C.addressof(scene.camera), C.byref(self.h)),
            "orc_scene_build")
        self.width, self.height = scene.camera.width, scene.camera.height
        self.num_entities = scene.desc.num_entities

    @classmethod
    def generated(cls, kind, seed, width, height, num_spheres=0, subdivision=0):
        """The seeded benchmark scene (kind: RB_SCENE_* of include/rbgpu.h) generated and built inside the oracle
        library; .triangles holds its triangle count."""
        self = cls.__new__(cls)
        self.scene = None
        self.h = C.c_void_p()
        tris = C.c_uint32()
        gp = _GenParams(kind, seed, num_spheres, subdivision, width, height)
        _ok(lib().orc_scene_generate(C.addressof(gp), C.byref(self.h), C.byref(tris)), "orc_scene_generate")
        self.width, self.height, self.triangles = width, height, tris.value
        self.num_entities = None
        return self

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_free(self.h)
            self.h = None

    def bvh(self):
        nn, npr = C.c_uint32(), C.c_uint32()
        _ok(lib().orc_export_bvh(self.h, None, None, None, C.byref(nn), C.byref(npr)), "orc_export_bvh")
        nodes = np.zeros((nn.value, 8), dtype=np.float32)
        pe = np.zeros(npr.value, dtype=np.uint32)
        pi = np.zeros(npr.value, dtype=np.uint32)
        _ok(lib().orc_export_bvh(self.h, nodes.ctypes.data, pe.ctypes.data, pi.ctypes.data, C.byref(nn), C.byref(npr)),
            "orc_export_bvh")
        return nodes, pe, pi

    def mesh_bvh(self, entity):
        """The reference's own tree of entity `entity`'s mesh (two-level case): nodes (n, 8) and leaf faces."""
        nn, npr = C.c_uint32(), C.c_uint32()
        _ok(lib().orc_export_mesh_bvh(self.h, entity, None, None, C.byref(nn), C.byref(npr)), "orc_export_mesh_bvh")
        nodes = np.zeros((nn.value, 8), dtype=np.float32)
        faces = np.zeros(npr.value, dtype=np.uint32)
        _ok(lib().orc_export_mesh_bvh(self.h, entity, nodes.ctypes.data, faces.ctypes.data, C.byref(nn), C.byref(npr)),
            "orc_export_mesh_bvh")
        return nodes, faces

    def camera_matrices(self):
        r2c = np.zeros(16, dtype=np.float32)
        c2w = np.zeros(16, dtype=np.float32)
        _ok(lib().orc_export_camera(self.h, r2c.ctypes.data, c2w.ctypes.data), "orc_export_camera")
        return r2c, c2w

    def areas(self):
        a = np.zeros(self.num_entities, dtype=np.float32)
        _ok(lib().orc_export_areas(self.h, a.ctypes.data), "orc_export_areas")
        return a

    def trace(self, rays, shadow=False, points=False):
        from rainbow_b200 import HIT_DTYPE, RAY_DTYPE
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
        pts = np.zeros((rays.shape[0], 3), dtype=np.float32) if points else None
        _ok(lib().orc_trace(self.h, rays.ctypes.data, rays.shape[0], int(shadow), hits.ctypes.data,
                            pts.ctypes.data if points else None), "orc_trace")
        return (hits, pts) if points else hits

    def make_rays(self, n, seed):
        from rainbow_b200 import RAY_DTYPE
        rays = np.zeros(n, dtype=RAY_DTYPE)
        _ok(lib().orc_make_rays(self.h, n, seed, rays.ctypes.data), "orc_make_rays")
        return rays

    def camera_rays(self, pixels, samples, seed=0):
        from rainbow_b200 import RAY_DTYPE
        px = np.ascontiguousarray(pixels, dtype=np.uint32)
        sm = np.ascontiguousarray(samples, dtype=np.uint32)
        rays = np.zeros(px.shape[0], dtype=RAY_DTYPE)
        _ok(lib().orc_camera_rays(self.h, px.ctypes.data, sm.ctypes.data, px.shape[0], seed, rays.ctypes.data),
            "orc_camera_rays")
        return rays

    def set_volume(self, volume: bool):
        """Trace with volume_path_integrator (True) or path_integrator (False)."""
        lib().orc_set_volume(self.h, 1 if volume else 0)

    def set_direct(self, emitter_samples: int, bsdf_samples: int):
        """Trace with direct_integrator(emitter_samples, bsdf_samples); (0, 0) goes back."""
        lib().orc_set_direct(self.h, emitter_samples, bsdf_samples)

    def trace_samples(self, pixels, samples, max_depth=5, rr=1.0, seed=0):
        px = np.ascontiguousarray(pixels, dtype=np.uint32)
        sm = np.ascontiguousarray(samples, dtype=np.uint32)
        out = np.zeros((px.shape[0], 3), dtype=np.float32)
        _ok(lib().orc_trace_samples(self.h, px.ctypes.data, sm.ctypes.data, px.shape[0], max_depth, rr, seed,
                                    out.ctypes.data), "orc_trace_samples")
        return out

    def render(self, spp, first_sample=0, max_depth=5, rr=1.0, seed=0, threads=0, rows=(0, 0)):
        """FP64 per-pixel sums (H, W, 3) of L and L^2 and the wall seconds."""
        s = np.zeros((self.height, self.width, 3), dtype=np.float64)
        q = np.zeros_like(s)
        sec = C.c_double()
        _ok(lib().orc_render(self.h, spp, first_sample, max_depth, rr, seed, threads, rows[0], rows[1], s.ctypes.data,
                             q.ctypes.data, C.byref(sec)), "orc_render")
        return s, q, sec.value

    def film(self):
        """The camera's film as an integrator left it: pixel::spectrum() of every pixel (H, W, 3)."""
        img = np.zeros((self.height, self.width, 3), dtype=np.float32)
        _ok(lib().orc_film_read(self.h, img.ctypes.data), "orc_film_read")
        return img

    def render_shipped(self, spp, max_depth=5, rr=1.0):
        img = np.zeros((self.height, self.width, 3), dtype=np.float32)
        sec = C.c_double()
        _ok(lib().orc_render_shipped(self.h, spp, max_depth, rr, img.ctypes.data, C.byref(sec)), "orc_render_shipped")
        return img, sec.value


    def render_photons(self, iterations, max_depth=5, photons=0, radius=1.0):
        """photon_mapping_integrator::render (iterations, max_depth, photons, radius) as shipped: the image."""
        img = np.zeros((self.height, self.width, 3), dtype=np.float32)
        sec = C.c_double()
        _ok(lib().orc_render_photons(self.h, iterations, max_depth, photons, radius, img.ctypes.data, C.byref(sec)),
            "orc_render_photons")
        return img, sec.value


def pcg32(seed, n):
    u = np.zeros(n, dtype=np.uint32)
    r = np.zeros(n, dtype=np.float32)
    _ok(lib().orc_pcg32(seed, n, u.ctypes.data, r.ctypes.data), "orc_pcg32")
    return u, r


def bsdf(material, wo, u, wi_eval, include):
    """scattering_function_collection sample / evaluate / pdf for one material
    (a descriptor, or a ctypes array of descriptors whose first entry is the
    material and whose other entries are a mixture's components)."""
    count = len(material) if isinstance(material, C.Array) else 1
    n = wo.shape[0]
    wo = np.ascontiguousarray(wo, dtype=np.float32)
    u = np.ascontiguousarray(u, dtype=np.float32)
    wie = np.ascontiguousarray(wi_eval, dtype=np.float32)
    out = dict(wi=np.zeros((n, 3), np.float32), f=np.zeros((n, 3), np.float32), pdf=np.zeros(n, np.float32),
               type=np.zeros(n, np.uint32), f_eval=np.zeros((n, 3), np.float32), pdf_eval=np.zeros(n, np.float32))
    _ok(lib().orc_bsdf(C.byref(material), count, n, wo.ctypes.data, u.ctypes.data, wie.ctypes.data, include,
                       out["wi"].ctypes.data, out["f"].ctypes.data, out["pdf"].ctypes.data, out["type"].ctypes.data,
                       out["f_eval"].ctypes.data, out["pdf_eval"].ctypes.data), "orc_bsdf")
    return out


def texture_sample(image, uv):
    """image_texture2d<spectrum>::sample at each uv of an (height, width, 3) image."""
    img = np.ascontiguousarray(image, dtype=np.float32)
    uv = np.ascontiguousarray(uv, dtype=np.float32)
    out = np.zeros((uv.shape[0], 3), np.float32)
    _ok(lib().orc_texture_sample(img.ctypes.data, img.shape[1], img.shape[0], uv.shape[0], uv.ctypes.data,
                                 out.ctypes.data), "orc_texture_sample")
    return out


ADAPTER_PATH = os.path.join(HERE, "_ref", "libadapter_check.so")
_ADAPTER = None


def adapter_available() -> bool:
    return os.path.exists(ADAPTER_PATH) and available()


def adapter_lib():
    """The drop-in adapter (rainbow_b200/adapter, wavefront_path_integrator) compiled against the reference,
    with its test entry points; it loads the reference library and the product library."""
    global _ADAPTER
    if _ADAPTER is None:
        lib()
        L = C.CDLL(ADAPTER_PATH)
        vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
        L.adp_render.restype, L.adp_render.argtypes = i32, [vp, u32, u32, f32, u32, C.c_char_p, u32]
        L.adp_render_photons.restype = i32
        L.adp_render_photons.argtypes = [vp, u32, u32, u32, f32, u32, C.c_char_p, u32]
        L.adp_export.restype = i32
        L.adp_export.argtypes = [vp, vp, vp, vp, C.POINTER(u32), C.POINTER(u32), vp, vp, vp, vp]
        L.adp_export_materials.restype = i32
        L.adp_export_materials.argtypes = [vp, vp, C.POINTER(u32), vp, C.POINTER(u32)]
        L.adp_export_texture.restype = i32
        L.adp_export_texture.argtypes = [vp, u32, vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), vp]
        _ADAPTER = L
    return _ADAPTER


def adapter_render(R, spp, max_depth=5, threshold=1.0, seed=0):
    """wavefront_path_integrator(random_sampler2d(spp), random_sampler1d(spp), max_depth, threshold)
    .render(camera, scene) on the reference scene of R; returns the camera's film (H, W, 3)."""
    err = C.create_string_buffer(512)
    st = adapter_lib().adp_render(R.h, spp, max_depth, threshold, seed, err, 512)
    if st != 0:
        raise RuntimeError(f"wavefront_path_integrator::render failed ({st}): {err.value.decode()}")
    return R.film()


def adapter_render_photons(R, iterations, max_depth=5, photons=0, radius=1.0, seed=0):
    """wavefront_photon_mapping_integrator(random_sampler2d(1), random_sampler1d(1), iterations, max_depth,
    photons, radius).render(camera, scene) on the reference scene of R; returns the camera's film (H, W, 3)."""
    err = C.create_string_buffer(512)
    st = adapter_lib().adp_render_photons(R.h, iterations, max_depth, photons, radius, seed, err, 512)
    if st != 0:
        raise RuntimeError(f"wavefront_photon_mapping_integrator::render failed ({st}): {err.value.decode()}")
    return R.film()


def adapter_export_materials(R, material_type):
    """The adapter's exported material list of R's reference scene and each entity's index into it."""
    L = adapter_lib()
    n, ne = C.c_uint32(), C.c_uint32()
    _ok(L.adp_export_materials(R.h, None, C.byref(n), None, C.byref(ne)), "adp_export_materials")
    mats = (material_type * max(1, n.value))()
    ent = np.zeros(max(1, ne.value), dtype=np.int32)
    _ok(L.adp_export_materials(R.h, C.addressof(mats), C.byref(n), ent.ctypes.data, C.byref(ne)), "adp_export_materials")
    return mats, ent[:ne.value]


def adapter_export_textures(R, texture_type):
    """The adapter's exported textures of R's reference scene in export order: (description with its rgb
    pointer cleared, (height, width, 3) texels of an image or None)."""
    L = adapter_lib()
    w, h, n = C.c_uint32(), C.c_uint32(), C.c_uint32()
    _ok(L.adp_export_texture(R.h, 0, None, C.byref(w), C.byref(h), C.byref(n), None), "adp_export_texture")
    out = []
    for t in range(n.value):
        d = texture_type()
        _ok(L.adp_export_texture(R.h, t, None, C.byref(w), C.byref(h), C.byref(n), C.byref(d)), "adp_export_texture")
        a = None
        if w.value and h.value:
            a = np.zeros((h.value, w.value, 3), dtype=np.float32)
            _ok(L.adp_export_texture(R.h, t, a.ctypes.data, C.byref(w), C.byref(h), C.byref(n), None),
                "adp_export_texture")
        out.append((d, a))
    return out


def adapter_export(R, material_type, emitter_type, camera_type):
    """The adapter's export of R's reference scene: (nodes, prim_entity, prim_index) of rb_bvh_build on it,
    per-entity material / emitter descriptions with presence flags, and the camera description."""
    L = adapter_lib()
    nn, npr = C.c_uint32(), C.c_uint32()
    _ok(L.adp_export(R.h, None, None, None, C.byref(nn), C.byref(npr), None, None, None, None), "adp_export")
    nodes = np.zeros((nn.value, 8), dtype=np.float32)
    pe = np.zeros(npr.value, dtype=np.uint32)
    pi = np.zeros(npr.value, dtype=np.uint32)
    ne = R.num_entities
    mats, ems = (material_type * ne)(), (emitter_type * ne)()
    has = np.zeros(2 * ne, dtype=np.int32)
    cam = camera_type()
    _ok(L.adp_export(R.h, nodes.ctypes.data, pe.ctypes.data, pi.ctypes.data, C.byref(nn), C.byref(npr), C.addressof(mats),
                     C.addressof(ems), has.ctypes.data, C.addressof(cam)), "adp_export")
    return (nodes, pe, pi), mats, ems, has.reshape(ne, 2), cam
