"""ctypes binding of librbgpu.so (include/rbgpu.h).

The structures below mirror the C ABI field for field. The library is loaded
from the package directory; importing this module fails loudly when it has not
been built (there is no Python or CPU fallback for any entry point).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librbgpu.so")

RB_OK = 0
STATUS_NAMES = {
    0: "RB_OK", 1: "RB_ERR_INVALID_ARGUMENT", 2: "RB_ERR_CUDA", 3: "RB_ERR_OUT_OF_MEMORY",
    4: "RB_ERR_NO_SCENE", 5: "RB_ERR_STACK_OVERFLOW", 6: "RB_ERR_QUEUE_OVERFLOW", 7: "RB_ERR_UNSUPPORTED",
    8: "RB_ERR_IO", 9: "RB_ERR_CHECKPOINT", 10: "RB_ERR_DEVICE_TIMEOUT", 11: "RB_ERR_NO_DEVICE",
    12: "RB_ERR_TOO_LARGE",
}

RB_MATERIAL_MATTE, RB_MATERIAL_METAL, RB_MATERIAL_GLASS, RB_MATERIAL_PLASTIC, RB_MATERIAL_MIRROR = 0, 1, 2, 3, 4
RB_MATERIAL_SUBSTRATE = 5
RB_MATERIAL_UBER = 6
RB_MATERIAL_TRANSLUCENT = 7
RB_MATERIAL_MIXTURE = 8
RB_MATERIAL_SUBSURFACE = 9
RB_TEXTURE_IMAGE = 0
RB_TEXTURE_SCALE = 1
RB_TEXTURE_MIXTURE = 2
RB_EMITTER_SURFACE, RB_EMITTER_ENVIRONMENT = 0, 1
RB_SCENE_BOX, RB_SCENE_SPHERES, RB_SCENE_SLIT_ROOM, RB_SCENE_FOG = 0, 1, 2, 3
RB_RENDER_RESET = 1
RB_RENDER_GUIDE = 2
RB_RENDER_TRAIN = 4
RB_RENDER_VOLUME = 8
RB_RENDER_DIRECT = 16
RB_GUIDE_SEQUENTIAL = 1
RB_GUIDE_NUM_PARAMS = 30000
RB_GUIDE_INPUTS = 9
RB_GUIDE_OUTPUTS = 48
RB_BVH_LEAF_FLAG = 0x80000000
RB_BVH_ALL_TRIANGLES = 0xFFFFFFFF
RB_SORT_MATERIAL, RB_SORT_NONE, RB_SORT_RAYS = 0, 1, 2
RB_TRAVERSAL_PER_THREAD, RB_TRAVERSAL_REFILL = 0, 1
RB_SHADOW_CLOSEST, RB_SHADOW_FIRST_OCCLUDER = 0, 1

F16 = C.c_float * 16
F3 = C.c_float * 3


class MeshDesc(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("tangents", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
                ("indices", C.POINTER(C.c_uint32)), ("num_vertices", C.c_uint32),
                ("num_triangles", C.c_uint32), ("reverse_orientation", C.c_int32), ("reserved", C.c_int32)]


class MaterialDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("remap_roughness", C.c_int32), ("diffuse", F3), ("sigma", C.c_float),
                ("eta", F3), ("k", F3), ("reflectance", F3), ("transmission", F3), ("ior", C.c_float),
                ("roughness_u", C.c_float), ("roughness_v", C.c_float), ("specular", F3), ("opacity", F3),
                ("components", C.c_int32 * 2), ("amount", F3), ("diffuse_texture", C.c_uint32),
                ("reflectance_texture", C.c_uint32), ("transmission_texture", C.c_uint32),
                ("specular_texture", C.c_uint32), ("opacity_texture", C.c_uint32), ("mfp", F3),
                ("roughness_u_texture", C.c_uint32), ("roughness_v_texture", C.c_uint32), ("ior_texture", C.c_uint32),
                ("sigma_texture", C.c_uint32), ("eta_texture", C.c_uint32), ("k_texture", C.c_uint32),
                ("mfp_texture", C.c_uint32)]


class TextureDesc(C.Structure):
    _fields_ = [("rgb", C.POINTER(C.c_float)), ("width", C.c_uint32), ("height", C.c_uint32), ("kind", C.c_uint32),
                ("inputs", C.c_uint32 * 3), ("constants", (C.c_float * 3) * 3)]


class MediumDesc(C.Structure):
    _fields_ = [("sigma_a", F3), ("sigma_s", F3), ("g", C.c_float), ("reserved", C.c_uint32)]


class MediaDesc(C.Structure):
    _fields_ = [("inside", C.c_int32), ("outside", C.c_int32)]


class EmitterDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("radiance", F3), ("radius", C.c_float)]


class EntityDesc(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("material", C.c_int32), ("emitter", C.c_int32), ("medium", C.c_int32),
                ("local_to_world", F16), ("world_to_local", F16)]


class BvhDesc(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_float)), ("num_nodes", C.c_uint32), ("num_prims", C.c_uint32),
                ("prim_entity", C.POINTER(C.c_uint32)), ("prim_index", C.POINTER(C.c_uint32))]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(MeshDesc)), ("num_meshes", C.c_uint32), ("num_entities", C.c_uint32),
                ("entities", C.POINTER(EntityDesc)), ("materials", C.POINTER(MaterialDesc)),
                ("num_materials", C.c_uint32), ("num_emitters", C.c_uint32), ("emitters", C.POINTER(EmitterDesc)),
                ("bvh", BvhDesc), ("mediums", C.POINTER(MediumDesc)), ("num_mediums", C.c_uint32),
                ("num_media", C.c_uint32), ("media", C.POINTER(MediaDesc)), ("textures", C.POINTER(TextureDesc)),
                ("num_textures", C.c_uint32), ("reserved", C.c_uint32)]


class CameraDesc(C.Structure):
    _fields_ = [("raster_to_camera", F16), ("camera_to_world", F16), ("eye", F3), ("target", F3), ("up", F3),
                ("fov_degrees", C.c_float), ("lens_radius", C.c_float), ("focus_distance", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]


class RenderParams(C.Structure):
    _fields_ = [("camera", CameraDesc), ("spp", C.c_uint32), ("first_sample", C.c_uint32),
                ("max_depth", C.c_uint32), ("rr_threshold", C.c_float), ("seed", C.c_uint32),
                ("flags", C.c_uint32), ("paths_per_wave", C.c_uint32), ("direct_samples", C.c_uint32)]


class PhotonParams(C.Structure):
    _fields_ = [("camera", CameraDesc), ("iterations", C.c_uint32), ("max_depth", C.c_uint32),
                ("photons", C.c_uint32), ("radius", C.c_float), ("seed", C.c_uint32), ("reserved", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("paths_per_wave", C.c_uint32), ("block_trace", C.c_uint32), ("block_shade", C.c_uint32),
                ("grid_per_sm", C.c_uint32), ("sort", C.c_uint32), ("tail_bounce", C.c_uint32),
                ("lanes", C.c_uint32), ("traversal", C.c_uint32), ("smem_carveout", C.c_uint32),
                ("shadow_test", C.c_uint32), ("reserved", C.c_uint32 * 2)]

    def as_dict(self):
        return {k: getattr(self, k) for k in ("paths_per_wave", "block_trace", "block_shade", "grid_per_sm", "sort",
                                              "tail_bounce", "lanes", "traversal", "smem_carveout", "shadow_test")}


class BatchView(C.Structure):
    _fields_ = [("camera", CameraDesc), ("spp", C.c_uint32), ("first_sample", C.c_uint32), ("seed", C.c_uint32),
                ("reserved", C.c_uint32)]


class BatchParams(C.Structure):
    _fields_ = [("views", C.POINTER(BatchView)), ("count", C.c_uint32), ("max_depth", C.c_uint32),
                ("rr_threshold", C.c_float), ("flags", C.c_uint32), ("order", C.POINTER(C.c_uint32))]


class RenderStats(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("extend_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("mis_rays", C.c_uint64), ("node_visits", C.c_uint64), ("triangle_tests", C.c_uint64),
                ("device_error", C.c_uint32), ("kernel_launches", C.c_uint32), ("elapsed_ms", C.c_float),
                ("extend_ms", C.c_float), ("secondary_ms", C.c_float), ("extend_launches", C.c_uint32),
                ("secondary_launches", C.c_uint32)]


class SceneGenParams(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("seed", C.c_uint32), ("num_spheres", C.c_uint32),
                ("subdivision", C.c_uint32), ("width", C.c_int32), ("height", C.c_int32)]


class GuideConfig(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("learning_rate", C.c_float), ("batch_size", C.c_uint32),
                ("steps_per_wave", C.c_uint32), ("max_samples", C.c_uint32), ("min_rows", C.c_uint32),
                ("weight_clip", C.c_float), ("warmup_steps", C.c_uint32)]


class GuideStats(C.Structure):
    _fields_ = [("steps", C.c_uint32), ("samples_last_wave", C.c_uint32), ("candidates_last_wave", C.c_uint32),
                ("device_error", C.c_uint32), ("last_loss", C.c_float), ("rows_last_step", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


# rb_guide_sample: inputs[9], direction[3], bsdf_pdf, weight, reserved[2] (64 bytes)
GUIDE_SAMPLE_DTYPE = np.dtype([("inputs", "<f4", 9), ("direction", "<f4", 3), ("bsdf_pdf", "<f4"),
                               ("weight", "<f4"), ("reserved", "<f4", 2)])
assert GUIDE_SAMPLE_DTYPE.itemsize == 64

RAY_DTYPE = np.dtype([("origin", "<f4", 3), ("direction", "<f4", 3), ("length", "<f4")])
HIT_DTYPE = np.dtype([("entity", "<i4"), ("triangle", "<i4"), ("t", "<f4"), ("b1", "<f4"), ("b2", "<f4")])
assert RAY_DTYPE.itemsize == 28 and HIT_DTYPE.itemsize == 20

# every entry point declared in include/rbgpu.h: name -> (restype, argtypes)
SIGNATURES = {
    "rb_status_string": (C.c_char_p, [C.c_int32]),
    "rb_context_create": (C.c_int32, [C.POINTER(C.c_void_p), C.c_int]),
    "rb_context_destroy": (C.c_int32, [C.c_void_p]),
    "rb_scene_upload": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc)]),
    "rb_trace_closest": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "rb_trace_shadow": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "rb_trace_closest_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "rb_trace_shadow_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "rb_render": (C.c_int32, [C.c_void_p, C.POINTER(RenderParams), C.c_void_p]),
    "rb_film_read": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rb_render_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(RenderStats)]),
    "rb_set_counting": (C.c_int32, [C.c_void_p, C.c_int]),
    "rb_set_profiling": (C.c_int32, [C.c_void_p, C.c_int]),
    "rb_checkpoint_save": (C.c_int32, [C.c_void_p, C.c_char_p]),
    "rb_checkpoint_load": (C.c_int32, [C.c_void_p, C.c_char_p]),
    "rb_bvh_build": (C.c_int32, [C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]),
    "rb_bvh_get": (C.c_int32, [C.c_void_p, C.POINTER(BvhDesc)]),
    "rb_bvh_depth": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "rb_render_async": (C.c_int32, [C.c_void_p, C.POINTER(RenderParams), C.c_void_p]),
    "rb_render_wait": (C.c_int32, [C.c_void_p]),
    "rb_film_to_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rb_film_from_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "rb_bvh_mesh_tree_count": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "rb_bvh_get_mesh_tree": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(BvhDesc)]),
    "rb_bvh_free": (None, [C.c_void_p]),
    "rb_scene_generate": (C.c_int32, [C.POINTER(SceneGenParams), C.POINTER(C.c_void_p)]),
    "rb_scene_get": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(CameraDesc)]),
    "rb_scene_free": (None, [C.c_void_p]),
    "rb_abi_version": (C.c_int32, []),
    "rb_render_photons": (C.c_int32, [C.c_void_p, C.POINTER(PhotonParams), C.c_void_p]),
    "rb_render_noalloc": (C.c_int32, [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rb_guide_init": (C.c_int32, [C.c_void_p, C.POINTER(GuideConfig)]),
    "rb_guide_get_params": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "rb_guide_set_params": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "rb_guide_forward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "rb_guide_train": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    "rb_guide_sample_dirs": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "rb_guide_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(GuideStats)]),
    "rb_guide_medium_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(GuideStats)]),
    "rb_check_bounded_wait": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(C.c_int32)]),
    "rb_inject_allocation_failure": (None, [C.c_int32]),
    "rb_set_tuning": (C.c_int32, [C.c_void_p, C.POINTER(Tuning)]),
    "rb_get_tuning": (C.c_int32, [C.c_void_p, C.POINTER(Tuning)]),
    "rb_tune_render": (C.c_int32, [C.c_void_p, C.POINTER(RenderParams), C.c_uint32, C.POINTER(Tuning),
                                   C.POINTER(C.c_float)]),
    "rb_batch_upload": (C.c_int32, [C.c_void_p, C.POINTER(SceneDesc), C.c_uint32]),
    "rb_batch_render": (C.c_int32, [C.c_void_p, C.POINTER(BatchParams), C.c_void_p]),
    "rb_batch_film_read": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rb_batch_image": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "rb_tune_batch": (C.c_int32, [C.c_void_p, C.POINTER(BatchParams), C.c_uint64, C.POINTER(Tuning),
                                  C.POINTER(C.c_float)]),
}


class RbError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


def load_library(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


def check(status: int, where: str) -> None:
    if status != RB_OK:
        raise RbError(status, where)
