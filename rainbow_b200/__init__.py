"""B200 wavefront path-tracing core, a drop-in for rainbow's path_integrator.

Python host layer over the C ABI of librbgpu.so (include/rbgpu.h). It mirrors
the reference's integrator interface for scripts and tests:

    scene = generate_scene(RB_SCENE_BOX, width=256, height=256)
    integrator = PathIntegrator(spp=16, max_depth=5, threshold=1.0)
    image = integrator.render(scene.camera, scene)   # (H, W, 3) float32 per-pixel means

`PathIntegrator(spp, max_depth=5, threshold=1)` takes the arguments of
`path_integrator(sampler2d(spp), sampler1d, max_depth, threshold)`
(rainbow-cpu/integrators/path_integrator.hpp:9-12); render(camera, scene)
follows integrator::render (integrator.hpp:64-66) and returns the film instead
of writing it. Every call runs the sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import (  # noqa: F401  (re-exported constants)
    GUIDE_SAMPLE_DTYPE, HIT_DTYPE, RAY_DTYPE, RB_BVH_ALL_TRIANGLES, RB_EMITTER_ENVIRONMENT, RB_EMITTER_SURFACE, RB_GUIDE_NUM_PARAMS,
    RB_GUIDE_OUTPUTS, RB_GUIDE_SEQUENTIAL, RB_MATERIAL_GLASS, RB_MATERIAL_MATTE, RB_MATERIAL_METAL, RB_MATERIAL_MIRROR, RB_MATERIAL_PLASTIC, RB_MATERIAL_SUBSTRATE,
    RB_MATERIAL_MIXTURE, RB_MATERIAL_SUBSURFACE, RB_MATERIAL_TRANSLUCENT, RB_MATERIAL_UBER, RB_TEXTURE_IMAGE, RB_TEXTURE_MIXTURE, RB_TEXTURE_SCALE,
    RB_RENDER_GUIDE,
    RB_RENDER_DIRECT, RB_RENDER_RESET, RB_RENDER_TRAIN, RB_RENDER_VOLUME, RB_SCENE_BOX, RB_SCENE_FOG, RB_SCENE_SLIT_ROOM, RB_SCENE_SPHERES,
    RB_SHADOW_CLOSEST, RB_SHADOW_FIRST_OCCLUDER, RB_SORT_MATERIAL, RB_SORT_NONE, RB_SORT_RAYS, RB_TRAVERSAL_PER_THREAD, RB_TRAVERSAL_REFILL, BatchParams, BatchView, Tuning,
    BvhDesc, CameraDesc, MaterialDesc, MediaDesc, MediumDesc, TextureDesc,
    GuideConfig, GuideStats, PhotonParams, RbError, RenderParams, RenderStats, SceneDesc, SceneGenParams, check, lib,
)

__all__ = ["Scene", "Context", "PathIntegrator", "generate_scene", "build_bvh", "RbError", "RAY_DTYPE", "HIT_DTYPE"]


class Scene:
    """A scene description (rb_scene_desc) plus its camera (rb_camera_desc).

    Generated scenes own their arrays inside the library; `desc` points into them.
    """

    def __init__(self, handle, desc: SceneDesc, camera: CameraDesc, keepalive=()):
        self._handle = handle
        self._free = lib().rb_scene_free  # held so that teardown at interpreter exit still frees
        self.desc = desc
        self.camera = camera
        self._keepalive = list(keepalive)

    def __del__(self):
        if getattr(self, "_handle", None):
            self._free(self._handle)
            self._handle = None

    @property
    def num_triangles(self) -> int:
        return sum(self.desc.meshes[i].num_triangles for i in range(self.desc.num_meshes))

    def with_materials(self, materials) -> "Scene":
        """A view of this scene with another materials array (a sequence of MaterialDesc)."""
        arr = (MaterialDesc * len(materials))(*materials)
        d = SceneDesc()
        C.pointer(d)[0] = self.desc
        d.materials = C.cast(arr, type(d.materials))
        d.num_materials = len(materials)
        return Scene(None, d, self.camera, keepalive=[self, arr])

    def with_textures(self, textures) -> "Scene":
        """A view of this scene with textures that materials refer to by index + 1 in their *_texture fields:
        each a (height, width, 3) float32 image, or a dict (kind=RB_TEXTURE_SCALE / RB_TEXTURE_MIXTURE,
        inputs=[texture index + 1 or 0], constants=[rgb of the constant inputs])."""
        arrs = []
        descs = (TextureDesc * max(1, len(textures)))()
        for k, t in enumerate(textures):
            if isinstance(t, dict):
                descs[k].kind = t["kind"]
                for i, v in enumerate(t.get("inputs", ())):
                    descs[k].inputs[i] = v
                for i, c in enumerate(t.get("constants", ())):
                    descs[k].constants[i][:] = [float(x) for x in c]
                continue
            a = np.ascontiguousarray(t, dtype=np.float32)
            arrs.append(a)
            descs[k].rgb = a.ctypes.data_as(C.POINTER(C.c_float))
            descs[k].height, descs[k].width = a.shape[0], a.shape[1]
        d = SceneDesc()
        C.pointer(d)[0] = self.desc
        d.textures = C.cast(descs, type(d.textures))
        d.num_textures = len(textures)
        return Scene(None, d, self.camera, keepalive=[self, descs] + arrs)

    def with_bvh(self, bvh: "Bvh") -> "Scene":
        """A view of this scene that carries a caller-supplied flattened BVH."""
        d = SceneDesc()
        C.pointer(d)[0] = self.desc
        d.bvh = bvh.desc
        return Scene(None, d, self.camera, keepalive=[self, bvh])


def generate_scene(kind: int, seed: int = 0, width: int = 256, height: int = 256, num_spheres: int = 200,
                   subdivision: int = 4) -> Scene:
    """Seeded synthetic scene of one of the benchmark configurations (rb_scene_generate)."""
    p = SceneGenParams(kind, seed, num_spheres, subdivision, width, height)
    h = C.c_void_p()
    check(lib().rb_scene_generate(C.byref(p), C.byref(h)), "rb_scene_generate")
    desc, cam = SceneDesc(), CameraDesc()
    check(lib().rb_scene_get(h, C.byref(desc), C.byref(cam)), "rb_scene_get")
    return Scene(h, desc, cam)


@dataclass
class Bvh:
    nodes: np.ndarray        # (num_nodes, 8) float32 words
    prim_entity: np.ndarray  # uint32
    prim_index: np.ndarray   # uint32 (RB_BVH_ALL_TRIANGLES: the entity's whole mesh, which has its own tree)
    depth: int
    desc: BvhDesc
    mesh_trees: list = None  # [(mesh index, nodes (n, 8) float32, faces uint32)] of the two-level case


def build_bvh(scene: Scene) -> Bvh:
    """The reference's median-split tree over the scene (rb_bvh_build), as arrays."""
    h = C.c_void_p()
    check(lib().rb_bvh_build(C.byref(scene.desc), C.byref(h)), "rb_bvh_build")
    try:
        d = BvhDesc()
        check(lib().rb_bvh_get(h, C.byref(d)), "rb_bvh_get")
        depth = C.c_uint32()
        check(lib().rb_bvh_depth(h, C.byref(depth)), "rb_bvh_depth")
        nodes = np.ctypeslib.as_array(d.nodes, (d.num_nodes * 8,)).reshape(-1, 8).copy()
        pe = np.ctypeslib.as_array(d.prim_entity, (d.num_prims,)).copy()
        pi = np.ctypeslib.as_array(d.prim_index, (d.num_prims,)).copy()
        count = C.c_uint32()
        check(lib().rb_bvh_mesh_tree_count(h, C.byref(count)), "rb_bvh_mesh_tree_count")
        trees = []
        for k in range(count.value):
            mesh = C.c_int32()
            t = BvhDesc()
            check(lib().rb_bvh_get_mesh_tree(h, k, C.byref(mesh), C.byref(t)), "rb_bvh_get_mesh_tree")
            trees.append((mesh.value, np.ctypeslib.as_array(t.nodes, (t.num_nodes * 8,)).reshape(-1, 8).copy(),
                          np.ctypeslib.as_array(t.prim_index, (t.num_prims,)).copy()))
    finally:
        lib().rb_bvh_free(h)
    b = bvh_from_arrays(nodes, pe, pi, int(depth.value))
    b.mesh_trees = trees
    return b


def bvh_from_arrays(nodes: np.ndarray, prim_entity: np.ndarray, prim_index: np.ndarray, depth: int = 0) -> Bvh:
    nodes = np.ascontiguousarray(nodes, dtype=np.float32).reshape(-1, 8)
    pe = np.ascontiguousarray(prim_entity, dtype=np.uint32)
    pi = np.ascontiguousarray(prim_index, dtype=np.uint32)
    d = BvhDesc(nodes.ctypes.data_as(C.POINTER(C.c_float)), nodes.shape[0], pe.shape[0],
                pe.ctypes.data_as(C.POINTER(C.c_uint32)), pi.ctypes.data_as(C.POINTER(C.c_uint32)))
    return Bvh(nodes, pe, pi, depth, d)


def camera_copy(cam: CameraDesc, **overrides) -> CameraDesc:
    c = CameraDesc()
    C.pointer(c)[0] = cam
    for k, v in overrides.items():
        if k in ("raster_to_camera", "camera_to_world"):
            getattr(c, k)[:] = [float(x) for x in np.asarray(v, dtype=np.float32).reshape(16)]
        else:
            setattr(c, k, v)
    return c


class Context:
    """One device context (rb_context): scene upload, ray tracing, rendering."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        check(lib().rb_context_create(C.byref(self._h), device), "rb_context_create")
        self.scene = None

    def close(self):
        if self._h:
            lib().rb_context_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def upload(self, scene: Scene) -> None:
        check(lib().rb_scene_upload(self._h, C.byref(scene.desc)), "rb_scene_upload")
        self.scene = scene

    def _trace(self, rays: np.ndarray, shadow: bool) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
        fn = lib().rb_trace_shadow if shadow else lib().rb_trace_closest
        check(fn(self._h, rays.ctypes.data, rays.shape[0], hits.ctypes.data), "rb_trace")
        return hits

    def trace_closest(self, rays: np.ndarray) -> np.ndarray:
        return self._trace(rays, False)

    def trace_shadow(self, rays: np.ndarray) -> np.ndarray:
        return self._trace(rays, True)

    def render(self, camera: CameraDesc, spp: int, first_sample: int = 0, max_depth: int = 5, threshold: float = 1.0,
               seed: int = 0, reset: bool = True, paths_per_wave: int = 0, want_image: bool = True,
               guide: bool = False, train: bool = False, volume: bool = False, out: np.ndarray = None,
               direct: tuple = None):
        """guide / train: learned path guiding (RB_RENDER_GUIDE / RB_RENDER_TRAIN); volume:
        volume_path_integrator instead of path_integrator (RB_RENDER_VOLUME); direct:
        (emitter_samples, bsdf_samples) renders with direct_integrator instead (RB_RENDER_DIRECT,
        the reference's default is (4, 4)). out: a
        C-contiguous float32 (height, width, 3) array to write the image into (when its memory
        is page-locked, slices are copied while later waves still run); returned instead of a
        new array."""
        p = RenderParams()
        p.camera = camera
        p.spp, p.first_sample, p.max_depth, p.rr_threshold = spp, first_sample, max_depth, threshold
        flags = (RB_RENDER_RESET if reset else 0) | (RB_RENDER_GUIDE if guide else 0) | (RB_RENDER_TRAIN if train else 0)
        flags |= RB_RENDER_VOLUME if volume else 0
        if direct is not None:
            flags |= RB_RENDER_DIRECT
            p.direct_samples = (int(direct[0]) & 0xFFFF) | ((int(direct[1]) & 0xFFFF) << 16)
        p.seed, p.flags, p.paths_per_wave = seed, flags, paths_per_wave
        if out is not None:
            if out.dtype != np.float32 or out.shape != (camera.height, camera.width, 3) or not out.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float32 array of shape (height, width, 3)")
            want_image = True
        img = out if out is not None else (np.zeros((camera.height, camera.width, 3), dtype=np.float32) if want_image else None)
        self._film_shape = (camera.width, camera.height)
        check(lib().rb_render(self._h, C.byref(p), img.ctypes.data if want_image else None), "rb_render")
        return img

    def render_photons(self, camera: CameraDesc, iterations: int = 64, max_depth: int = 5, photons: int = 0,
                       radius: float = 1.0, seed: int = 0) -> np.ndarray:
        """rb_render_photons: photon_mapping_integrator(iterations, max_depth, photons, radius)::render,
        stochastic progressive photon mapping; returns the (height, width, 3) image."""
        p = PhotonParams()
        p.camera = camera
        p.iterations, p.max_depth, p.photons, p.radius, p.seed = iterations, max_depth, photons, radius, seed
        img = np.zeros((camera.height, camera.width, 3), dtype=np.float32)
        check(lib().rb_render_photons(self._h, C.byref(p), img.ctypes.data), "rb_render_photons")
        return img

    def render_async(self, camera: CameraDesc, spp: int, first_sample: int = 0, max_depth: int = 5,
                     threshold: float = 1.0, seed: int = 0, reset: bool = False, paths_per_wave: int = 0,
                     out_ptr: int = 0) -> None:
        """rb_render_async: plain path tracing enqueued without waiting (calls overlap on the GPU; the film
        adds them in order). out_ptr: address of page-locked float32 (height, width, 3) memory for the image,
        or 0; it is complete at render_wait."""
        p = RenderParams()
        p.camera = camera
        p.spp, p.first_sample, p.max_depth, p.rr_threshold = spp, first_sample, max_depth, threshold
        p.seed, p.flags, p.paths_per_wave = seed, RB_RENDER_RESET if reset else 0, paths_per_wave
        self._film_shape = (camera.width, camera.height)
        check(lib().rb_render_async(self._h, C.byref(p), C.c_void_p(out_ptr) if out_ptr else None), "rb_render_async")

    def render_wait(self) -> None:
        """rb_render_wait: every pending render_async call has finished (first device error raised)."""
        check(lib().rb_render_wait(self._h), "rb_render_wait")

    def film(self):
        """(sum, sum_sq, count) FP64 accumulators of every pixel."""
        s = lib()
        cam = self._last_camera_shape()
        sum_ = np.zeros((cam[1], cam[0], 3), dtype=np.float64)
        sq = np.zeros_like(sum_)
        cnt = np.zeros((cam[1], cam[0]), dtype=np.uint32)
        check(s.rb_film_read(self._h, sum_.ctypes.data, sq.ctypes.data, cnt.ctypes.data), "rb_film_read")
        return sum_, sq, cnt

    def _last_camera_shape(self):
        if not hasattr(self, "_film_shape"):
            raise RbError(4, "film")
        return self._film_shape

    def stats(self) -> RenderStats:
        st = RenderStats()
        check(lib().rb_render_stats_get(self._h, C.byref(st)), "rb_render_stats_get")
        return st

    def set_counting(self, enabled: bool) -> None:
        check(lib().rb_set_counting(self._h, int(enabled)), "rb_set_counting")

    def set_profiling(self, enabled: bool) -> None:
        check(lib().rb_set_profiling(self._h, int(enabled)), "rb_set_profiling")

    def checkpoint_save(self, path: str) -> None:
        check(lib().rb_checkpoint_save(self._h, path.encode()), "rb_checkpoint_save")

    def checkpoint_load(self, path: str) -> None:
        check(lib().rb_checkpoint_load(self._h, path.encode()), "rb_checkpoint_load")

    # ---- learned path guiding
    def guide_init(self, seed: int = 0, learning_rate: float = 1e-3, batch_size: int = 1 << 18, steps_per_wave: int = 8,
                   max_samples: int = 1 << 21, min_rows: int = 4096, weight_clip: float = 0.0,
                   warmup_steps: int = 0) -> None:
        cfg = GuideConfig(seed, learning_rate, batch_size, steps_per_wave, max_samples, min_rows, weight_clip,
                          warmup_steps)
        check(lib().rb_guide_init(self._h, C.byref(cfg)), "rb_guide_init")

    def guide_params(self) -> np.ndarray:
        out = np.zeros(RB_GUIDE_NUM_PARAMS, dtype=np.float32)
        check(lib().rb_guide_get_params(self._h, out.ctypes.data, out.size), "rb_guide_get_params")
        return out

    def guide_set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, dtype=np.float32)
        check(lib().rb_guide_set_params(self._h, params.ctypes.data, params.size), "rb_guide_set_params")

    def guide_forward(self, inputs: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, 9)
        out = np.zeros((x.shape[0], RB_GUIDE_OUTPUTS), dtype=np.float32)
        check(lib().rb_guide_forward(self._h, x.ctypes.data, x.shape[0], out.ctypes.data), "rb_guide_forward")
        return out

    def guide_train(self, samples: np.ndarray, steps: int = 1, sequential: bool = False):
        """Training steps on host samples (GUIDE_SAMPLE_DTYPE); returns (gradient of the last step, its loss)."""
        samples = np.ascontiguousarray(samples, dtype=GUIDE_SAMPLE_DTYPE)
        grad = np.zeros(RB_GUIDE_NUM_PARAMS, dtype=np.float32)
        loss = C.c_float()
        check(lib().rb_guide_train(self._h, samples.ctypes.data, samples.shape[0], steps,
                                   RB_GUIDE_SEQUENTIAL if sequential else 0, grad.ctypes.data, C.byref(loss)),
              "rb_guide_train")
        return grad, loss.value

    def guide_sample(self, outputs: np.ndarray, u: np.ndarray):
        """Decode raw outputs and draw one direction per row; returns (directions, guide pdf)."""
        raw = np.ascontiguousarray(outputs, dtype=np.float32).reshape(-1, RB_GUIDE_OUTPUTS)
        uu = np.ascontiguousarray(u, dtype=np.float32).reshape(-1, 3)
        d = np.zeros((raw.shape[0], 3), dtype=np.float32)
        pdf = np.zeros(raw.shape[0], dtype=np.float32)
        check(lib().rb_guide_sample_dirs(self._h, raw.ctypes.data, uu.ctypes.data, raw.shape[0], d.ctypes.data,
                                         pdf.ctypes.data), "rb_guide_sample_dirs")
        return d, pdf

    def guide_stats(self) -> GuideStats:
        st = GuideStats()
        check(lib().rb_guide_stats_get(self._h, C.byref(st)), "rb_guide_stats_get")
        return st

    def guide_medium_stats(self) -> GuideStats:
        """Counters of the medium guide of guided volume renders."""
        st = GuideStats()
        check(lib().rb_guide_medium_stats_get(self._h, C.byref(st)), "rb_guide_medium_stats_get")
        return st


    # ---- launch tuning (rb_set_tuning / rb_tune_render)
    def set_tuning(self, tuning: Tuning | None = None, **fields) -> None:
        t = Tuning()
        if tuning is not None:
            C.pointer(t)[0] = tuning
        for k, v in fields.items():
            setattr(t, k, v)
        check(lib().rb_set_tuning(self._h, C.byref(t)), "rb_set_tuning")

    def tuning(self) -> Tuning:
        t = Tuning()
        check(lib().rb_get_tuning(self._h, C.byref(t)), "rb_get_tuning")
        return t

    def tune_render(self, camera: CameraDesc, probe_spp: int = 1, max_depth: int = 5, threshold: float = 1.0,
                    seed: int = 0, volume: bool = False, direct: tuple = None):
        """Autotune the launch shapes on `probe_spp` samples per pixel (of a volume or direct-lighting
        render when asked); returns (Tuning, ms)."""
        p = RenderParams()
        p.camera = camera
        p.spp, p.max_depth, p.rr_threshold, p.seed = probe_spp, max_depth, threshold, seed
        p.flags = RB_RENDER_VOLUME if volume else 0
        if direct is not None:
            p.flags |= RB_RENDER_DIRECT
            p.direct_samples = (int(direct[0]) & 0xFFFF) | ((int(direct[1]) & 0xFFFF) << 16)
        t, ms = Tuning(), C.c_float()
        check(lib().rb_tune_render(self._h, C.byref(p), probe_spp, C.byref(t), C.byref(ms)), "rb_tune_render")
        self._film_shape = (camera.width, camera.height)
        return t, float(ms.value)

    # ---- batched rendering (rb_batch_*)
    def batch_upload(self, scenes) -> None:
        """Upload many scenes at once (rb_batch_upload); replaces any scene."""
        scenes = list(scenes)
        arr = (SceneDesc * len(scenes))()
        for k, sc in enumerate(scenes):
            arr[k] = sc.desc
        check(lib().rb_batch_upload(self._h, arr, len(scenes)), "rb_batch_upload")
        self.batch_scenes = scenes
        self.scene = None

    def _batch_params(self, views, max_depth, threshold, reset, order):
        arr = (BatchView * len(views))()
        for k, v in enumerate(views):
            arr[k].camera = v["camera"]
            arr[k].spp = v["spp"]
            arr[k].first_sample = v.get("first_sample", 0)
            arr[k].seed = v.get("seed", 0)
        p = BatchParams()
        p.views = arr
        p.count = len(views)
        p.max_depth, p.rr_threshold, p.flags = max_depth, threshold, RB_RENDER_RESET if reset else 0
        keep = [arr]
        if order is not None:
            o = (C.c_uint32 * len(order))(*[int(x) for x in order])
            p.order = o
            keep.append(o)
        return p, keep

    def batch_render(self, views, max_depth: int = 5, threshold: float = 1.0, reset: bool = True, order=None):
        """Render every uploaded scene (views: dicts of camera, spp, first_sample, seed);
        returns each scene's completion time in ms from the call's start."""
        p, keep = self._batch_params(views, max_depth, threshold, reset, order)
        ms = np.zeros(len(views), dtype=np.float32)
        check(lib().rb_batch_render(self._h, C.byref(p), ms.ctypes.data), "rb_batch_render")
        self._batch_shapes = [(v["camera"].width, v["camera"].height) for v in views]
        return ms

    def tune_batch(self, views, probe_items: int, max_depth: int = 5, threshold: float = 1.0, order=None):
        p, keep = self._batch_params(views, max_depth, threshold, True, order)
        t, ms = Tuning(), C.c_float()
        check(lib().rb_tune_batch(self._h, C.byref(p), int(probe_items), C.byref(t), C.byref(ms)), "rb_tune_batch")
        self._batch_shapes = [(v["camera"].width, v["camera"].height) for v in views]
        return t, float(ms.value)

    def batch_film(self, scene: int):
        w, h = self._batch_shapes[scene]
        sum_ = np.zeros((h, w, 3), dtype=np.float64)
        sq = np.zeros_like(sum_)
        cnt = np.zeros((h, w), dtype=np.uint32)
        check(lib().rb_batch_film_read(self._h, scene, sum_.ctypes.data, sq.ctypes.data, cnt.ctypes.data),
              "rb_batch_film_read")
        return sum_, sq, cnt

    def batch_image(self, scene: int) -> np.ndarray:
        w, h = self._batch_shapes[scene]
        img = np.zeros((h, w, 3), dtype=np.float32)
        check(lib().rb_batch_image(self._h, scene, img.ctypes.data), "rb_batch_image")
        return img


    # ---- failure detection
    def check_bounded_wait(self, limit_us: int) -> int:
        """Runs one bounded device wait that nothing completes; returns the status it led to."""
        st = C.c_int32()
        check(lib().rb_check_bounded_wait(self._h, limit_us, C.byref(st)), "rb_check_bounded_wait")
        return st.value


def inject_allocation_failure(after: int) -> None:
    """The `after`-th device allocation from now on fails as out-of-memory (after < 0: off)."""
    lib().rb_inject_allocation_failure(after)


class PathIntegrator:
    """path_integrator(sampler2d(spp), sampler1d, max_depth=5, threshold=1) on the GPU."""

    def __init__(self, spp: int, max_depth: int = 5, threshold: float = 1.0, seed: int = 0, device: int = 0):
        self.spp, self.max_depth, self.threshold, self.seed = spp, max_depth, threshold, seed
        self.context = Context(device)
        self._uploaded = None

    def render(self, camera: CameraDesc, scene: Scene) -> np.ndarray:
        if self._uploaded is not scene:
            self.context.upload(scene)
            self._uploaded = scene
        return self.context.render(camera, self.spp, max_depth=self.max_depth, threshold=self.threshold, seed=self.seed)
