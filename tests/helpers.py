"""Shared test helpers: scene regeneration from fixture parameters and the
test-only host build of the stage functions (tests/native/libhostpaths.so)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

import rainbow_b200 as rb

HERE = os.path.dirname(os.path.abspath(__file__))
HOSTPATHS = os.path.join(HERE, "native", "libhostpaths.so")


def scene_from_params(params) -> rb.Scene:
    kind, seed, w, h, n, sub = (int(x) for x in params)
    return rb.generate_scene(kind, seed=seed, width=w, height=h, num_spheres=n, subdivision=sub)


def extra_materials_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with every fourth material (from the second) plastic, every
    fourth (from the third) a mirror and every eighth (from the fourth) a
    substrate; the rest unchanged."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if k % 4 == 1:
            src = m
            m = rb.MaterialDesc()
            m.kind = rb.RB_MATERIAL_PLASTIC
            m.diffuse[:] = (0.6, 0.3, 0.2) if k % 8 == 1 else (0.0, 0.0, 0.0)
            m.reflectance[:] = (0.5, 0.45, 0.4)
            m.roughness_u = 0.05 + 0.1 * (k % 5)
            m.remap_roughness = 1
            m.ior = 1.49
            del src
        elif k % 4 == 2:
            m = rb.MaterialDesc()
            m.kind = rb.RB_MATERIAL_MIRROR
            m.reflectance[:] = (0.9, 0.85, 0.8)
        elif k % 8 == 3:
            m = rb.MaterialDesc()
            m.kind = rb.RB_MATERIAL_SUBSTRATE
            m.diffuse[:] = (0.5, 0.35, 0.2)
            m.reflectance[:] = (0.05, 0.05, 0.05)
            m.roughness_u, m.roughness_v = 0.1, 0.25
            m.remap_roughness = 1
        mats.append(m)
    return scene.with_materials(mats)


class HostPaths:
    """Stage functions of the kernels compiled for the host (bit-exact reference arithmetic)."""

    def __init__(self, scene: rb.Scene):
        L = C.CDLL(HOSTPATHS)
        L.hp_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.hp_free.argtypes = [C.c_void_p]
        L.hp_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        L.hp_samples.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                                 C.c_uint32, C.c_void_p]
        L.hp_direct_samples.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                        C.c_uint32, C.c_uint32, C.c_void_p]
        L.hp_direct_staged_samples.argtypes = L.hp_direct_samples.argtypes
        self.L, self.scene = L, scene
        self.h = C.c_void_p()
        assert L.hp_create(C.byref(scene.desc), C.byref(self.h)) == 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.hp_free(self.h)
            self.h = None

    def trace(self, rays, shadow=False):
        rays = np.ascontiguousarray(rays, dtype=rb.RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=rb.HIT_DTYPE)
        self.L.hp_trace(self.h, rays.ctypes.data, rays.shape[0], int(shadow), hits.ctypes.data)
        return hits

    def samples(self, camera, pixels, samples, max_depth, rr=1.0, seed=0):
        px = np.ascontiguousarray(pixels, dtype=np.uint32)
        sm = np.ascontiguousarray(samples, dtype=np.uint32)
        out = np.zeros((px.shape[0], 3), dtype=np.float32)
        self.L.hp_samples(self.h, C.byref(camera), px.ctypes.data, sm.ctypes.data, px.shape[0], max_depth, rr, seed,
                          out.ctypes.data)
        return out


    def direct_samples(self, camera, pixels, samples, emitter_samples=4, bsdf_samples=4, seed=0, staged=False):
        """direct_integrator radiance of (pixel, sample) pairs on the host: pt::direct_radiance, or
        (staged) its stage functions in the staged kernels' order."""
        px = np.ascontiguousarray(pixels, dtype=np.uint32)
        sm = np.ascontiguousarray(samples, dtype=np.uint32)
        out = np.zeros((px.shape[0], 3), dtype=np.float32)
        fn = self.L.hp_direct_staged_samples if staged else self.L.hp_direct_samples
        assert fn(self.h, C.byref(camera), px.ctypes.data, sm.ctypes.data, px.shape[0], emitter_samples, bsdf_samples,
                  seed, out.ctypes.data) == 0
        return out


def assert_hits_equal(got, want, what=""):
    assert np.array_equal(got["entity"], want["entity"]), f"{what}: entity ids differ at " \
        f"{np.flatnonzero(got['entity'] != want['entity'])[:8]}"
    assert np.array_equal(got["triangle"], want["triangle"]), f"{what}: triangle ids differ"
    bad = got["t"].view(np.uint32) != want["t"].view(np.uint32)
    assert not bad.any(), f"{what}: {bad.sum()} hit distances differ in their bits"


class HostBatch:
    """Several scenes merged as rb_batch_upload merges them, on the host build of the stages."""

    def __init__(self, scenes):
        L = C.CDLL(HOSTPATHS)
        L.hp_batch_create.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]
        L.hp_batch_free.argtypes = [C.c_void_p]
        L.hp_batch_trace.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        L.hp_batch_samples.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                       C.c_uint32, C.c_float, C.c_uint32, C.c_void_p]
        self.L, self.scenes = L, list(scenes)
        arr = (rb.SceneDesc * len(self.scenes))()
        for k, sc in enumerate(self.scenes):
            arr[k] = sc.desc
        self.h = C.c_void_p()
        assert L.hp_batch_create(arr, len(self.scenes), C.byref(self.h)) == 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.hp_batch_free(self.h)
            self.h = None

    def trace(self, scene, rays, shadow=False):
        rays = np.ascontiguousarray(rays, dtype=rb.RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=rb.HIT_DTYPE)
        assert self.L.hp_batch_trace(self.h, scene, rays.ctypes.data, rays.shape[0], int(shadow), hits.ctypes.data) == 0
        return hits

    def samples(self, scene, camera, pixels, samples, max_depth, rr=1.0, seed=0):
        px = np.ascontiguousarray(pixels, dtype=np.uint32)
        sm = np.ascontiguousarray(samples, dtype=np.uint32)
        out = np.zeros((px.shape[0], 3), dtype=np.float32)
        assert self.L.hp_batch_samples(self.h, scene, C.byref(camera), px.ctypes.data, sm.ctypes.data, px.shape[0],
                                       max_depth, rr, seed, out.ctypes.data) == 0
        return out


def random_rays(scene, n, seed):
    """Rays toward random surface points of the scene: half from the camera eye,
    half from other surface points (as bounce rays leave surfaces); length +inf."""
    rng = np.random.default_rng(seed)
    d = scene.desc
    pts = []
    for e in range(d.num_entities):
        ent = d.entities[e]
        if ent.mesh < 0:
            continue
        md = d.meshes[ent.mesh]
        P = np.ctypeslib.as_array(md.positions, (md.num_vertices * 3,)).reshape(-1, 3).astype(np.float64)
        I = np.ctypeslib.as_array(md.indices, (md.num_triangles * 3,)).reshape(-1, 3)
        t = rng.integers(0, md.num_triangles, 64)
        u, v = rng.random(64), rng.random(64)
        flip = u + v > 1
        u[flip], v[flip] = 1 - u[flip], 1 - v[flip]
        local = P[I[t, 0]] * (1 - u - v)[:, None] + P[I[t, 1]] * u[:, None] + P[I[t, 2]] * v[:, None]
        M = np.array(ent.local_to_world[:], dtype=np.float64).reshape(4, 4).T  # column-major storage
        pts.append(local @ M[:3, :3].T + M[:3, 3])
    pts = np.concatenate(pts)
    targets = pts[rng.integers(0, len(pts), n)]
    eye = np.array(scene.camera.eye[:], dtype=np.float64)
    origins = np.repeat(eye[None], n, axis=0)
    half = n // 2
    origins[half:] = pts[rng.integers(0, len(pts), n - half)] + rng.normal(scale=1e-2, size=(n - half, 3))
    dirs = targets - origins
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.zeros(n, dtype=rb.RAY_DTYPE)
    rays["origin"] = origins.astype(np.float32)
    rays["direction"] = dirs.astype(np.float32)
    rays["length"] = np.inf
    return rays
