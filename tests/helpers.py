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


class HostPaths:
    """Stage functions of the kernels compiled for the host (bit-exact reference arithmetic)."""

    def __init__(self, scene: rb.Scene):
        L = C.CDLL(HOSTPATHS)
        L.hp_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.hp_free.argtypes = [C.c_void_p]
        L.hp_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        L.hp_samples.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                                 C.c_uint32, C.c_void_p]
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


def assert_hits_equal(got, want, what=""):
    assert np.array_equal(got["entity"], want["entity"]), f"{what}: entity ids differ at " \
        f"{np.flatnonzero(got['entity'] != want['entity'])[:8]}"
    assert np.array_equal(got["triangle"], want["triangle"]), f"{what}: triangle ids differ"
    bad = got["t"].view(np.uint32) != want["t"].view(np.uint32)
    assert not bad.any(), f"{what}: {bad.sum()} hit distances differ in their bits"
