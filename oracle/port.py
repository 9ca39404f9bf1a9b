"""ctypes wrapper of oracle/_ref/liboracle_port.so, the plain-C restatement of
the reference path integrator (oracle/restate/rb_port.c). TEST INFRASTRUCTURE
ONLY: used as a checker by the tests and as the port CPU baseline."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle_port.so")
_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(LIB_PATH)
        vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
        L.port_pcg32.argtypes = [C.c_uint64, u32, vp, vp]
        L.port_trace.argtypes = [vp, vp, u32, i32, vp]
        L.port_samples.argtypes = [vp, vp, vp, vp, u32, u32, f32, u32, vp]
        L.port_render.argtypes = [vp, vp, u32, u32, u32, f32, u32, i32, i32, i32, vp, vp, C.POINTER(C.c_double)]
        for f in (L.port_pcg32, L.port_trace, L.port_samples, L.port_render):
            f.restype = i32
        _LIB = L
    return _LIB


def _ok(st, where):
    if st != 0:
        raise RuntimeError(f"{where} returned {st}")


def pcg32(seed, n):
    u = np.zeros(n, dtype=np.uint32)
    r = np.zeros(n, dtype=np.float32)
    _ok(lib().port_pcg32(seed, n, u.ctypes.data, r.ctypes.data), "port_pcg32")
    return u, r


def scene_with_bvh(scene, bvh):
    """The scene description carrying a flattened tree (the port walks it)."""
    return scene.with_bvh(bvh)


def trace(scene, rays, shadow=False):
    from rainbow_b200 import HIT_DTYPE, RAY_DTYPE
    rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
    hits = np.zeros(rays.shape[0], dtype=HIT_DTYPE)
    _ok(lib().port_trace(C.byref(scene.desc), rays.ctypes.data, rays.shape[0], int(shadow), hits.ctypes.data), "port_trace")
    return hits


def samples(scene, camera, pixels, samples_, max_depth, rr=1.0, seed=0):
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    sm = np.ascontiguousarray(samples_, dtype=np.uint32)
    out = np.zeros((px.shape[0], 3), dtype=np.float32)
    _ok(lib().port_samples(C.byref(scene.desc), C.byref(camera), px.ctypes.data, sm.ctypes.data, px.shape[0], max_depth,
                           rr, seed, out.ctypes.data), "port_samples")
    return out


def render(scene, camera, spp, first_sample=0, max_depth=5, rr=1.0, seed=0, threads=1, rows=(0, 0)):
    s = np.zeros((camera.height, camera.width, 3), dtype=np.float64)
    q = np.zeros_like(s)
    sec = C.c_double()
    _ok(lib().port_render(C.byref(scene.desc), C.byref(camera), spp, first_sample, max_depth, rr, seed, threads, rows[0],
                          rows[1], s.ctypes.data, q.ctypes.data, C.byref(sec)), "port_render")
    return s, q, sec.value
