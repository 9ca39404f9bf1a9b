"""Shared test helpers: scene regeneration from fixture parameters and the
test-only host build of the stage functions (tests/native/libhostpaths.so)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

import rainbow_b200 as rb
from rainbow_b200 import _native

HERE = os.path.dirname(os.path.abspath(__file__))
HOSTPATHS = os.path.join(HERE, "native", "libhostpaths.so")


def scene_from_params(params) -> rb.Scene:
    kind, seed, w, h, n, sub = (int(x) for x in params)
    return rb.generate_scene(kind, seed=seed, width=w, height=h, num_spheres=n, subdivision=sub)


def material_from_bytes(raw: bytes, count: int = 1):
    """Material descriptors from a fixture's bytes (`count` of them, a mixture
    and its components when more than one); fields added to the descriptor
    after the fixture was written (at its end) read as zero."""
    size = C.sizeof(rb.MaterialDesc)
    raw = bytes(raw)
    old = len(raw) // count
    parts = [raw[k * old:(k + 1) * old][:size].ljust(size, b"\0") for k in range(count)]
    if count == 1:
        return rb.MaterialDesc.from_buffer_copy(parts[0])
    return (rb.MaterialDesc * count).from_buffer_copy(b"".join(parts))


_LOBE_NAMES = {0: "lambert", 1: "microfacet_reflection", 2: "microfacet_transmission", 3: "fresnel_specular",
               4: "specular_reflection", 5: "fresnel_blend", 6: "oren_nayar", 7: "lambert",
               8: "lambert_transmission", 9: "microfacet_reflection", 10: "microfacet_transmission",
               11: "specular_reflection", 12: "specular_transmission"}


def material_lobes(md: rb.MaterialDesc) -> list:
    """Names of the lobes that the host packing of one material gives, in
    collection order (host build of the kernels' make_bsdf)."""
    L = C.CDLL(HOSTPATHS)
    L.hp_material_lobes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    kinds = (C.c_uint32 * 8)()
    n = C.c_uint32(0)
    rb.check(L.hp_material_lobes(C.byref(md), kinds, C.byref(n)), "hp_material_lobes")
    return [_LOBE_NAMES[kinds[i]] for i in range(n.value)]


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

    def photon_render(self, camera, iterations, max_depth=5, photons=0, radius=1.0, streams=0, seed=0):
        """photon_mapping_integrator::render through the photon stage functions: streams 0 in the
        reference's order and streams (bit-equal to it), 1 with the kernels' per-pixel and
        per-photon streams. Returns the (height, width, 3) image."""
        self.L.hp_photon_render.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                            C.c_int, C.c_uint32, C.c_void_p]
        out = np.zeros((camera.height, camera.width, 3), dtype=np.float32)
        assert self.L.hp_photon_render(self.h, C.byref(camera), iterations, max_depth, photons, radius, streams, seed,
                                       out.ctypes.data) == 0
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


def _normalize32(x, y, z):
    inv = np.float32(1.0) / np.sqrt((x * x + y * y) + z * z)
    return x * inv, y * inv, z * inv


def camera_ray_batch(camera, n, seed):
    """n seeded camera rays of `camera`: raster point (x + u, y + v) of a random
    pixel through raster_to_camera, normalised, then camera_to_world. Written as
    element-wise float32 operations (each exactly rounded, no FMA, no BLAS), so
    the batch is the same on every host."""
    rng = np.random.default_rng(seed)
    W, H = camera.width, camera.height
    px = rng.integers(0, W * H, n)
    jit = rng.random((n, 2)).astype(np.float32)
    fx = (px % W).astype(np.float32) + jit[:, 0]
    fy = (px // W).astype(np.float32) + jit[:, 1]
    R = np.array(camera.raster_to_camera[:], dtype=np.float32)
    Cw = np.array(camera.camera_to_world[:], dtype=np.float32)
    cx, cy, cz = ((R[r] * fx + R[4 + r] * fy) + R[12 + r] for r in range(3))
    cx, cy, cz = _normalize32(cx, cy, cz)
    dx, dy, dz = ((Cw[r] * cx + Cw[4 + r] * cy) + Cw[8 + r] * cz for r in range(3))
    dx, dy, dz = _normalize32(dx, dy, dz)
    rays = np.zeros(n, dtype=rb.RAY_DTYPE)
    rays["origin"] = np.array([Cw[12], Cw[13], Cw[14]], dtype=np.float32)
    rays["direction"] = np.stack([dx, dy, dz], axis=1)
    rays["length"] = np.inf
    return rays


def bounce_ray_batch(rays, hits, seed):
    """One secondary ray from every hit of `rays`: origin at the hit point
    o + t d stepped back toward the ray's origin by 1e-3 (1 + max |p|), direction
    uniform over the hemisphere facing back along the ray (the side the ray came
    from), length +inf. Element-wise float32 arithmetic on the given hits, so two
    hosts with the same hits make the same rays."""
    sel = np.flatnonzero(hits["entity"] >= 0)
    o, d, t = rays["origin"][sel], rays["direction"][sel], hits["t"][sel]
    p = o + t[:, None] * d
    step = np.float32(1e-3) * (np.float32(1.0) + np.abs(p).max(axis=1))
    org = p - d * step[:, None]
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(sel.shape[0], 3))
    norm = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
    v = (v / norm[:, None]).astype(np.float32)
    facing = (v[:, 0] * d[:, 0] + v[:, 1] * d[:, 1]) + v[:, 2] * d[:, 2]
    v[facing > 0] *= np.float32(-1.0)
    out = np.zeros(sel.shape[0], dtype=rb.RAY_DTYPE)
    out["origin"], out["direction"], out["length"] = org, v, np.inf
    return out


def ray_levels(camera, trace, n0, seed, levels=3):
    """Camera rays, then levels - 1 generations of bounce rays from the previous
    generation's hits; trace(rays) -> hits. Returns [(rays, hits)] per level."""
    out = []
    rays = camera_ray_batch(camera, n0, seed)
    for k in range(levels):
        hits = trace(rays)
        out.append((rays, hits))
        if k + 1 < levels:
            rays = bounce_ray_batch(rays, hits, seed + 1 + k)
    return out


def hit_digests(hits, chunk=4096):
    """SHA-256 per chunk of `chunk` hits over entity, triangle and the bits of t."""
    import hashlib
    out = []
    for a in range(0, hits.shape[0], chunk):
        h = hashlib.sha256()
        b = hits[a:a + chunk]
        for col in (b["entity"].astype(np.int32), b["triangle"].astype(np.int32), b["t"].astype(np.float32).view(np.uint32)):
            h.update(np.ascontiguousarray(col).tobytes())
        out.append(h.hexdigest()[:16])
    return np.array(out)


SAMPLE_RTOL = 1e-3  # per-channel agreement of one sample: |a - b| <= 1e-3 * max(1, |b|)


def sample_agreement(got, want):
    """Per sample: every channel within SAMPLE_RTOL of the reference."""
    return (np.abs(got - want) <= SAMPLE_RTOL * np.maximum(1.0, np.abs(want))).all(axis=1)


def _material_kind(scene, entity):
    if entity < 0:
        return "miss"
    e = scene.desc.entities[int(entity)]
    if e.material < 0:
        return "invisible"
    return {0: "matte", 1: "metal", 2: "glass", 3: "plastic", 4: "mirror", 5: "substrate"}.get(
        scene.desc.materials[e.material].kind, "other")


def assert_disagreements_unbiased(scene, got, want, first_entity, what=""):
    """The samples that differ from the reference (paths that diverged where
    CUDA's and glibc's transcendental functions round differently) must scatter
    around it without a systematic sign, overall and per material of the first
    hit: with d the luminance difference of each disagreeing sample,
    |sum d| <= 4 sqrt(sum d^2) (a zero-mean sum of n terms has that spread), and
    the count of d > 0 is within 4 sigma of n / 2."""
    ok = sample_agreement(got, want)
    lum = np.array([0.212671, 0.715160, 0.072169])
    d = (got.astype(np.float64) - want.astype(np.float64)) @ lum
    kinds = np.array([_material_kind(scene, e) for e in first_entity])
    groups = [("all", np.ones_like(ok))] + [(k, kinds == k) for k in np.unique(kinds)]
    for name, sel in groups:
        m = sel & ~ok & (d != 0)
        n = int(m.sum())
        if n < 8:
            continue
        dd = d[m]
        assert abs(dd.sum()) <= 4.0 * np.sqrt((dd ** 2).sum()), \
            f"{what}: {n} disagreeing samples on {name} are biased (sum {dd.sum():.4g}, rms {np.sqrt((dd ** 2).mean()):.4g})"
        pos = int((dd > 0).sum())
        assert abs(pos - n / 2) <= 4.0 * np.sqrt(n / 4), f"{what}: {pos} of {n} disagreeing samples on {name} are higher"


def per_sample_radiance(ctx, scene, pixels, samples, depth, volume=False):
    """Radiance of (pixel, sample) pairs: one one-sample render per distinct sample index."""
    got = np.zeros((pixels.shape[0], 3), dtype=np.float32)
    for s in np.unique(samples):
        ctx.render(scene.camera, spp=1, first_sample=int(s), max_depth=depth, want_image=False, volume=volume)
        sums, _, cnt = ctx.film()
        sel = samples == s
        got[sel] = sums.reshape(-1, 3)[pixels[sel]]
        assert (cnt.reshape(-1)[pixels[sel]] == 1).all()
    return got


def block_z(mean, ref_mean, ref_var, n, n_ref, block=4, var=None):
    """z-scores of block means (block x block pixels, per channel) of an n-spp
    render against an n_ref-spp reference. The standard error uses each
    render's own per-sample variance (var for the render; without it the
    reference's stands for both). In heavy-tailed scenes the reference's own
    estimate alone is too small wherever its samples missed the rare bright
    paths: two independent reference renders of the slit room at 1024 spp then
    put 4.8% of 4 x 4 blocks outside 3 sigma (mean z 0.30), and 0% with both
    variances."""
    H, W, _ = mean.shape
    h, w = H // block * block, W // block * block

    def blocks(a):
        return a[:h, :w].reshape(h // block, block, w // block, block, 3)

    bm = blocks(mean).mean(axis=(1, 3))
    br = blocks(ref_mean).mean(axis=(1, 3))
    bv_ref = blocks(ref_var).sum(axis=(1, 3)) / block ** 4
    bv = bv_ref if var is None else blocks(var).sum(axis=(1, 3)) / block ** 4
    se = np.sqrt(bv / n + bv_ref / n_ref)
    return np.where(se > 0, (bm - br) / np.where(se > 0, se, 1), 0.0)


def two_level_scene(width=64, height=48):
    """A scene that needs the reference's two-level tree (scene.cpp:41-75): the
    seeded sphere field of 6 spheres (1,280 triangles each) with spheres 1 and 2
    sharing sphere 1's mesh (each keeps its own transform), plus one sphere of
    327,680 triangles (icosphere subdivision 7, more than 2^17) taken from a
    second seeded scene. Meshes used by one entity and below 2^17 triangles
    keep one leaf per triangle."""
    base = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=9, width=width, height=height, num_spheres=6, subdivision=3)
    big = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=10, width=width, height=height, num_spheres=1, subdivision=7)
    d = base.desc
    meshes = [_native.MeshDesc.from_buffer_copy(bytes(d.meshes[i])) for i in range(d.num_meshes)]
    ents = [_native.EntityDesc.from_buffer_copy(bytes(d.entities[i])) for i in range(d.num_entities)]
    sphere_ents = [k for k, e in enumerate(ents) if e.mesh >= 0 and e.emitter < 0 and
                   d.meshes[e.mesh].num_triangles == 1280]
    a, b = sphere_ents[1], sphere_ents[2]
    ents[b].mesh = ents[a].mesh
    bd = big.desc
    big_ent = next(k for k in range(bd.num_entities) if bd.entities[k].mesh >= 0 and
                   bd.meshes[bd.entities[k].mesh].num_triangles == 327680)
    meshes.append(_native.MeshDesc.from_buffer_copy(bytes(bd.meshes[bd.entities[big_ent].mesh])))
    e = _native.EntityDesc.from_buffer_copy(bytes(bd.entities[big_ent]))
    e.mesh = len(meshes) - 1
    e.material = ents[sphere_ents[0]].material
    e.emitter = -1
    ents.append(e)
    mesh_arr = (_native.MeshDesc * len(meshes))(*meshes)
    ent_arr = (_native.EntityDesc * len(ents))(*ents)
    nd = rb.SceneDesc()
    C.pointer(nd)[0] = d
    nd.meshes = C.cast(mesh_arr, type(nd.meshes))
    nd.num_meshes = len(meshes)
    nd.entities = C.cast(ent_arr, type(nd.entities))
    nd.num_entities = len(ents)
    return rb.Scene(None, nd, base.camera, keepalive=[base, big, mesh_arr, ent_arr])



def layered_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with every third material (from the second, the floor's) an
    uber material (uber_material.cpp; opacity below one on every other one, so
    that its pass-through specular transmission is in the lobe list) and every
    third (from the first) a translucent material (translucent_material.cpp;
    every fourth of those without its specular lobes); the rest unchanged."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if k % 3 == 1:
            m = rb.MaterialDesc()
            m.kind = rb.RB_MATERIAL_UBER
            m.remap_roughness = 1
            m.diffuse[:] = (0.5, 0.3, 0.2)
            m.specular[:] = (0.3, 0.3, 0.25)
            m.reflectance[:] = (0.1, 0.1, 0.1) if k % 4 == 1 else (0.0, 0.0, 0.0)
            m.transmission[:] = (0.2, 0.25, 0.3) if k % 5 == 1 else (0.0, 0.0, 0.0)
            m.opacity[:] = (0.7, 0.8, 0.9) if k % 2 == 1 else (1.0, 1.0, 1.0)
            m.roughness_u, m.roughness_v = 0.1 + 0.05 * (k % 4), 0.2
            m.ior = 1.5
        elif k % 3 == 0:
            m = rb.MaterialDesc()
            m.kind = rb.RB_MATERIAL_TRANSLUCENT
            m.remap_roughness = 1
            m.diffuse[:] = (0.6, 0.5, 0.4)
            m.specular[:] = (0.0, 0.0, 0.0) if k % 4 == 0 else (0.4, 0.4, 0.4)
            m.reflectance[:] = (0.5, 0.5, 0.5)
            m.transmission[:] = (0.4, 0.45, 0.5)
            m.roughness_u = m.roughness_v = 0.15 + 0.05 * (k % 3)  # translucent reads roughness_u alone
        mats.append(m)
    return scene.with_materials(mats)


def _desc(kind, **kw) -> rb.MaterialDesc:
    m = rb.MaterialDesc()
    m.kind = kind
    for k, v in kw.items():
        if isinstance(v, tuple):
            getattr(m, k)[:] = v
        else:
            setattr(m, k, v)
    return m


def mixture_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with every third material (from the second, the floor's) a
    mixture (mixture_material.cpp) of two component materials appended after
    the scene's own: Oren-Nayar matte with metal, translucent with smooth
    glass, uber with metal, and a mixture of plastic and mirror mixed with
    substrate (nested), in turn; the rest unchanged."""
    mats = [rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k])) for k in range(scene.desc.num_materials)]
    n = len(mats)
    extra = []

    def add(m):
        extra.append(m)
        return n + len(extra) - 1

    metal = dict(remap_roughness=1, eta=(0.200438, 0.924033, 1.102212), k=(3.912949, 2.452848, 2.142188),
                 roughness_u=0.2, roughness_v=0.3)
    for k in range(1, n, 3):
        variant = (k // 3) % 4
        if variant == 0:
            c = (add(_desc(rb.RB_MATERIAL_MATTE, diffuse=(0.7, 0.5, 0.3), sigma=25.0)),
                 add(_desc(rb.RB_MATERIAL_METAL, **metal)))
        elif variant == 1:
            c = (add(_desc(rb.RB_MATERIAL_TRANSLUCENT, remap_roughness=1, diffuse=(0.6, 0.5, 0.4),
                           specular=(0.4, 0.4, 0.4), reflectance=(0.5, 0.5, 0.5), transmission=(0.4, 0.45, 0.5),
                           roughness_u=0.2, roughness_v=0.2)),
                 add(_desc(rb.RB_MATERIAL_GLASS, reflectance=(1.0, 1.0, 1.0), transmission=(1.0, 1.0, 1.0), ior=1.5)))
        elif variant == 2:
            c = (add(_desc(rb.RB_MATERIAL_UBER, remap_roughness=1, diffuse=(0.5, 0.3, 0.2), specular=(0.3, 0.3, 0.25),
                           reflectance=(0.1, 0.1, 0.1), opacity=(0.8, 0.9, 1.0), roughness_u=0.15, roughness_v=0.2,
                           ior=1.5)),
                 add(_desc(rb.RB_MATERIAL_METAL, **metal)))
        else:
            inner = add(_desc(rb.RB_MATERIAL_MIXTURE, amount=(0.5, 0.6, 0.7),
                              components=(add(_desc(rb.RB_MATERIAL_PLASTIC, remap_roughness=1, diffuse=(0.6, 0.3, 0.2),
                                                    reflectance=(0.5, 0.45, 0.4), roughness_u=0.1, ior=1.49)),
                                          add(_desc(rb.RB_MATERIAL_MIRROR, reflectance=(0.9, 0.85, 0.8))))))
            c = (inner, add(_desc(rb.RB_MATERIAL_SUBSTRATE, remap_roughness=1, diffuse=(0.5, 0.35, 0.2),
                                  reflectance=(0.05, 0.05, 0.05), roughness_u=0.1, roughness_v=0.25)))
        mats[k] = _desc(rb.RB_MATERIAL_MIXTURE, amount=(0.25 + 0.1 * (k % 3), 0.5, 0.75), components=c)
    return scene.with_materials(mats + extra)


def texture_images():
    """Two seeded RGB images: 16 x 8 random texels and a 5 x 3 checker of two colours."""
    rng = np.random.default_rng(23)
    noise = rng.random((8, 16, 3), dtype=np.float32) * 0.8 + 0.1
    yy, xx = np.mgrid[0:3, 0:5]
    checker = np.where(((xx + yy) % 2 == 0)[..., None], np.float32([0.8, 0.2, 0.1]), np.float32([0.1, 0.3, 0.7]))
    return [noise, checker.astype(np.float32)]


def scene_textures():
    """texture_images, then a scale texture (a constant times the checker) and a mixture texture (noise and
    checker mixed by the noise's first channel), as textures 1-4."""
    return texture_images() + [
        dict(kind=rb.RB_TEXTURE_SCALE, inputs=[0, 2], constants=[(0.5, 0.7, 0.9)]),
        dict(kind=rb.RB_TEXTURE_MIXTURE, inputs=[1, 2, 1]),
    ]


def textured_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with textures (scene_textures): every matte material's diffuse
    from the noise image or (every other one) the mixture texture; every third
    material (from the second, the floor's) a plastic with its diffuse from the
    scale texture and its specular from the noise, every third (from the third)
    in turn a translucent material with a textured transmission, an uber
    material with a textured opacity, and a glass whose transmission is the
    mixture texture."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if k % 3 == 1:
            m = _desc(rb.RB_MATERIAL_PLASTIC, remap_roughness=1, diffuse=(0.5, 0.5, 0.5), reflectance=(0.3, 0.3, 0.3),
                      roughness_u=0.15, ior=1.49, diffuse_texture=3, reflectance_texture=1)
        elif k % 3 == 2:
            variant = (k // 3) % 3
            if variant == 0:
                m = _desc(rb.RB_MATERIAL_TRANSLUCENT, remap_roughness=1, diffuse=(0.6, 0.5, 0.4), specular=(0.4, 0.4, 0.4),
                          reflectance=(0.5, 0.5, 0.5), transmission=(0.4, 0.45, 0.5), roughness_u=0.2, roughness_v=0.2,
                          transmission_texture=1)
            elif variant == 1:
                m = _desc(rb.RB_MATERIAL_UBER, remap_roughness=1, diffuse=(0.5, 0.3, 0.2), specular=(0.3, 0.3, 0.25),
                          reflectance=(0.1, 0.1, 0.1), opacity=(1.0, 1.0, 1.0), roughness_u=0.15, roughness_v=0.2, ior=1.5,
                          opacity_texture=2)
            else:
                m = _desc(rb.RB_MATERIAL_GLASS, reflectance=(1.0, 1.0, 1.0), transmission=(1.0, 1.0, 1.0), ior=1.5,
                          transmission_texture=4)
        elif m.kind == rb.RB_MATERIAL_MATTE:
            m.diffuse_texture = 1 if k % 2 == 0 else 4
        mats.append(m)
    return scene.with_materials(mats).with_textures(scene_textures())


def real_texture_images():
    """Textures 5-13 after scene_textures: images for real parameters (channel 0 read; all three channels
    equal): roughness 0.02-0.5 (7 x 5), IOR 1.2-1.8 (4 x 6), Oren-Nayar sigma 0-60 degrees with zeros
    (5 x 5), a checker of roughness 0 and 0.3 (3 x 2: glass is Fresnel-specular where both roughnesses
    are 0); RGB images of conductor eta, k and mean free paths; a scale texture (the roughness image
    times 0.5) and a mixture texture (the roughness image and 0.05, mixed by the checker) of reals."""
    rng = np.random.default_rng(29)

    def grey(v):
        return np.repeat(v[..., None], 3, axis=2).astype(np.float32)
    rough = grey(0.02 + 0.48 * rng.random((5, 7)))
    ior = grey(1.2 + 0.6 * rng.random((6, 4)))
    sigma = 60.0 * rng.random((5, 5))
    sigma[rng.random((5, 5)) < 0.3] = 0.0
    yy, xx = np.mgrid[0:2, 0:3]
    checker = np.where((xx + yy) % 2 == 0, 0.0, 0.3)
    eta = (0.2 + rng.random((4, 4, 3))).astype(np.float32)
    k = (2.0 + 2.0 * rng.random((3, 5, 3))).astype(np.float32)
    mfp = (0.05 + 0.35 * rng.random((4, 3, 3))).astype(np.float32)
    return [rough, ior, grey(sigma), grey(checker), eta, k, mfp,
            dict(kind=rb.RB_TEXTURE_SCALE, inputs=[5, 0], constants=[(0.0, 0.0, 0.0), (0.5, 0.5, 0.5)]),
            dict(kind=rb.RB_TEXTURE_MIXTURE, inputs=[5, 0, 8], constants=[(0.0, 0.0, 0.0), (0.05, 0.05, 0.05)])]


def real_textured_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with textured real parameters (real_texture_images as textures 5-13 after
    scene_textures): every matte material's sigma from the sigma image; every third material (from
    the second, the floor's) in turn a metal with its roughnesses from the real scale and mixture
    textures and its eta and k from images, a glass
    whose roughnesses follow the 0 / 0.3 checker and whose IOR follows the IOR image, and a plastic
    with textured roughness, IOR and diffuse; every third (from the third) in turn an uber with a
    textured IOR and roughness u, a substrate with textured roughness v, and a subsurface material
    with textured roughnesses, IOR and mean free path."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if k % 3 == 1:
            variant = (k // 3) % 3
            if variant == 0:
                m = _desc(rb.RB_MATERIAL_METAL, remap_roughness=1, eta=(0.200438, 0.924033, 1.102212),
                          k=(3.912949, 2.452848, 2.142188), roughness_u=0.2, roughness_v=0.3, roughness_u_texture=12,
                          roughness_v_texture=13, eta_texture=9, k_texture=10)
            elif variant == 1:
                m = _desc(rb.RB_MATERIAL_GLASS, remap_roughness=1, reflectance=(1.0, 1.0, 1.0),
                          transmission=(1.0, 1.0, 1.0), ior=1.5, roughness_u_texture=8, roughness_v_texture=8,
                          ior_texture=6)
            else:
                m = _desc(rb.RB_MATERIAL_PLASTIC, remap_roughness=1, diffuse=(0.5, 0.5, 0.5),
                          reflectance=(0.3, 0.3, 0.3), roughness_u=0.15, ior=1.49, diffuse_texture=1,
                          roughness_u_texture=5, ior_texture=6)
        elif k % 3 == 2:
            variant = (k // 3) % 3
            if variant == 0:
                m = _desc(rb.RB_MATERIAL_UBER, remap_roughness=1, diffuse=(0.5, 0.3, 0.2), specular=(0.3, 0.3, 0.25),
                          reflectance=(0.1, 0.1, 0.1), opacity=(1.0, 1.0, 1.0), roughness_u=0.15, roughness_v=0.2,
                          ior=1.5, ior_texture=6, roughness_u_texture=5)
            elif variant == 1:
                m = _desc(rb.RB_MATERIAL_SUBSTRATE, remap_roughness=1, diffuse=(0.5, 0.35, 0.2),
                          reflectance=(0.05, 0.05, 0.05), roughness_u=0.1, roughness_v=0.25, roughness_v_texture=5)
            else:
                m = _desc(rb.RB_MATERIAL_SUBSURFACE, remap_roughness=1, reflectance=(1.0, 1.0, 1.0),
                          transmission=(1.0, 1.0, 1.0), diffuse=(0.8, 0.5, 0.3), mfp=(0.4, 0.2, 0.05), ior=1.33,
                          roughness_u_texture=8, roughness_v_texture=8, ior_texture=6, mfp_texture=11)
        elif m.kind == rb.RB_MATERIAL_MATTE:
            m.sigma_texture = 7
        mats.append(m)
    return scene.with_materials(mats).with_textures(scene_textures() + real_texture_images())


def subsurface_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with every third material (from the second, the floor's) a
    subsurface material (subsurface_material.cpp: glass lobes over a
    normalized-diffusion BSSRDF), smooth and rough in turn, mean free paths
    of 0.05-0.4 scene units; the rest unchanged."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if k % 3 == 1:
            rough = 0.0 if (k // 3) % 2 == 0 else 0.2
            m = _desc(rb.RB_MATERIAL_SUBSURFACE, remap_roughness=1, reflectance=(1.0, 1.0, 1.0),
                      transmission=(1.0, 1.0, 1.0), diffuse=(0.8, 0.5, 0.3), mfp=(0.4, 0.2, 0.05), ior=1.33,
                      roughness_u=rough, roughness_v=rough)
        mats.append(m)
    return scene.with_materials(mats)


def oren_nayar_scene(scene: rb.Scene) -> rb.Scene:
    """The scene with every matte material given an Oren-Nayar sigma of
    10-50 degrees (matte_material.cpp:13-29 then builds oren_nayar_reflection),
    the rest unchanged."""
    mats = []
    for k in range(scene.desc.num_materials):
        m = rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k]))
        if m.kind == rb.RB_MATERIAL_MATTE:
            m.sigma = 10.0 + 10.0 * (k % 5)
        mats.append(m)
    return scene.with_materials(mats)
