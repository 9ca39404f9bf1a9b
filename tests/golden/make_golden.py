"""Regenerates the golden fixtures in tests/golden/ from the oracle.

The reference ships no tests or known-answer vectors, so the fixtures are
outputs of the reference renderer itself, compiled from its sources as
oracle/_ref/liboracle_ref.so (`make -C oracle ref`), on inputs made by the
product's seeded scene generator:

  pcg32          uniform_uint32 / uniform_real streams of pcg32(seed)
  box_rays       4096 seeded rays (camera rays and 1-2 diffuse bounces) in the box
                 room: scene::intersect and intersect_with_shadow_ray results
  spheres_rays   the same on a 30-sphere displaced-icosphere scene
  box_samples    radiance of 1024 (pixel, sample) pairs, path_integrator::trace, depth 5
  spheres_samples  the same at depth 8 (metal, glass, quad lights, environment)
  bsdf_*         scattering_function_collection sample / evaluate / pdf per material
  box_image      32 x 32 box room, 256 spp, FP64 per-pixel sums of L and L^2
  bvh_c2         SHA-256 of the reference BVH of the 1,024,010-triangle sphere scene
  fog_samples    radiance of 1024 (pixel, sample) pairs, volume_path_integrator::trace,
                 depth 12, displaced spheres inside a homogeneous medium box
  fog_image      32 x 32 fog scene, 256 spp, volume_path_integrator, FP64 sums of L and L^2
  direct_spheres radiance of 1024 (pixel, sample) pairs, direct_integrator::trace with the
                 default 4 emitter and 4 BSDF samples, on the spheres scene above
  direct_fog     512 pairs, direct_integrator(2 emitter, 3 BSDF samples), fog scene (rays
                 pass through the medium's invisible boundary)
  materials_samples  radiance of 1024 pairs, path_integrator::trace depth 8, on the spheres
                 scene with plastic and mirror materials (tests.helpers.extra_materials_scene)
  bsdf_plastic_*, bsdf_mirror_*, bsdf_substrate_*  the BSDF tables of those materials
  oren_nayar_samples  radiance of 1024 pairs, path_integrator::trace depth 8, on the spheres
                 scene with Oren-Nayar matte (tests.helpers.oren_nayar_scene)
  bsdf_oren_nayar_*  the BSDF tables of a matte material with sigma 20 (--only oren_nayar)
  layered_samples, mixture_samples, texture_samples, subsurface_samples  radiance of 1024
                 pairs, path_integrator::trace depth 8, on the spheres scene with uber and
                 translucent, mixture, textured and subsurface materials (tests.helpers
                 layered_scene, mixture_scene, textured_scene, subsurface_scene; --only
                 layered|mixture|textures|subsurface), with first_entity
  bsdf_uber_*, bsdf_translucent_*, bsdf_mixture_*  the BSDF tables of those materials
  real_texture_samples  the same on tests.helpers.real_textured_scene (roughness, IOR and
                 sigma from image textures; --only real_textures)
  photons_box, photons_spheres, photons_materials  photon_mapping_integrator::render images
                 (stochastic progressive photon mapping) of PHOTON_CASES (--only photons)

The benchmark configurations themselves (--only baseline):
  config1_image  configuration 1 as specified (box room, 256 x 256, depth 5):
                 per-pixel mean and per-sample variance of a 512-spp render
  c2_ray_levels  the 1,024,010-triangle sphere field of configuration 2: 2^19
                 seeded camera rays and two generations of bounce rays from their
                 hits (tests.helpers.ray_levels), traced by scene::intersect;
                 per level the ray count, hit count, SHA-256 of every 4096 hits
                 (entity, triangle, bits of t) and the first 4096 hits in full
  slit_samples   configuration 4's slit room (2,048,018 triangles) at 64 x 64:
                 radiance of 1024 (pixel, sample) pairs, path_integrator, depth 8
  slit_image     the same room, 64 x 64, 1024 spp: per-pixel mean and variance
  fog5_samples   configuration 5's fog (8,192,046 triangles) at 64 x 36: 512 pairs,
                 volume_path_integrator, depth 12
  fog5_image     the same fog, 64 x 36, 1024 spp: per-pixel mean and variance
  box_converged  box room, 64 x 64, depth 5, 8192 spp: FP64 per-pixel means (the
                 high-spp plain render that relMSE is measured against)
  first_entity   added to box_samples, spheres_samples, materials_samples and
                 fog_samples: the entity of each sample's camera-ray hit

The reference's two-level tree (--only two_level):
  two_level      tests.helpers.two_level_scene (a 327,680-triangle mesh and a mesh
                 shared by two entities): 8192 seeded rays with scene::intersect and
                 intersect_with_shadow_ray hits, and the radiance of 512 (pixel,
                 sample) pairs, path_integrator, depth 5

Usage: python tests/golden/make_golden.py [--only fog|direct|materials|baseline|two_level|oren_nayar|layered|
       mixture|textures|subsurface|photons|real_textures]
"""
from __future__ import annotations

import hashlib
import os
import sys

import ctypes as C

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import rainbow_b200 as rb  # noqa: E402
from oracle import ref  # noqa: E402

BOX = dict(kind=rb.RB_SCENE_BOX, seed=0, width=64, height=64, num_spheres=0, subdivision=0)
SPHERES = dict(kind=rb.RB_SCENE_SPHERES, seed=1, width=96, height=96, num_spheres=30, subdivision=2)
C2 = dict(kind=rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4)
FOG = dict(kind=rb.RB_SCENE_FOG, seed=4, width=48, height=48, num_spheres=24, subdivision=2)


def scene_of(p):
    return rb.generate_scene(p["kind"], seed=p["seed"], width=p["width"], height=p["height"],
                             num_spheres=p["num_spheres"], subdivision=p["subdivision"])


def params_array(p):
    return np.array([p["kind"], p["seed"], p["width"], p["height"], p["num_spheres"], p["subdivision"]], dtype=np.int64)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
    print("wrote", name, {k: v.shape for k, v in arrays.items()})


def bvh_digest(nodes, pe, pi):
    h = hashlib.sha256()
    for a in (nodes.astype(np.float32).view(np.uint32), pe.astype(np.uint32), pi.astype(np.uint32)):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


C1 = dict(kind=rb.RB_SCENE_BOX, seed=0, width=256, height=256, num_spheres=0, subdivision=0)
SLIT = dict(kind=rb.RB_SCENE_SLIT_ROOM, seed=3, width=64, height=64, num_spheres=100, subdivision=5)
FOG5 = dict(kind=rb.RB_SCENE_FOG, seed=5, width=64, height=36, num_spheres=400, subdivision=5)


def parallel_trace(R, rays, chunk=1 << 14):
    """scene::intersect of a large batch on all host threads (ctypes releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    hits = np.zeros(rays.shape[0], dtype=rb.HIT_DTYPE)

    def part(a):
        hits[a:a + chunk] = R.trace(rays[a:a + chunk])
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        list(ex.map(part, range(0, rays.shape[0], chunk)))
    return hits


def mean_var(sums, sq, n):
    mean = sums / n
    var = np.maximum(sq / n - mean ** 2, 0.0)
    return mean.astype(np.float32), var.astype(np.float32)


def baseline_fixtures():
    from tests.helpers import hit_digests, ray_levels
    s = scene_of(C1)
    R = ref.RefScene(s)
    n = 512
    sums, sq, sec = R.render(n, 0, 5, 1.0, 0, 0)
    mean, var = mean_var(sums, sq, n)
    save("config1_image", params=params_array(C1), spp=np.array(n), max_depth=np.array(5), mean=mean, var=var,
         seconds=np.array(sec))

    s = scene_of(dict(BOX, width=64, height=64))
    R = ref.RefScene(s)
    n = 8192
    sums, _, sec = R.render(n, 0, 5, 1.0, 0, 0)
    save("box_converged", params=params_array(dict(BOX, width=64, height=64)), spp=np.array(n), max_depth=np.array(5),
         mean=sums / n)

    s = scene_of(C2)
    R = ref.RefScene(s)
    levels = ray_levels(s.camera, lambda r: parallel_trace(R, r), 1 << 19, 21)
    out = dict(params=params_array(C2), seed=np.array(21), n0=np.array(1 << 19))
    for k, (rays, hits) in enumerate(levels):
        out[f"count{k}"] = np.array(rays.shape[0])
        out[f"hit_count{k}"] = np.array((hits["entity"] >= 0).sum())
        out[f"digests{k}"] = hit_digests(hits)
        out[f"head{k}"] = hits[:4096]
    save("c2_ray_levels", **out)

    for name, p, vol, depth, npairs in (("slit", SLIT, False, 8, 1024), ("fog5", FOG5, True, 12, 512)):
        s = scene_of(p)
        R = ref.RefScene(s)
        R.set_volume(vol)
        rng = np.random.default_rng(23)
        px = rng.integers(0, p["width"] * p["height"], npairs).astype(np.uint32)
        sm = rng.integers(0, 4096, npairs).astype(np.uint32)
        L = R.trace_samples(px, sm, max_depth=depth, rr=1.0, seed=0)
        save(f"{name}_samples", params=params_array(p), pixels=px, samples=sm, radiance=L, max_depth=np.array(depth),
             first_entity=first_entity(R, px, sm))
        n = 1024
        sums, sq, sec = R.render(n, 0, depth, 1.0, 0, 0)
        mean, var = mean_var(sums, sq, n)
        save(f"{name}_image", params=params_array(p), spp=np.array(n), max_depth=np.array(depth), mean=mean, var=var,
             seconds=np.array(sec))
    add_first_entity()


def two_level_fixtures():
    from tests.helpers import random_rays, two_level_scene
    s = two_level_scene()
    R = ref.RefScene(s)
    rays = random_rays(s, 8192, 35)
    rng = np.random.default_rng(29)
    px = rng.integers(0, s.camera.width * s.camera.height, 512).astype(np.uint32)
    sm = rng.integers(0, 4096, 512).astype(np.uint32)
    save("two_level", rays=rays, hits_closest=R.trace(rays), hits_shadow=R.trace(rays, shadow=True), pixels=px,
         samples=sm, radiance=R.trace_samples(px, sm, max_depth=5, rr=1.0, seed=0), max_depth=np.array(5),
         first_entity=first_entity(R, px, sm))


def first_entity(R, px, sm):
    """Entity ordinal of each (pixel, sample)'s camera-ray hit (-1: miss)."""
    return R.trace(R.camera_rays(px, sm, 0))["entity"].astype(np.int32)


def add_first_entity():
    """Adds first_entity to the per-sample fixtures, leaving their other arrays as they are."""
    from tests import golden
    for name in ("box_samples", "spheres_samples", "materials_samples", "fog_samples"):
        fx = golden.load(name)
        sc = scene_of(dict(zip(("kind", "seed", "width", "height", "num_spheres", "subdivision"),
                               (int(x) for x in fx["params"]))))
        if name == "materials_samples":
            from tests.helpers import extra_materials_scene
            sc = extra_materials_scene(sc)
        fx["first_entity"] = first_entity(ref.RefScene(sc), fx["pixels"], fx["samples"])
        save(name, **fx)


def fog_fixtures():
    s = scene_of(FOG)
    R = ref.RefScene(s)
    R.set_volume(True)
    rng = np.random.default_rng(13)
    px = rng.integers(0, FOG["width"] * FOG["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=12, rr=1.0, seed=0)
    save("fog_samples", params=params_array(FOG), pixels=px, samples=sm, radiance=L, max_depth=np.array(12))
    small = dict(FOG, width=32, height=32)
    R = ref.RefScene(scene_of(small))
    R.set_volume(True)
    sums, sq, _ = R.render(256, 0, 12, 1.0, 0, 0)
    save("fog_image", params=params_array(small), spp=np.array(256), max_depth=np.array(12), sum=sums, sum_sq=sq)


def direct_fixtures():
    for name, p, n, E, B in (("direct_spheres", SPHERES, 1024, 4, 4), ("direct_fog", FOG, 512, 2, 3)):
        R = ref.RefScene(scene_of(p))
        R.set_direct(E, B)
        rng = np.random.default_rng(17)
        px = rng.integers(0, p["width"] * p["height"], n).astype(np.uint32)
        sm = rng.integers(0, 4096, n).astype(np.uint32)
        L = R.trace_samples(px, sm, seed=0)
        save(name, params=params_array(p), pixels=px, samples=sm, radiance=L, emitter_samples=np.array(E),
             bsdf_samples=np.array(B))


def oren_nayar_fixtures():
    from tests.helpers import oren_nayar_scene
    R = ref.RefScene(oren_nayar_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(37)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("oren_nayar_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8),
         first_entity=first_entity(R, px, sm))
    bsdf_fixtures({"oren_nayar": dict(kind=rb.RB_MATERIAL_MATTE, diffuse=(0.7, 0.4, 0.2), sigma=20.0)})


def layered_fixtures():
    from tests.helpers import layered_scene
    R = ref.RefScene(layered_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(41)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("layered_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8),
         first_entity=first_entity(R, px, sm))
    bsdf_fixtures({"uber": dict(kind=rb.RB_MATERIAL_UBER, opacity=(0.7, 0.8, 0.9)),
                   "uber_opaque": dict(kind=rb.RB_MATERIAL_UBER, opacity=(1.0, 1.0, 1.0)),
                   "translucent": dict(kind=rb.RB_MATERIAL_TRANSLUCENT)})


def mixture_fixtures():
    from tests.helpers import _desc, mixture_scene
    R = ref.RefScene(mixture_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(43)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("mixture_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8),
         first_entity=first_entity(R, px, sm))
    # BSDF tables of a mixture of an Oren-Nayar matte and a rough glass (its array: mixture, then the two)
    mats = (rb.MaterialDesc * 3)(
        _desc(rb.RB_MATERIAL_MIXTURE, amount=(0.3, 0.5, 0.7), components=(1, 2)),
        _desc(rb.RB_MATERIAL_MATTE, diffuse=(0.7, 0.5, 0.3), sigma=25.0),
        _desc(rb.RB_MATERIAL_GLASS, remap_roughness=1, reflectance=(1.0, 1.0, 1.0), transmission=(1.0, 1.0, 1.0),
              ior=1.5, roughness_u=0.2, roughness_v=0.2))
    bsdf_tables("mixture", mats)


def texture_fixtures():
    from tests.helpers import textured_scene
    R = ref.RefScene(textured_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(47)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("texture_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8),
         first_entity=first_entity(R, px, sm))


def subsurface_fixtures():
    from tests.helpers import subsurface_scene
    R = ref.RefScene(subsurface_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(53)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("subsurface_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8),
         first_entity=first_entity(R, px, sm))


def real_texture_fixtures():
    from tests.helpers import real_textured_scene
    R = ref.RefScene(real_textured_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(59)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("real_texture_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L,
         max_depth=np.array(8), first_entity=first_entity(R, px, sm))


# photon_mapping_integrator::render cases: (name, scene params, scene variant,
# iterations, max_depth, photons, radius)
PHOTON_CASES = (
    ("box", dict(BOX, width=32, height=32), None, 3, 5, 0, 0.1),
    ("spheres", dict(SPHERES, width=48, height=40, num_spheres=12), None, 3, 5, 0, 0.5),
    ("materials", dict(SPHERES, width=48, height=40, num_spheres=12), "extra_materials_scene", 4, 6, 3000, 0.3),
)


def photon_scene(params, variant):
    import tests.helpers as H
    sc = scene_of(params)
    return getattr(H, variant)(sc) if variant else sc


def photon_fixtures():
    for name, params, variant, it, depth, photons, radius in PHOTON_CASES:
        R = ref.RefScene(photon_scene(params, variant))
        img, _ = R.render_photons(it, depth, photons, radius)
        save(f"photons_{name}", params=params_array(params), image=img, iterations=np.array(it), max_depth=np.array(depth),
             photons=np.array(photons), radius=np.array(radius, np.float32))


def materials_fixtures():
    from tests.helpers import extra_materials_scene
    R = ref.RefScene(extra_materials_scene(scene_of(SPHERES)))
    rng = np.random.default_rng(19)
    px = rng.integers(0, SPHERES["width"] * SPHERES["height"], 1024).astype(np.uint32)
    sm = rng.integers(0, 4096, 1024).astype(np.uint32)
    L = R.trace_samples(px, sm, max_depth=8, rr=1.0, seed=0)
    save("materials_samples", params=params_array(SPHERES), pixels=px, samples=sm, radiance=L, max_depth=np.array(8))
    bsdf_fixtures({"plastic": dict(kind=rb.RB_MATERIAL_PLASTIC, rough=0.3),
                   "mirror": dict(kind=rb.RB_MATERIAL_MIRROR),
                   "substrate": dict(kind=rb.RB_MATERIAL_SUBSTRATE, rough=0.2)})


def bsdf_fixtures(mats):
    for key, m in mats.items():
        bsdf_tables(key, material_desc(m))


def bsdf_tables(key, md):
    # BSDF known answers on the shading frame = world axes; md: one descriptor,
    # or an array whose first entry is the material (a mixture's components after it)
    rng = np.random.default_rng(5)
    n = 512
    wo = rng.normal(size=(n, 3)).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3)).astype(np.float32)
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    u = rng.random((n, 2), dtype=np.float32)
    for include_name, include in (("all", 31), ("nonspec", 27)):
        out = ref.bsdf(md, wo, u, wi, include)
        save(f"bsdf_{key}_{include_name}", wo=wo, u=u, wi_eval=wi, include=np.array(include),
             material=np.frombuffer(bytes(md), dtype=np.uint8),
             material_count=np.array(len(md) if isinstance(md, C.Array) else 1), **out)


def main():
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if only == "materials":
        return materials_fixtures()
    if only == "fog":
        return fog_fixtures()
    if only == "direct":
        return direct_fixtures()
    if only == "baseline":
        return baseline_fixtures()
    if only == "two_level":
        return two_level_fixtures()
    if only == "oren_nayar":
        return oren_nayar_fixtures()
    if only == "layered":
        return layered_fixtures()
    if only == "mixture":
        return mixture_fixtures()
    if only == "textures":
        return texture_fixtures()
    if only == "subsurface":
        return subsurface_fixtures()
    if only == "photons":
        return photon_fixtures()
    if only == "real_textures":
        return real_texture_fixtures()
    seeds = np.array([0, 1, 2, 3, 0xDEADBEEF, (1 << 48) | 12345], dtype=np.uint64)
    u32 = np.zeros((len(seeds), 64), np.uint32)
    reals = np.zeros((len(seeds), 64), np.float32)
    for i, s in enumerate(seeds):
        u32[i], reals[i] = ref.pcg32(int(s), 64)
    save("pcg32", seeds=seeds, u32=u32, reals=reals)

    for name, p, nrays, depth in (("box", BOX, 4096, 5), ("spheres", SPHERES, 8192, 8)):
        s = scene_of(p)
        R = ref.RefScene(s)
        rays = R.make_rays(nrays, 7)
        hc, pc = R.trace(rays, shadow=False, points=True)
        hs = R.trace(rays, shadow=True)
        r2c, c2w = R.camera_matrices()
        nodes, pe, pi = R.bvh()
        save(f"{name}_rays", params=params_array(p), rays=rays, hits_closest=hc, points_closest=pc, hits_shadow=hs,
             raster_to_camera=r2c, camera_to_world=c2w, areas=R.areas(), bvh_nodes=nodes, bvh_prim_entity=pe,
             bvh_prim_index=pi)
        rng = np.random.default_rng(11)
        W, H = p["width"], p["height"]
        px = rng.integers(0, W * H, 1024).astype(np.uint32)
        sm = rng.integers(0, 4096, 1024).astype(np.uint32)
        L = R.trace_samples(px, sm, max_depth=depth, rr=1.0, seed=0)
        save(f"{name}_samples", params=params_array(p), pixels=px, samples=sm, radiance=L, max_depth=np.array(depth))

    bsdf_fixtures({
        "lambert": dict(kind=rb.RB_MATERIAL_MATTE, diffuse=(0.7, 0.4, 0.2)),
        "metal": dict(kind=rb.RB_MATERIAL_METAL, rough=0.3),
        "glass_rough": dict(kind=rb.RB_MATERIAL_GLASS, rough=0.2),
        "glass_smooth": dict(kind=rb.RB_MATERIAL_GLASS, rough=0.0),
    })

    s = scene_of(dict(BOX, width=32, height=32))
    R = ref.RefScene(s)
    sums, sq, sec = R.render(256, 0, 5, 1.0, 0, 0)
    save("box_image", params=params_array(dict(BOX, width=32, height=32)), spp=np.array(256), sum=sums, sum_sq=sq)

    s = scene_of(C2)
    R = ref.RefScene(s)
    nodes, pe, pi = R.bvh()
    save("bvh_c2", params=params_array(C2), digest=np.array(bvh_digest(nodes, pe, pi)),
         num_nodes=np.array(nodes.shape[0]), num_prims=np.array(pe.shape[0]))
    fog_fixtures()
    direct_fixtures()
    materials_fixtures()
    baseline_fixtures()
    two_level_fixtures()
    oren_nayar_fixtures()
    layered_fixtures()
    mixture_fixtures()
    texture_fixtures()
    subsurface_fixtures()
    real_texture_fixtures()
    photon_fixtures()


def material_desc(m):
    md = rb._native.MaterialDesc()
    md.kind = m["kind"]
    if m["kind"] == rb.RB_MATERIAL_MATTE:
        md.diffuse[:] = m["diffuse"]
        md.sigma = m.get("sigma", 0.0)
    elif m["kind"] == rb.RB_MATERIAL_PLASTIC:
        md.remap_roughness = 1
        md.diffuse[:] = (0.6, 0.3, 0.2)
        md.reflectance[:] = (0.5, 0.45, 0.4)
        md.roughness_u = m["rough"]
        md.ior = 1.49
    elif m["kind"] == rb.RB_MATERIAL_MIRROR:
        md.reflectance[:] = (0.9, 0.85, 0.8)
    elif m["kind"] == rb.RB_MATERIAL_SUBSTRATE:
        md.remap_roughness = 1
        md.diffuse[:] = (0.5, 0.35, 0.2)
        md.reflectance[:] = (0.05, 0.05, 0.05)
        md.roughness_u, md.roughness_v = m["rough"], 0.5 * m["rough"]
    elif m["kind"] == rb.RB_MATERIAL_UBER:
        md.remap_roughness = 1
        md.diffuse[:] = (0.5, 0.3, 0.2)
        md.specular[:] = (0.3, 0.3, 0.25)
        md.reflectance[:] = (0.1, 0.1, 0.1)
        md.transmission[:] = (0.2, 0.25, 0.3)
        md.opacity[:] = m["opacity"]
        md.roughness_u, md.roughness_v = 0.15, 0.3
        md.ior = 1.5
    elif m["kind"] == rb.RB_MATERIAL_TRANSLUCENT:
        md.remap_roughness = 1
        md.diffuse[:] = (0.6, 0.5, 0.4)
        md.specular[:] = (0.4, 0.4, 0.4)
        md.reflectance[:] = (0.5, 0.5, 0.5)
        md.transmission[:] = (0.4, 0.45, 0.5)
        md.roughness_u = 0.2
    elif m["kind"] == rb.RB_MATERIAL_METAL:
        md.remap_roughness = 1
        md.eta[:] = (0.200438, 0.924033, 1.102212)
        md.k[:] = (3.912949, 2.452848, 2.142188)
        md.roughness_u = md.roughness_v = m["rough"]
    else:
        md.remap_roughness = 1
        md.reflectance[:] = (1.0, 1.0, 1.0)
        md.transmission[:] = (1.0, 1.0, 1.0)
        md.ior = 1.5
        md.roughness_u = md.roughness_v = m["rough"]
    return md


if __name__ == "__main__":
    main()
