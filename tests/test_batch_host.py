"""Batched scenes on the host build of the kernels' stages: several scenes
merged into one set of arrays (the merge rb_batch_upload performs) and traced
or path-traced from each scene's own root, emitters and environments give bit
for bit the hits and radiance of the same scene uploaded alone."""
import numpy as np

import rainbow_b200 as rb
from tests.helpers import (HostBatch, HostPaths, assert_hits_equal, mixture_scene, random_rays, subsurface_scene,
                           textured_scene)


def batch_scenes():
    """Four scenes; the first and the last with image textures (the last's texture references and texels are
    relocated by the merge), the second with a subsurface material (the merged scene takes its profile table,
    and every scene's bounces then run staged with the subsurface stage), the third with mixtures (component
    records relocated)."""
    return [
        textured_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=5, width=40, height=30, num_spheres=12, subdivision=2)),
        subsurface_scene(rb.generate_scene(rb.RB_SCENE_BOX, seed=0, width=32, height=32)),
        mixture_scene(rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=36, height=36, num_spheres=6, subdivision=2)),
        textured_scene(rb.generate_scene(rb.RB_SCENE_SPHERES, seed=9, width=24, height=24, num_spheres=3, subdivision=1)),
    ]


def test_merged_traversal_matches_each_scene_alone():
    scenes = batch_scenes()
    hb = HostBatch(scenes)
    for k, sc in enumerate(scenes):
        rays = random_rays(sc, 3000, 40 + k)
        alone = HostPaths(sc)
        for shadow in (False, True):
            want = alone.trace(rays, shadow)
            assert (want["entity"] >= 0).mean() > 0.05, "the ray set should hit the scene"
            assert_hits_equal(hb.trace(k, rays, shadow), want, f"scene {k} shadow={shadow}")


def test_merged_paths_match_each_scene_alone():
    scenes = batch_scenes()
    hb = HostBatch(scenes)
    rng = np.random.default_rng(7)
    for k, sc in enumerate(scenes):
        n = sc.camera.width * sc.camera.height
        px = rng.integers(0, n, 400).astype(np.uint32)
        sm = rng.integers(0, 64, 400).astype(np.uint32)
        want = HostPaths(sc).samples(sc.camera, px, sm, 6, seed=11)
        got = hb.samples(k, sc.camera, px, sm, 6, seed=11)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"scene {k}"
        assert want.max() > 0


def test_single_scene_batch_equals_scene():
    sc = rb.generate_scene(rb.RB_SCENE_BOX, seed=0, width=32, height=32)
    hb = HostBatch([sc])
    rays = random_rays(sc, 1000, 3)
    assert_hits_equal(hb.trace(0, rays), HostPaths(sc).trace(rays), "single")
