"""Closest-hit parity of the sm_100a traversal kernels against the reference.

Per ray: entity and triangle ids equal, and the hit distance equal to the bit
(stronger than the 1e-5 relative bound), for scene::intersect and
scene::intersect_with_shadow_ray (rainbow-cpu/scenes/scene.cpp:82-112).
"""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.helpers import assert_hits_equal, scene_from_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["box_rays", "spheres_rays"])
def test_trace_matches_reference_fixture(name):
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        assert_hits_equal(ctx.trace_closest(fx["rays"]), fx["hits_closest"], f"{name} closest")
        assert_hits_equal(ctx.trace_shadow(fx["rays"]), fx["hits_shadow"], f"{name} shadow")


def test_trace_with_reference_bvh_layout():
    """Uploading the reference's exported tree gives the same hits as the built one."""
    fx = golden.load("spheres_rays")
    scene = scene_from_params(fx["params"])
    bvh = rb.bvh_from_arrays(fx["bvh_nodes"], fx["bvh_prim_entity"], fx["bvh_prim_index"])
    with rb.Context(0) as ctx:
        ctx.upload(scene.with_bvh(bvh))
        assert_hits_equal(ctx.trace_closest(fx["rays"]), fx["hits_closest"], "exported tree")


def test_trace_full_size_scene_against_host_stage_build():
    """1,024,010 triangles: the kernels agree with the host build of the same
    arithmetic (which the CPU tests pin to the reference) on 65,536 rays."""
    from tests.helpers import HostPaths
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4)
    rng = np.random.default_rng(3)
    n = 1 << 16
    rays = np.zeros(n, dtype=rb.RAY_DTYPE)
    # camera-like rays from above the field plus random rays from inside it
    o = np.where(rng.random((n, 1)) < 0.5, np.array([5.0, 9.0, 25.0]), rng.uniform(0, 10, (n, 3)))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["origin"], rays["direction"], rays["length"] = o, d, np.inf
    hp = HostPaths(scene)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        for shadow in (False, True):
            got = ctx.trace_shadow(rays) if shadow else ctx.trace_closest(rays)
            assert_hits_equal(got, hp.trace(rays, shadow), f"full size shadow={shadow}")
            assert (got["entity"] >= 0).mean() > 0.05


def test_trace_empty_and_errors():
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=16, height=16)
    with rb.Context(0) as ctx:
        with pytest.raises(rb.RbError):
            ctx.trace_closest(np.zeros(4, dtype=rb.RAY_DTYPE))  # no scene yet
        ctx.upload(scene)
        assert ctx.trace_closest(np.zeros(0, dtype=rb.RAY_DTYPE)).shape == (0,)
        # a ray of zero length hits nothing; a ray with a NaN direction hits nothing
        r = np.zeros(2, dtype=rb.RAY_DTYPE)
        r["origin"] = [0.5, 0.5, 0.5]
        r["direction"][0] = [0, 1, 0]
        r["direction"][1] = [np.nan, 0, 0]
        r["length"] = [0.0, np.inf]
        h = ctx.trace_closest(r)
        assert h["entity"][0] == -1


def test_two_level_scene_hits_match_reference():
    """A 327,680-triangle mesh and a mesh shared by two entities: the scene tree
    holds those entities whole and their meshes have their own trees (the
    reference's two-level case). Hits bit-equal to scene::intersect and
    intersect_with_shadow_ray, on the 4-wide path and on the reference-order
    path (counting launches walk that one)."""
    from tests.helpers import two_level_scene
    fx = golden.load("two_level")
    scene = two_level_scene()
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        assert_hits_equal(ctx.trace_closest(fx["rays"]), fx["hits_closest"], "two-level closest")
        assert_hits_equal(ctx.trace_shadow(fx["rays"]), fx["hits_shadow"], "two-level shadow")
        ctx.set_counting(True)
        assert_hits_equal(ctx.trace_closest(fx["rays"]), fx["hits_closest"], "two-level closest, reference order")


def test_two_level_scene_samples_match_reference():
    from tests.helpers import assert_disagreements_unbiased, per_sample_radiance, sample_agreement, two_level_scene
    fx = golden.load("two_level")
    scene = two_level_scene()
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, fx["pixels"], fx["samples"], int(fx["max_depth"]))
        assert ctx.stats().device_error == 0
        # and whole renders on wave lanes with the 4-wide traversal
        ctx.set_tuning(lanes=2, paths_per_wave=1024)
        img = ctx.render(scene.camera, 8, max_depth=5, seed=3)
        assert ctx.stats().device_error == 0 and np.isfinite(img).all()
    agree = sample_agreement(got, fx["radiance"]).mean()
    assert agree >= 0.97, f"only {agree:.4f} of samples agree with the reference"
    assert_disagreements_unbiased(scene, got, fx["radiance"], fx["first_entity"], "two-level")
