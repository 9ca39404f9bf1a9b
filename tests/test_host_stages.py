"""The kernels' stage functions compiled for the host (tests/native) reproduce
the reference bit for bit: hits of the child-box traversal and of the
reference-order traversal, and the radiance of single (pixel, sample) paths."""
import ctypes

import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import port, ref
from tests import golden
from tests.helpers import HostPaths, assert_hits_equal, scene_from_params


@pytest.mark.parametrize("name", ["box_rays", "spheres_rays"])
@pytest.mark.parametrize("mode", [0, 1])
def test_host_traversal_matches_fixture(name, mode):
    fx = golden.load(name)
    hp = HostPaths(scene_from_params(fx["params"]))
    hp.L.hp_set_mode.argtypes = [ctypes.c_int]
    hp.L.hp_set_mode(mode)
    try:
        assert_hits_equal(hp.trace(fx["rays"], False), fx["hits_closest"], "closest")
        assert_hits_equal(hp.trace(fx["rays"], True), fx["hits_shadow"], "shadow")
    finally:
        hp.L.hp_set_mode(0)


@pytest.mark.parametrize("name", ["box_samples", "spheres_samples"])
def test_host_stages_match_fixture_samples(name):
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    got = HostPaths(scene).samples(scene.camera, fx["pixels"], fx["samples"], int(fx["max_depth"]))
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))


def test_host_stages_slit_room_against_port():
    scene = rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=48, height=48, num_spheres=20, subdivision=2)
    sb = scene.with_bvh(rb.build_bvh(scene))
    rng = np.random.default_rng(2)
    px = rng.integers(0, 48 * 48, 600).astype(np.uint32)
    sm = rng.integers(0, 100, 600).astype(np.uint32)
    a = port.samples(sb, scene.camera, px, sm, 8)
    b = HostPaths(scene).samples(scene.camera, px, sm, 8)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_host_traversal_full_size_against_reference():
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4)
    R = ref.RefScene(scene)
    rays = R.make_rays(20000, 21)
    hp = HostPaths(scene)
    for shadow in (False, True):
        assert_hits_equal(hp.trace(rays, shadow), R.trace(rays, shadow), f"shadow={shadow}")
