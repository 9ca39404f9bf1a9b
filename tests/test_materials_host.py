"""Plastic, mirror, substrate and Oren-Nayar matte materials (plastic_material.cpp,
mirror_material.cpp, substrate_material.cpp, matte_material.cpp with sigma != 0) in
the path integrator's stages and in direct lighting, compiled for the host,
against the reference (fixture from the compiled reference, and the reference
itself where it is built): bit-equal radiance per (pixel, sample)."""
import numpy as np
import pytest

from oracle import ref
from tests import golden
from tests.helpers import HostPaths, extra_materials_scene, oren_nayar_scene, scene_from_params


def test_host_stages_extra_materials_match_fixture():
    fx = golden.load("materials_samples")
    scene = extra_materials_scene(scene_from_params(fx["params"]))
    got = HostPaths(scene).samples(scene.camera, fx["pixels"], fx["samples"], int(fx["max_depth"]))
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_host_direct_extra_materials_against_reference():
    fx = golden.load("materials_samples")
    scene = extra_materials_scene(scene_from_params(fx["params"]))
    R = ref.RefScene(scene)
    R.set_direct(3, 2)
    want = R.trace_samples(fx["pixels"], fx["samples"])
    for staged in (False, True):
        got = HostPaths(scene).direct_samples(scene.camera, fx["pixels"], fx["samples"], 3, 2, staged=staged)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), staged


def test_host_stages_oren_nayar_match_fixture():
    fx = golden.load("oren_nayar_samples")
    scene = oren_nayar_scene(scene_from_params(fx["params"]))
    got = HostPaths(scene).samples(scene.camera, fx["pixels"], fx["samples"], int(fx["max_depth"]))
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))
