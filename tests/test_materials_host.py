"""Plastic, mirror, substrate, Oren-Nayar matte, uber and translucent materials
(plastic_material.cpp, mirror_material.cpp, substrate_material.cpp, matte_material.cpp
with sigma != 0, uber_material.cpp, translucent_material.cpp) in
the path integrator's stages and in direct lighting, compiled for the host,
against the reference (fixture from the compiled reference, and the reference
itself where it is built): bit-equal radiance per (pixel, sample)."""
import numpy as np
import pytest

import rainbow_b200 as rb

from oracle import ref
from tests import golden
from tests.helpers import (HostPaths, extra_materials_scene, layered_scene, material_lobes, oren_nayar_scene,
                           scene_from_params)


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


def test_host_stages_layered_materials_match_fixture():
    fx = golden.load("layered_samples")
    scene = layered_scene(scene_from_params(fx["params"]))
    got = HostPaths(scene).samples(scene.camera, fx["pixels"], fx["samples"], int(fx["max_depth"]))
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_host_direct_layered_materials_against_reference():
    fx = golden.load("layered_samples")
    scene = layered_scene(scene_from_params(fx["params"]))
    R = ref.RefScene(scene)
    R.set_direct(3, 2)
    want = R.trace_samples(fx["pixels"], fx["samples"])
    for staged in (False, True):
        got = HostPaths(scene).direct_samples(scene.camera, fx["pixels"], fx["samples"], 3, 2, staged=staged)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), staged


def test_layered_lobe_lists():
    """Lobe lists of the packed records: uber drops black lobes and adds the
    pass-through transmission only when opacity is below one; translucent has
    no lobes when reflectance and transmission are both black."""
    def lobes(**kw):
        md = rb.MaterialDesc()
        for k, v in kw.items():
            if isinstance(v, tuple):
                getattr(md, k)[:] = v
            else:
                setattr(md, k, v)
        return material_lobes(md)

    assert lobes(kind=rb.RB_MATERIAL_UBER, ior=1.5, opacity=(1.0, 1.0, 1.0), diffuse=(0.5, 0.5, 0.5)) == ["lambert"]
    assert lobes(kind=rb.RB_MATERIAL_UBER, ior=1.5, opacity=(0.5, 1.0, 1.0), diffuse=(0.5, 0.5, 0.5),
                 specular=(0.1, 0.1, 0.1), reflectance=(0.2, 0.2, 0.2), transmission=(0.3, 0.3, 0.3)) == [
        "specular_transmission", "lambert", "microfacet_reflection", "specular_reflection", "specular_transmission"]
    assert lobes(kind=rb.RB_MATERIAL_UBER, ior=1.5) == ["specular_transmission"]  # opacity 0: all pass-through
    assert lobes(kind=rb.RB_MATERIAL_TRANSLUCENT, diffuse=(0.5, 0.5, 0.5), specular=(0.5, 0.5, 0.5)) == []
    assert lobes(kind=rb.RB_MATERIAL_TRANSLUCENT, diffuse=(0.5, 0.5, 0.5), specular=(0.5, 0.5, 0.5),
                 transmission=(0.3, 0.3, 0.3)) == ["lambert_transmission", "microfacet_transmission"]
    with pytest.raises(rb.RbError):
        lobes(kind=rb.RB_MATERIAL_UBER, ior=0.0)
