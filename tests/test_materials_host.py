"""Plastic, mirror, substrate, Oren-Nayar matte, uber, translucent, mixture and subsurface
materials (plastic_material.cpp, mirror_material.cpp, substrate_material.cpp,
matte_material.cpp with sigma != 0, uber_material.cpp, translucent_material.cpp,
mixture_material.cpp, subsurface_material.cpp with the normalized-diffusion BSSRDF), and
image textures (textures/detail/image_texture.hpp) of spectra and of real parameters, in
the path integrator's stages and in direct lighting, compiled for the host,
against the reference (fixture from the compiled reference, and the reference
itself where it is built): bit-equal radiance per (pixel, sample)."""
import numpy as np
import pytest

import rainbow_b200 as rb

import ctypes as C

from oracle import ref
from tests import golden
from tests.helpers import (HOSTPATHS, _LOBE_NAMES, HostPaths, _desc, extra_materials_scene, layered_scene, material_lobes,
                           mixture_scene, oren_nayar_scene, real_textured_scene, scene_from_params, subsurface_scene,
                           texture_images, textured_scene)


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


@pytest.mark.parametrize("name,make", [("mixture_samples", mixture_scene), ("texture_samples", textured_scene),
                                       ("subsurface_samples", subsurface_scene),
                                       ("real_texture_samples", real_textured_scene)])
def test_host_stages_mixture_match_fixture(name, make):
    fx = golden.load(name)
    scene = make(scene_from_params(fx["params"]))
    got = HostPaths(scene).samples(scene.camera, fx["pixels"], fx["samples"], int(fx["max_depth"]))
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
@pytest.mark.parametrize("name,make", [("mixture_samples", mixture_scene), ("texture_samples", textured_scene),
                                       ("subsurface_samples", subsurface_scene),
                                       ("real_texture_samples", real_textured_scene)])
def test_host_direct_mixture_against_reference(name, make):
    fx = golden.load(name)
    scene = make(scene_from_params(fx["params"]))
    R = ref.RefScene(scene)
    R.set_direct(3, 2)
    want = R.trace_samples(fx["pixels"], fx["samples"])
    for staged in (False, True):
        got = HostPaths(scene).direct_samples(scene.camera, fx["pixels"], fx["samples"], 3, 2, staged=staged)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), staged


def test_mixture_lobe_lists_and_refusals():
    """A mixture's lobes are its components' in order, black ones dropped after
    the weights apply; more than six lobes, a cycle or a component out of range
    are refused."""
    metal = dict(eta=(0.2, 0.9, 1.1), k=(3.9, 2.4, 2.1), roughness_u=0.2, roughness_v=0.2)

    def lobes(*mats):
        L = C.CDLL(HOSTPATHS)
        L.hp_material_set_lobes.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        arr = (rb.MaterialDesc * len(mats))(*mats)
        kinds = (C.c_uint32 * 8)()
        n = C.c_uint32(0)
        rb.check(L.hp_material_set_lobes(arr, len(mats), kinds, C.byref(n)), "hp_material_set_lobes")
        return [_LOBE_NAMES[kinds[i]] for i in range(n.value)]

    mix = _desc(rb.RB_MATERIAL_MIXTURE, amount=(0.5, 0.5, 0.5), components=(1, 2))
    assert lobes(mix, _desc(rb.RB_MATERIAL_MATTE, diffuse=(0.5, 0.5, 0.5)), _desc(rb.RB_MATERIAL_METAL, **metal)) == [
        "lambert", "microfacet_reflection"]
    # amount 1: the second component's weight clamp(1 - 1) = 0 makes a matte black; metal keeps its lobe
    one = _desc(rb.RB_MATERIAL_MIXTURE, amount=(1.0, 1.0, 1.0), components=(1, 2))
    assert lobes(one, _desc(rb.RB_MATERIAL_METAL, **metal), _desc(rb.RB_MATERIAL_MATTE, diffuse=(0.5, 0.5, 0.5))) == [
        "microfacet_reflection"]
    uber = _desc(rb.RB_MATERIAL_UBER, ior=1.5, opacity=(0.5, 0.5, 0.5), diffuse=(0.5, 0.5, 0.5), specular=(0.2, 0.2, 0.2),
                 reflectance=(0.1, 0.1, 0.1), transmission=(0.1, 0.1, 0.1), roughness_u=0.2, roughness_v=0.2)
    with pytest.raises(rb.RbError):  # 5 + 2 lobes
        lobes(mix, uber, _desc(rb.RB_MATERIAL_PLASTIC, ior=1.5, diffuse=(0.5, 0.5, 0.5), reflectance=(0.5, 0.5, 0.5),
                               roughness_u=0.2))
    with pytest.raises(rb.RbError):  # a mixture that contains itself
        lobes(_desc(rb.RB_MATERIAL_MIXTURE, amount=(0.5, 0.5, 0.5), components=(0, 1)),
              _desc(rb.RB_MATERIAL_MATTE, diffuse=(0.5, 0.5, 0.5)))
    with pytest.raises(rb.RbError):
        lobes(_desc(rb.RB_MATERIAL_MIXTURE, amount=(0.5, 0.5, 0.5), components=(1, 5)),
              _desc(rb.RB_MATERIAL_MATTE, diffuse=(0.5, 0.5, 0.5)))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_texture_lookup_matches_reference():
    """pt::sample_texture against image_texture2d<spectrum>::sample, bit for bit,
    at coordinates inside, outside (wrapping, negative) and on texel borders,
    for images of 1 x 1 up to 16 x 8 texels."""
    rng = np.random.default_rng(31)
    uv = np.concatenate([rng.uniform(-3.0, 3.0, (4096, 2)), rng.integers(-4, 5, (256, 2)) / 4.0,
                         rng.integers(0, 33, (256, 2)) / 32.0]).astype(np.float32)
    L = C.CDLL(HOSTPATHS)
    L.hp_texture_sample.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    for img in texture_images() + [np.float32([[[0.25, 0.5, 0.75]]]), rng.random((2, 3, 3), dtype=np.float32)]:
        img = np.ascontiguousarray(img, dtype=np.float32)
        got = np.zeros((uv.shape[0], 3), np.float32)
        L.hp_texture_sample(img.ctypes.data, img.shape[1], img.shape[0], uv.shape[0], uv.ctypes.data, got.ctypes.data)
        want = ref.texture_sample(img, uv)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), img.shape


def test_subsurface_walks_change_the_samples():
    """About half the subsurface fixture's samples go through the BSSRDF: the
    same scene with the subsurface materials made plain glass (the same lobes,
    no BSSRDF) changes them, and leaves the rest bit-equal."""
    fx = golden.load("subsurface_samples")
    scene = subsurface_scene(scene_from_params(fx["params"]))
    mats = [rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k])) for k in range(scene.desc.num_materials)]
    for m in mats:
        if m.kind == rb.RB_MATERIAL_SUBSURFACE:
            m.kind = rb.RB_MATERIAL_GLASS
    glass = scene.with_materials(mats)
    args = (fx["pixels"], fx["samples"], int(fx["max_depth"]))
    got = HostPaths(glass).samples(glass.camera, *args)
    changed = (got.view(np.uint32) != fx["radiance"].view(np.uint32)).any(axis=1).mean()
    assert 0.3 < changed < 0.7, changed


def test_subsurface_profile_table():
    """The normalized-diffusion inverse CDF (normalized_diffusion.cpp): knot k
    of the d = 1 table is the radius where cdf(r) = 1 - e^-r / 4 - 3 e^(-r / 3) / 4
    reaches k / 2047, the last knot the reference's finite end value, and a
    sample interpolates the knots linearly and scales by d."""
    lib = C.CDLL(HOSTPATHS)
    lib.hp_sss_table.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(3)
    du = np.stack([rng.random(256) * 2.0 + 0.01, rng.random(256)], axis=1).astype(np.float32)
    table = np.zeros(2048, np.float32)
    r = np.zeros(256, np.float32)
    assert lib.hp_sss_table(table.ctypes.data, 256, du.ctypes.data, r.ctypes.data) == 2048
    assert table[0] == 0.0 and np.all(np.diff(table) > 0)
    assert table[-1] == np.float32(111.686673513429369)
    k = np.arange(1, 2047)
    x = table[1:-1].astype(np.float64)
    cdf = 1.0 - np.exp(-x) / 4.0 - 0.75 * np.exp(-x / 3.0)
    assert np.all(np.abs(cdf - k / 2047.0) < 1e-6)
    u = du[:, 1] * np.float32(2047)
    which = np.minimum(u.astype(np.int64), 2046)
    t = u - which.astype(np.float32)
    want = (table[which] * (np.float32(1) - t) + table[which + 1] * t) * du[:, 0]
    assert np.array_equal(r, want.astype(np.float32))
