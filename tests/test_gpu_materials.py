"""Plastic, mirror, substrate, Oren-Nayar, uber, translucent, mixture and subsurface materials and image
textures on the GPU: with spp = 1 the film sum of a pixel
is one sample's radiance, against the reference's path_integrator::trace on the
spheres scene with plastic, mirror and substrate materials (golden fixture), and the same
scene in direct lighting against the host build."""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.helpers import (HostPaths, assert_disagreements_unbiased, extra_materials_scene, layered_scene,
                           mixture_scene, oren_nayar_scene, per_sample_radiance, real_textured_scene, scene_from_params,
                           subsurface_scene, textured_scene, two_level_scene)

pytestmark = pytest.mark.gpu

SAMPLE_RTOL = 1e-3


def _agreement(gpu, want):
    ok = np.abs(gpu - want) <= SAMPLE_RTOL * np.maximum(1.0, np.abs(want))
    return ok.all(axis=1).mean()


def test_extra_materials_samples_match_reference():
    fx = golden.load("materials_samples")
    scene = extra_materials_scene(scene_from_params(fx["params"]))
    depth = int(fx["max_depth"])
    px, sm, want = fx["pixels"], fx["samples"], fx["radiance"]
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, px, sm, depth)
        assert ctx.stats().device_error == 0
    agree = _agreement(got, want)
    assert agree >= 0.97, f"only {agree:.4f} of samples agree with the reference"
    assert_disagreements_unbiased(scene, got, want, fx["first_entity"], "materials")


def test_oren_nayar_samples_match_reference():
    fx = golden.load("oren_nayar_samples")
    scene = oren_nayar_scene(scene_from_params(fx["params"]))
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, fx["pixels"], fx["samples"], int(fx["max_depth"]))
        assert ctx.stats().device_error == 0
    agree = _agreement(got, fx["radiance"])
    assert agree >= 0.97, f"only {agree:.4f} of samples agree with the reference"
    assert_disagreements_unbiased(scene, got, fx["radiance"], fx["first_entity"], "oren-nayar")


@pytest.mark.parametrize("name,make", [("layered_samples", layered_scene), ("mixture_samples", mixture_scene),
                                       ("texture_samples", textured_scene), ("subsurface_samples", subsurface_scene),
                                       ("real_texture_samples", real_textured_scene)])
def test_layered_samples_match_reference(name, make):
    fx = golden.load(name)
    scene = make(scene_from_params(fx["params"]))
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, fx["pixels"], fx["samples"], int(fx["max_depth"]))
        assert ctx.stats().device_error == 0
    agree = _agreement(got, fx["radiance"])
    assert agree >= 0.97, f"only {agree:.4f} of samples agree with the reference"
    assert_disagreements_unbiased(scene, got, fx["radiance"], fx["first_entity"], name)


@pytest.mark.parametrize("name,make", [("layered_samples", layered_scene), ("mixture_samples", mixture_scene),
                                       ("texture_samples", textured_scene), ("subsurface_samples", subsurface_scene),
                                       ("real_texture_samples", real_textured_scene)])
def test_layered_direct_matches_host_build(name, make):
    fx = golden.load(name)
    scene = make(scene_from_params(fx["params"]))
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).direct_samples(scene.camera, px, np.full_like(px, 2), 4, 4)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=1, first_sample=2, want_image=False, direct=(4, 4))
        sums, _, cnt = ctx.film()
    assert (cnt == 1).all()
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"only {agree:.4f} of pixels agree"


def test_extra_materials_direct_matches_host_build():
    fx = golden.load("materials_samples")
    scene = extra_materials_scene(scene_from_params(fx["params"]))
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).direct_samples(scene.camera, px, np.full_like(px, 2), 4, 4)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=1, first_sample=2, want_image=False, direct=(4, 4))
        sums, _, cnt = ctx.film()
    assert (cnt == 1).all()
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"only {agree:.4f} of pixels agree"


@pytest.mark.parametrize("tuning", [dict(), dict(sort=rb.RB_SORT_NONE), dict(tail_bounce=2),
                                    dict(traversal=rb.RB_TRAVERSAL_REFILL), dict(lanes=2, paths_per_wave=3000)])
def test_subsurface_image_matches_host_build(tuning):
    """Whole 1-spp image of the subsurface scene against the host build of the
    same stages (every pixel's sample 5), under several launch shapes (a tail
    bounce below the depth is ignored: subsurface scenes run every bounce
    staged); the BSSRDF stage is taken by about half the paths."""
    fx = golden.load("subsurface_samples")
    scene = subsurface_scene(scene_from_params(fx["params"]))
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).samples(scene.camera, px, np.full_like(px, 5), 8)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        if tuning:
            ctx.set_tuning(**tuning)
        ctx.render(scene.camera, spp=1, first_sample=5, max_depth=8, want_image=False)
        sums, _, cnt = ctx.film()
        st = ctx.stats()
    assert (cnt == 1).all() and st.device_error == 0
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"only {agree:.4f} of pixels agree ({tuning})"


def test_subsurface_refuses_guided_and_volume_renders():
    fx = golden.load("subsurface_samples")
    scene = subsurface_scene(scene_from_params(fx["params"]))
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        for kw in (dict(volume=True), dict(guide=True), dict(train=True)):
            with pytest.raises(rb.RbError) as e:
                ctx.render(scene.camera, spp=1, max_depth=8, want_image=False, **kw)
            assert e.value.status == 7, kw  # RB_ERR_UNSUPPORTED
        ctx.render(scene.camera, spp=1, max_depth=8, want_image=False)  # the context stays usable
        assert ctx.stats().device_error == 0


def test_subsurface_two_level_image_matches_host_build():
    """The subsurface stage on a scene with the two-level tree (instance slots: a shared mesh and a
    327,680-triangle mesh, every third material subsurface): whole 1-spp image against the host build."""
    scene = subsurface_scene(two_level_scene(48, 40))
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).samples(scene.camera, px, np.full_like(px, 4), 8)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=1, first_sample=4, max_depth=8, want_image=False)
        sums, _, cnt = ctx.film()
        assert ctx.stats().device_error == 0
    assert (cnt == 1).all()
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"only {agree:.4f} of pixels agree"
