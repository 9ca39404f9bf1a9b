"""rb_render_photons (stochastic progressive photon mapping, photon_mapping_integrator.cpp)
on the GPU: against the host build of the same stage functions with the same per-pixel
and per-photon streams (the kernels' float sums of the photon flux run in another order,
so pixels agree to a tolerance), and against the compiled reference's images (golden
fixtures): the mean over several seeds within a few standard errors, per 8 x 8 block."""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.golden.make_golden import PHOTON_CASES, photon_scene
from tests.helpers import HostPaths, two_level_scene

pytestmark = pytest.mark.gpu

PIXEL_RTOL = 1e-3


def _case(name):
    return next(c for c in PHOTON_CASES if c[0] == name)


@pytest.mark.parametrize("name", ["box", "spheres", "materials"])
def test_photon_render_matches_host_build(name):
    _, params, variant, it, depth, photons, radius = _case(name)
    scene = photon_scene(params, variant)
    want = HostPaths(scene).photon_render(scene.camera, it, depth, photons, radius, streams=1, seed=7)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = ctx.render_photons(scene.camera, it, depth, photons, radius, seed=7)
    assert np.isfinite(got).all()
    close = (np.abs(got - want) <= PIXEL_RTOL * np.maximum(np.abs(want), 1e-2)).all(axis=2)
    assert close.mean() >= 0.95, f"only {close.mean():.4f} of pixels agree"
    assert abs(got.mean() / want.mean() - 1.0) < 2e-3


@pytest.mark.parametrize("name", ["box", "spheres", "materials"])
def test_photon_render_estimates_the_reference_image(name):
    _, params, variant, it, depth, photons, radius = _case(name)
    fx = golden.load(f"photons_{name}")
    scene = photon_scene(params, variant)
    H, W = fx["image"].shape[:2]
    seeds = 8
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        runs = np.stack([ctx.render_photons(scene.camera, it, depth, photons, radius, seed=s) for s in range(seeds)])
    hb, wb = H // 8, W // 8
    blocks = runs[:, :hb * 8, :wb * 8].reshape(seeds, hb, 8, wb, 8, 3).mean(axis=(2, 4))
    want = fx["image"][:hb * 8, :wb * 8].reshape(hb, 8, wb, 8, 3).mean(axis=(1, 3))
    mean, sd = blocks.mean(axis=0), blocks.std(axis=0, ddof=1)
    z = (mean - want) / np.maximum(sd * np.sqrt(1 + 1 / seeds), 1e-3 * np.abs(want) + 1e-6)
    assert np.abs(z).max() < 6.0, np.abs(z).max()
    assert abs(mean.mean() / want.mean() - 1.0) < 0.05


def test_photon_render_arguments():
    scene = photon_scene(_case("box")[1], None)
    with rb.Context(0) as ctx:
        with pytest.raises(rb.RbError):
            ctx.render_photons(scene.camera, 2, 5, 0, 0.1)  # no scene yet
        ctx.upload(scene)
        for kw in (dict(iterations=0), dict(radius=0.0), dict(max_depth=0), dict(max_depth=65)):
            args = dict(iterations=2, max_depth=5, photons=0, radius=0.1)
            args.update(kw)
            with pytest.raises(rb.RbError):
                ctx.render_photons(scene.camera, **args)
        img = ctx.render_photons(scene.camera, 2, 5, 1000, 0.1)
        assert np.isfinite(img).all() and img.mean() > 0.0
        ctx.render(scene.camera, 1, max_depth=5)  # the context stays usable for path tracing
        assert ctx.stats().device_error == 0


def test_photon_render_two_level_scene_matches_host_build():
    """A scene with the two-level tree (a shared mesh and a 327,680-triangle mesh): the photon kernels'
    instance-slot traversal against the host build with the same streams."""
    scene = two_level_scene(48, 40)
    want = HostPaths(scene).photon_render(scene.camera, 3, 5, 0, 0.3, streams=1, seed=3)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = ctx.render_photons(scene.camera, 3, 5, 0, 0.3, seed=3)
    close = (np.abs(got - want) <= PIXEL_RTOL * np.maximum(np.abs(want), 1e-2)).all(axis=2)
    assert close.mean() >= 0.95, f"only {close.mean():.4f} of pixels agree"
    assert want.mean() > 0.0 and abs(got.mean() / want.mean() - 1.0) < 2e-3
