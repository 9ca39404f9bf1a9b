"""Stochastic progressive photon mapping (photon_mapping_integrator.cpp) through the
photon stage functions compiled for the host (pt/pt_photon.h), run in the reference's
own order and streams: bit-equal to the compiled reference's render (golden fixtures,
and the reference itself where it is built), on the box room, the sphere scene and the
sphere scene with plastic, mirror and substrate materials; more scenes (layered,
mixture, textured and subsurface materials, invisible medium boundaries) against the
reference directly; with real parameters from textures too."""
import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import ref
from tests import golden
from tests.golden.make_golden import PHOTON_CASES, photon_scene
from tests.helpers import (HostPaths, layered_scene, mixture_scene, real_textured_scene, scene_from_params, subsurface_scene,
                           textured_scene, two_level_scene)


@pytest.mark.parametrize("case", PHOTON_CASES, ids=[c[0] for c in PHOTON_CASES])
def test_host_photon_render_matches_fixture(case):
    name, params, variant, it, depth, photons, radius = case
    fx = golden.load(f"photons_{name}")
    scene = photon_scene(params, variant)
    assert np.array_equal(fx["params"], np.array([params[k] for k in ("kind", "seed", "width", "height", "num_spheres",
                                                                       "subdivision")]))
    got = HostPaths(scene).photon_render(scene.camera, it, depth, photons, radius, streams=0)
    assert np.array_equal(got.view(np.uint32), fx["image"].view(np.uint32))
    assert fx["image"].mean() > 0.0


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
@pytest.mark.parametrize("variant", ["layered", "mixture", "textured", "real_textured", "subsurface", "fog", "two_level"])
def test_host_photon_render_against_reference(variant):
    base = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=3, width=40, height=32, num_spheres=10, subdivision=2)
    scene = {"layered": lambda: layered_scene(base), "mixture": lambda: mixture_scene(base),
             "textured": lambda: textured_scene(base), "real_textured": lambda: real_textured_scene(base),
             "subsurface": lambda: subsurface_scene(base),
             "fog": lambda: rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=40, height=30, num_spheres=6,
                                              subdivision=2),
             "two_level": lambda: two_level_scene(40, 30)}[variant]()
    want, _ = ref.RefScene(scene).render_photons(4, 6, 2500, 0.3)
    got = HostPaths(scene).photon_render(scene.camera, 4, 6, 2500, 0.3, streams=0)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_host_photon_streams_estimate_the_same_image():
    """The kernels' per-pixel and per-photon streams give an estimate of the same
    image: over the box room, the mean of several seeds is within a few standard
    errors of the reference-order render (blocks of 8 x 8 pixels)."""
    fx = golden.load("photons_box")
    scene = scene_from_params(fx["params"])
    it, depth, photons, radius = int(fx["iterations"]), int(fx["max_depth"]), int(fx["photons"]), float(fx["radius"])
    hp = HostPaths(scene)
    runs = np.stack([hp.photon_render(scene.camera, it, depth, photons, radius, streams=1, seed=s) for s in range(6)])
    blocks = runs.reshape(6, 4, 8, 4, 8, 3).mean(axis=(2, 4))
    want = fx["image"].reshape(4, 8, 4, 8, 3).mean(axis=(1, 3))
    mean, sd = blocks.mean(axis=0), blocks.std(axis=0, ddof=1)
    z = (mean - want) / np.maximum(sd * np.sqrt(1 + 1 / 6), 1e-3 * np.abs(want) + 1e-6)
    assert np.abs(z).max() < 6.0, np.abs(z).max()
    assert abs(mean.mean() / want.mean() - 1.0) < 0.05
