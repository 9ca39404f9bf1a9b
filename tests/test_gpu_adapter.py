"""The drop-in on the reference side: wavefront_path_integrator
(rainbow_b200/adapter), compiled against the reference's headers, renders a
reference `scene` through the reference's own entry point
integrator::render(camera, scene) (integrator.hpp:64-66) and leaves its result
in the reference `film` through film::set_pixel (film.cpp:197-205). The film
must hold what rb_render computes for the same samples, and lie within 3 sigma
of path_integrator::render as shipped (the reference's own per-tile sampler
streams) on the same scene."""
import ctypes

import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import ref
from tests import golden
from tests.helpers import scene_from_params

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.adapter_available(), reason="oracle/_ref/libadapter_check.so not built")]


def test_adapter_film_equals_rb_render():
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=48, height=40, num_spheres=12, subdivision=2)
    R = ref.RefScene(scene)
    film = ref.adapter_render(R, 16, max_depth=8, threshold=1.0, seed=5)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        img = ctx.render(scene.camera, 16, max_depth=8, seed=5)
    np.testing.assert_array_equal(film, img)


def test_adapter_film_within_three_sigma_of_shipped_path_integrator():
    fx = golden.load("box_image")  # per-pixel variance of the reference's 256-spp render
    scene = scene_from_params(fx["params"])
    n = int(fx["spp"])
    var = np.maximum(fx["sum_sq"] / n - (fx["sum"] / n) ** 2, 0.0)
    R = ref.RefScene(scene)
    film = ref.adapter_render(R, n, max_depth=5, threshold=1.0, seed=2).astype(np.float64)
    shipped, _ = R.render_shipped(n, max_depth=5, rr=1.0)
    se = np.sqrt(2.0 * var / n)
    z = np.where(se > 0, (film - shipped) / np.where(se > 0, se, 1), 0.0)
    assert (np.abs(z) > 3).mean() < 0.01, f"{(np.abs(z) > 3).mean():.4f} of pixel channels outside 3 sigma"
    assert abs(z.mean()) < 0.1, z.mean()


def test_adapter_two_level_scene_and_refusal():
    """The two-level scene renders through the adapter. A scene the core does
    not render (no emitter: uniform_sample_one_emitter needs one) makes render()
    throw with the C ABI's reason and leaves the film as it was."""
    from tests.helpers import two_level_scene
    scene = two_level_scene(32, 24)
    R = ref.RefScene(scene)
    film = ref.adapter_render(R, 4, max_depth=5)
    assert np.isfinite(film).all() and film.mean() > 0
    dark = rb.SceneDesc.from_buffer_copy(bytes(scene.desc))
    ents = (rb._native.EntityDesc * dark.num_entities)()
    for k in range(dark.num_entities):
        ents[k] = scene.desc.entities[k]
        ents[k].emitter = -1
    dark.entities = ctypes.cast(ents, ctypes.POINTER(rb._native.EntityDesc))
    dark.num_emitters = 0
    R2 = ref.RefScene(rb.Scene(None, dark, scene.camera, keepalive=[scene, ents]))
    before = R2.film()
    with pytest.raises(RuntimeError, match="invalid argument"):
        ref.adapter_render(R2, 4)
    np.testing.assert_array_equal(R2.film(), before)


def test_photon_adapter_film_matches_rb_render_photons_and_the_reference():
    """wavefront_photon_mapping_integrator::render on a reference scene writes what
    rb_render_photons computes (up to the order of the photon flux sums), and over
    several seeds estimates the image of photon_mapping_integrator::render as shipped."""
    from tests.golden.make_golden import PHOTON_CASES, photon_scene
    _, params, variant, it, depth, photons, radius = next(c for c in PHOTON_CASES if c[0] == "box")
    scene = photon_scene(params, variant)
    R = ref.RefScene(scene)
    films = np.stack([ref.adapter_render_photons(R, it, depth, photons, radius, seed=s) for s in range(6)])
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        img = ctx.render_photons(scene.camera, it, depth, photons, radius, seed=0)
    close = (np.abs(films[0] - img) <= 1e-3 * np.maximum(np.abs(img), 1e-2)).all(axis=2)
    assert close.mean() >= 0.95, close.mean()
    shipped = golden.load("photons_box")["image"]
    blocks = films.reshape(6, 4, 8, 4, 8, 3).mean(axis=(2, 4))
    want = shipped.reshape(4, 8, 4, 8, 3).mean(axis=(1, 3))
    mean, sd = blocks.mean(axis=0), blocks.std(axis=0, ddof=1)
    z = (mean - want) / np.maximum(sd * np.sqrt(1 + 1 / 6), 1e-3 * np.abs(want) + 1e-6)
    assert np.abs(z).max() < 6.0, np.abs(z).max()
