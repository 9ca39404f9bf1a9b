"""direct_integrator (RB_RENDER_DIRECT) on the host: pt::direct_radiance, the
function the k_direct kernel runs, compiled for the CPU with the kernels'
traversal, against the reference's own direct_integrator::trace (golden
fixtures made by tests/golden/make_golden.py from the compiled reference):
bit-equal radiance per (pixel, sample), with the default 4 + 4 samples on the
spheres scene (environment light, quad lights, metal and glass) and with
2 + 3 samples on the fog scene (rays through an invisible boundary)."""
import numpy as np
import pytest

from oracle import ref
from tests import golden
from tests.helpers import HostPaths, scene_from_params


@pytest.mark.parametrize("staged", [False, True])
@pytest.mark.parametrize("name", ["direct_spheres", "direct_fog"])
def test_host_direct_matches_fixture(name, staged):
    """Both forms: the one-function sample and the stage functions in the staged kernels' order."""
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    got = HostPaths(scene).direct_samples(scene.camera, fx["pixels"], fx["samples"], int(fx["emitter_samples"]),
                                          int(fx["bsdf_samples"]), staged=staged)
    assert np.array_equal(got.view(np.uint32), fx["radiance"].view(np.uint32))


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
def test_host_direct_against_reference_other_counts():
    """Sample counts the fixtures do not cover, straight against the compiled reference."""
    import rainbow_b200 as rb
    scene = rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=40, height=40, num_spheres=12, subdivision=2)
    R = ref.RefScene(scene)
    rng = np.random.default_rng(3)
    px = rng.integers(0, 40 * 40, 400).astype(np.uint32)
    sm = rng.integers(0, 500, 400).astype(np.uint32)
    hp = HostPaths(scene)
    for E, B in ((1, 1), (3, 1), (1, 5), (8, 2)):
        R.set_direct(E, B)
        want = R.trace_samples(px, sm)
        for staged in (False, True):
            got = hp.direct_samples(scene.camera, px, sm, E, B, staged=staged)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (E, B, staged)
