"""Scenes with invisible entities (here the boundary of the fog's medium): a
pass through one is not a bounce, so a wave keeps bouncing after max_depth
iterations until its paths are done. That drain loop runs inside each wave's
CUDA graph as a conditional WHILE node, on one or several wave lanes; the
host-driven loop of direct launches (the profiling path) must give the same
paths and the same film."""
import pytest

import rainbow_b200 as rb
from tests.test_gpu_batch import assert_films_close

pytestmark = pytest.mark.gpu


def _fog():
    return rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=64, height=48, num_spheres=12, subdivision=2)


@pytest.mark.parametrize("volume", [True, False])
def test_drain_graph_equals_host_loop(volume):
    sc = _fog()
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        # depth 3: most paths cross the medium's boundary more often than that
        ctx.set_profiling(True)
        ctx.render(sc.camera, 8, max_depth=3, seed=3, volume=volume, want_image=False, paths_per_wave=4096)
        want, want_rays = ctx.film(), ctx.stats().extend_rays
        assert ctx.stats().device_error == 0
        ctx.set_profiling(False)
        for tuning in (dict(lanes=1, paths_per_wave=4096), dict(lanes=3, paths_per_wave=4096),
                       dict(lanes=2, paths_per_wave=7000, sort=rb.RB_SORT_NONE)):
            ctx.set_tuning(**tuning)
            ctx.render(sc.camera, 8, max_depth=3, seed=3, volume=volume, want_image=False)
            st = ctx.stats()
            assert st.device_error == 0, tuning
            assert st.extend_rays == want_rays, tuning
            assert_films_close(ctx.film(), want, str(tuning))


def test_guided_waves_on_lanes_with_invisible_entities():
    """Guided path tracing with online training on wave lanes, on a scene whose
    waves drain past max_depth: no device error, the guide trains, and the
    image mean agrees with a converged plain render."""
    sc = rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=32, height=24, num_spheres=12, subdivision=2)
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        ref = ctx.render(sc.camera, 8192, max_depth=5, seed=100)
        ctx.set_tuning(lanes=2, paths_per_wave=8192)
        ctx.guide_init(seed=0, batch_size=8192, min_rows=1024, steps_per_wave=2)
        ctx.render(sc.camera, 512, max_depth=5, seed=7, guide=True, train=True, want_image=False)
        assert ctx.guide_stats().steps > 0
        img = ctx.render(sc.camera, 4096, max_depth=5, seed=9, guide=True)
        assert ctx.stats().device_error == 0
    assert abs(float(img.mean()) / float(ref.mean()) - 1.0) < 0.02, (img.mean(), ref.mean())


@pytest.mark.parametrize("wave,lanes", [(0, 1), (3000, 2)])
def test_batch_with_invisible_entities_equals_separate_renders(wave, lanes):
    """A batch holding a scene with invisible entities drains each wave inside
    its graph too: every scene's film equals the film of rendering it alone."""
    from tests.test_gpu_batch import alone, views
    scenes = [_fog(), rb.generate_scene(rb.RB_SCENE_SPHERES, seed=5, width=40, height=30, num_spheres=12, subdivision=2)]
    vs = views(scenes)
    want = [alone(sc, v, 4) for sc, v in zip(scenes, vs)]
    with rb.Context(0) as ctx:
        ctx.set_tuning(paths_per_wave=wave, lanes=lanes)
        ctx.batch_upload(scenes)
        ctx.batch_render(vs, max_depth=4)
        for k in range(len(scenes)):
            assert_films_close(ctx.batch_film(k), want[k], f"scene {k}")
        assert ctx.stats().device_error == 0
