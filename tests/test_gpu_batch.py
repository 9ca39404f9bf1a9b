"""Batched rendering of many scenes in one wavefront (rb_batch_*) and the
launch-shape autotuner (rb_set_tuning / rb_tune_*), on the GPU.

A batch gives each scene the samples rb_render gives it alone (same per-sample
streams), so the films agree up to the grouping of FP64 additions across
waves: sums within 1e-12 relative, sample counts exactly. Launch shapes change
only speed, never the image."""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests.test_batch_host import batch_scenes

pytestmark = pytest.mark.gpu

FILM_RTOL = 1e-12


def views(scenes, spp=3):
    return [dict(camera=sc.camera, spp=spp + (k % 2), first_sample=5 * k, seed=17 + k) for k, sc in enumerate(scenes)]


def alone(scene, v, depth):
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(v["camera"], v["spp"], first_sample=v["first_sample"], max_depth=depth, seed=v["seed"],
                   want_image=False)
        return ctx.film()


def assert_films_close(got, want, what):
    s, q, c = got
    ws, wq, wc = want
    assert np.array_equal(c, wc), f"{what}: sample counts differ"
    np.testing.assert_allclose(s, ws, rtol=FILM_RTOL, atol=0, err_msg=f"{what}: sums")
    np.testing.assert_allclose(q, wq, rtol=FILM_RTOL, atol=0, err_msg=f"{what}: squared sums")


@pytest.mark.parametrize("order", [None, [2, 0, 3, 1]])
@pytest.mark.parametrize("wave,lanes", [(4096, 1), (0, 1), (3000, 3)])
def test_batch_films_equal_separate_renders(order, wave, lanes):
    scenes = batch_scenes()
    vs = views(scenes)
    depth = 6
    want = [alone(sc, v, depth) for sc, v in zip(scenes, vs)]
    with rb.Context(0) as ctx:
        # small waves hold the tail of one scene and the head of the next
        ctx.set_tuning(paths_per_wave=wave, lanes=lanes)
        ctx.batch_upload(scenes)
        ms = ctx.batch_render(vs, max_depth=depth, order=order)
        for k in range(len(scenes)):
            assert_films_close(ctx.batch_film(k), want[k], f"scene {k}")
            s, _, c = ctx.batch_film(k)
            np.testing.assert_array_equal(ctx.batch_image(k), (s / c[..., None]).astype(np.float32))
        st = ctx.stats()
        assert st.device_error == 0
        assert st.samples == sum(v["camera"].width * v["camera"].height * v["spp"] for v in vs)
    seq = list(order) if order is not None else list(range(len(scenes)))
    done = ms[seq]
    assert (done > 0).all() and (np.diff(done) >= 0).all(), f"completion times out of render order: {done}"


def test_batch_accumulates_and_refuses_single_scene_calls():
    scenes = batch_scenes()[:2]
    vs = views(scenes, spp=2)
    with rb.Context(0) as ctx:
        ctx.batch_upload(scenes)
        ctx.batch_render(vs, max_depth=5)
        vs2 = [dict(v, first_sample=v["first_sample"] + v["spp"]) for v in vs]
        ctx.batch_render(vs2, max_depth=5, reset=False)
        _, _, c = ctx.batch_film(1)
        assert (c == vs[1]["spp"] + vs2[1]["spp"]).all()
        with pytest.raises(rb.RbError):
            ctx.render(scenes[0].camera, 1)
        with pytest.raises(rb.RbError):
            ctx.batch_render(vs[:1], max_depth=5)  # one view per uploaded scene
        with pytest.raises(rb.RbError):
            ctx.batch_render(vs, max_depth=5, order=[0, 0])
        ctx.upload(scenes[0])  # a single scene replaces the batch
        ctx.render(scenes[0].camera, 1, max_depth=5, want_image=False)


@pytest.mark.parametrize("tuning", [dict(sort=rb.RB_SORT_NONE), dict(block_trace=256, block_shade=64, grid_per_sm=2),
                                    dict(block_trace=64, block_shade=256, grid_per_sm=16, paths_per_wave=1000),
                                    dict(tail_bounce=1), dict(tail_bounce=64), dict(tail_bounce=2, sort=rb.RB_SORT_NONE),
                                    dict(lanes=2, paths_per_wave=5000), dict(lanes=3, paths_per_wave=4096, tail_bounce=3),
                                    dict(lanes=4, paths_per_wave=20000), dict(traversal=rb.RB_TRAVERSAL_PER_THREAD),
                                    dict(traversal=rb.RB_TRAVERSAL_REFILL, block_trace=64, grid_per_sm=1),
                                    dict(smem_carveout=26, block_trace=256), dict(sort=rb.RB_SORT_RAYS),
                                    dict(sort=rb.RB_SORT_RAYS, lanes=2, paths_per_wave=6000, tail_bounce=4),
                                    dict(shadow_test=rb.RB_SHADOW_FIRST_OCCLUDER),
                                    dict(shadow_test=rb.RB_SHADOW_FIRST_OCCLUDER, lanes=2, paths_per_wave=6000)])
def test_launch_shapes_do_not_change_the_image(tuning):
    sc = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=96, height=64, num_spheres=30, subdivision=3)
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        ctx.render(sc.camera, 4, max_depth=8, seed=3, want_image=False)
        want = ctx.film()
        ctx.set_tuning(**tuning)
        ctx.render(sc.camera, 4, max_depth=8, seed=3, want_image=False)
        assert_films_close(ctx.film(), want, str(tuning))


def test_autotuners_pick_valid_shapes():
    sc = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=128, height=128, num_spheres=30, subdivision=3)
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        t, ms = ctx.tune_render(sc.camera, probe_spp=2, max_depth=6)
        assert ms > 0 and t.block_trace in (64, 128, 256) and t.block_shade in (64, 128, 256)
        assert t.grid_per_sm in (2, 4, 8, 16) and t.sort in (0, 1, 2) and t.paths_per_wave > 0
        assert t.tail_bounce in (1, 2, 3, 4, 6, 64) and t.lanes in (1, 2, 3, 4, 6, 8) and t.traversal in (0, 1)
        assert ctx.tuning().as_dict() == t.as_dict()
        ctx.render(sc.camera, 2, max_depth=6, want_image=False)
        assert ctx.stats().device_error == 0
        scenes = batch_scenes()
        ctx.batch_upload(scenes)
        vs = views(scenes)
        t2, ms2 = ctx.tune_batch(vs, probe_items=8000, max_depth=6)
        assert ms2 > 0
        ctx.batch_render(vs, max_depth=6)
        want = alone(scenes[2], vs[2], 6)
        assert_films_close(ctx.batch_film(2), want, "after tuning")
