"""rb_render_async / rb_render_wait: consecutive one-sample calls enqueued
without waiting overlap on the GPU, and must leave exactly what the same
synchronous rb_render calls leave: the film (sums, squared sums, counts) and
every call's image in its own page-locked buffer."""
import ctypes

import numpy as np
import pytest
import torch

import rainbow_b200 as rb
from tests.test_gpu_batch import assert_films_close

pytestmark = pytest.mark.gpu

STEPS = 5


def _scene():
    return rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=96, height=64, num_spheres=30, subdivision=3)


# lanes=4 with one wave per call and lanes=3 with two: the calls' waves take the lanes in turn across calls
@pytest.mark.parametrize("tuning", [dict(lanes=1, paths_per_wave=3000), dict(lanes=3, paths_per_wave=2048),
                                    dict(lanes=4, paths_per_wave=6144), dict(lanes=3, paths_per_wave=4096)])
def test_async_calls_equal_sync_calls(tuning):
    sc = _scene()
    W, H = sc.camera.width, sc.camera.height
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        ctx.set_tuning(**tuning)
        want_imgs = []
        for k in range(STEPS):
            want_imgs.append(ctx.render(sc.camera, 1, first_sample=k, max_depth=8, seed=3, reset=(k == 0)))
        want = ctx.film()
        bufs = [torch.zeros((H, W, 3), dtype=torch.float32, pin_memory=True) for _ in range(STEPS)]
        for k in range(STEPS):
            ctx.render_async(sc.camera, 1, first_sample=k, max_depth=8, seed=3, reset=(k == 0),
                             out_ptr=bufs[k].data_ptr())
        ctx.render_wait()
        st = ctx.stats()
        assert st.device_error == 0 and st.samples == STEPS * W * H
        assert_films_close(ctx.film(), want, str(tuning))
        for k in range(STEPS):
            np.testing.assert_allclose(bufs[k].numpy(), want_imgs[k], rtol=1e-6, atol=1e-7, err_msg=f"call {k}")


def test_async_rules():
    sc = _scene()
    W, H = sc.camera.width, sc.camera.height
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        p = rb.RenderParams()
        p.camera = sc.camera
        p.spp, p.max_depth, p.rr_threshold, p.flags = 1, 5, 1.0, rb.RB_RENDER_VOLUME
        assert rb.lib().rb_render_async(ctx._h, ctypes.byref(p), None) == 7  # RB_ERR_UNSUPPORTED
        pageable = np.zeros((H, W, 3), dtype=np.float32)
        p.flags = 0
        assert rb.lib().rb_render_async(ctx._h, ctypes.byref(p), pageable.ctypes.data) == 1
        # a synchronous call after pending async calls waits for them first, and the film holds all samples
        ctx.render_async(sc.camera, 2, first_sample=0, max_depth=5, reset=True)
        ctx.render_async(sc.camera, 2, first_sample=2, max_depth=5)
        ctx.render(sc.camera, 2, first_sample=4, max_depth=5, reset=False, want_image=False)
        assert (ctx.film()[2] == 6).all()
        assert rb.lib().rb_render_wait(ctx._h) == 0  # nothing pending
