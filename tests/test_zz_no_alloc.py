"""rb_render_noalloc: the render for callers that cannot allocate device memory
while rendering (a framework that owns the device memory pool, or a loop where
cudaMalloc's implicit synchronisation is not allowed).

The entry point keeps all of its scratch in a fixed static device array and
adds its samples to device accumulators the caller owns. This test calls it
through the C ABI twice in a row and checks the accumulators against the ones
rb_render (which allocates its own buffers) produces for the same samples. The
test allocates its own buffers with torch; the entry point allocates nothing.
"""
import ctypes

import numpy as np
import pytest
import torch

import rainbow_b200 as rb
from rainbow_b200 import _native

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 2  # per call: 64 * 64 * 2 = 8192 paths, within the 16,384-path limit


def _params(camera, first_sample):
    p = rb.RenderParams()
    p.camera = camera
    p.spp, p.first_sample, p.max_depth, p.rr_threshold, p.seed = SPP, first_sample, 5, 1.0, 0
    return p


def test_noalloc_render_matches_allocating_render_on_two_calls():
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=W, height=H)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        # the existing entry point: two calls, accumulating
        ctx.render(scene.camera, spp=SPP, first_sample=0, max_depth=5, reset=True, want_image=False)
        ctx.render(scene.camera, spp=SPP, first_sample=SPP, max_depth=5, reset=False, want_image=False)
        want_sum, want_sq, want_cnt = ctx.film()

        d_sum = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
        d_sq = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
        d_cnt = torch.zeros(W * H, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        lib = rb.lib()
        for first in (0, SPP):
            st = lib.rb_render_noalloc(ctx._h, ctypes.byref(_params(scene.camera, first)), d_sum.data_ptr(),
                                       d_sq.data_ptr(), d_cnt.data_ptr(), None)
            assert st == 0, _native.STATUS_NAMES.get(st, st)
        torch.cuda.synchronize()
        got_cnt = d_cnt.cpu().numpy().reshape(H, W).view(np.uint32)
        assert np.array_equal(got_cnt, want_cnt)
        assert (got_cnt == 2 * SPP).all()
        np.testing.assert_allclose(d_sum.cpu().numpy().reshape(H, W, 3), want_sum, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(d_sq.cpu().numpy().reshape(H, W, 3), want_sq, rtol=1e-12, atol=1e-12)


def test_noalloc_rejects_work_beyond_its_scratch():
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=128, height=128)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        buf = torch.zeros(128 * 128 * 3, dtype=torch.float64, device="cuda")
        cnt = torch.zeros(128 * 128, dtype=torch.int32, device="cuda")
        st = rb.lib().rb_render_noalloc(ctx._h, ctypes.byref(_params(scene.camera, 0)), buf.data_ptr(), buf.data_ptr(),
                                        cnt.data_ptr(), None)
        assert st == 12  # RB_ERR_TOO_LARGE: 128 * 128 * 2 paths > 16,384
        assert b"scratch" in rb.lib().rb_status_string(st)
        assert rb.lib().rb_render_noalloc(ctx._h, None, buf.data_ptr(), buf.data_ptr(), cnt.data_ptr(), None) == 1
