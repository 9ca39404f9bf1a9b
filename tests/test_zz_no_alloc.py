"""rb_render_noalloc: the render for callers that cannot allocate device memory
while rendering (a framework that owns the device memory pool, or a loop where
cudaMalloc's implicit synchronisation is not allowed).

The entry point keeps all of its scratch in a fixed static device array and
adds its samples to device accumulators the caller owns. This test calls it
through the C ABI twice in a row and checks the accumulators against the ones
rb_render (which allocates its own buffers) produces for the same samples: on
the box room, and on a fog scene whose invisible medium boundary makes paths
outlive max_depth iterations (the drain loop), also right after a volume
render on the same context. It also checks that the integrators the entry
point does not run (volume, direct lighting, guiding) are refused rather than
replaced by plain path tracing. The test allocates its own buffers with torch;
the entry point allocates nothing.
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


def _params(camera, first_sample, depth=5, flags=0):
    p = rb.RenderParams()
    p.camera = camera
    p.spp, p.first_sample, p.max_depth, p.rr_threshold, p.seed = SPP, first_sample, depth, 1.0, 0
    p.flags = flags
    return p


def _accumulators(w, h):
    d_sum = torch.zeros(w * h * 3, dtype=torch.float64, device="cuda")
    d_sq = torch.zeros(w * h * 3, dtype=torch.float64, device="cuda")
    d_cnt = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    return d_sum, d_sq, d_cnt


def _noalloc_calls(ctx, camera, acc, depth, flags_first=0):
    d_sum, d_sq, d_cnt = acc
    for k, first in enumerate((0, SPP)):
        p = _params(camera, first, depth, flags_first if k == 0 else 0)
        st = rb.lib().rb_render_noalloc(ctx._h, ctypes.byref(p), d_sum.data_ptr(), d_sq.data_ptr(), d_cnt.data_ptr(), None)
        assert st == 0, _native.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()


def _assert_equal_films(acc, want, w, h):
    d_sum, d_sq, d_cnt = acc
    want_sum, want_sq, want_cnt = want
    got_cnt = d_cnt.cpu().numpy().reshape(h, w).view(np.uint32)
    assert np.array_equal(got_cnt, want_cnt)
    assert (got_cnt == 2 * SPP).all()
    np.testing.assert_allclose(d_sum.cpu().numpy().reshape(h, w, 3), want_sum, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(d_sq.cpu().numpy().reshape(h, w, 3), want_sq, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("subsurface", [False, True])
def test_noalloc_render_matches_allocating_render_on_two_calls(subsurface):
    """Also on the box room with a subsurface material (the subsurface stage's queue lives in the scratch)."""
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=W, height=H)
    if subsurface:
        from tests.helpers import subsurface_scene
        scene = subsurface_scene(scene)
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


def test_noalloc_drains_paths_through_invisible_entities():
    """Fog scene (an invisible box holding the medium around the clutter),
    plain path tracing at depth 3: most paths pass the boundary more often than
    that, so the film is only complete if the call keeps bouncing until every
    path is done. A volume render first leaves the context set up for media; the
    no-alloc call must still run the plain integrator on its own buffers. The
    first call also passes RB_RENDER_RESET over accumulators that hold junk."""
    w, h = 48, 32
    scene = rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=w, height=h, num_spheres=12, subdivision=2)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=SPP, first_sample=0, max_depth=3, reset=True, want_image=False)
        ctx.render(scene.camera, spp=SPP, first_sample=SPP, max_depth=3, reset=False, want_image=False)
        want = ctx.film()
        assert ctx.stats().device_error == 0
        ctx.render(scene.camera, spp=1, max_depth=3, reset=True, volume=True, want_image=False)
        acc = _accumulators(w, h)
        for t in acc:
            t.fill_(7)
        _noalloc_calls(ctx, scene.camera, acc, depth=3, flags_first=rb.RB_RENDER_RESET)
        _assert_equal_films(acc, want, w, h)


@pytest.mark.parametrize("flag", ["RB_RENDER_VOLUME", "RB_RENDER_DIRECT", "RB_RENDER_GUIDE", "RB_RENDER_TRAIN"])
def test_noalloc_refuses_other_integrators(flag):
    scene = rb.generate_scene(rb.RB_SCENE_BOX, width=W, height=H)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        d_sum, d_sq, d_cnt = _accumulators(W, H)
        p = _params(scene.camera, 0, flags=getattr(rb, flag))
        st = rb.lib().rb_render_noalloc(ctx._h, ctypes.byref(p), d_sum.data_ptr(), d_sq.data_ptr(), d_cnt.data_ptr(), None)
        assert st == 7, _native.STATUS_NAMES.get(st, st)  # RB_ERR_UNSUPPORTED
        assert int(d_cnt.sum().item()) == 0


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
        # a camera too large for any film is refused before its paths are counted
        p = _params(scene.camera, 0)
        p.camera.width = p.camera.height = 1 << 15
        assert rb.lib().rb_render_noalloc(ctx._h, ctypes.byref(p), buf.data_ptr(), buf.data_ptr(), cnt.data_ptr(),
                                          None) == 1
