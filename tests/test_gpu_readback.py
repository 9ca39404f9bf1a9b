"""rb_render into page-locked memory copies each slice of the image as soon as
its pixels have all of the call's samples, while later waves still run; the
image must be the one a pageable buffer receives after the call (one copy at
the end), for any wave size, lane count and samples per pixel."""
import numpy as np
import pytest

import rainbow_b200 as rb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spp,tuning", [(1, dict(lanes=4, paths_per_wave=1500)), (3, dict(lanes=2, paths_per_wave=2500)),
                                        (2, dict(lanes=1, paths_per_wave=1000)), (5, dict(lanes=3, paths_per_wave=64 * 40))])
def test_page_locked_output_equals_pageable(spp, tuning):
    torch = pytest.importorskip("torch")
    sc = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=2, width=64, height=40, num_spheres=20, subdivision=2)
    with rb.Context(0) as ctx:
        ctx.upload(sc)
        ctx.set_tuning(**tuning)
        want = ctx.render(sc.camera, spp, max_depth=6, seed=3)
        pinned = torch.full((40, 64, 3), -1.0, dtype=torch.float32, pin_memory=True).numpy()
        got = ctx.render(sc.camera, spp, max_depth=6, seed=3, out=pinned)
        assert got is pinned
        assert np.array_equal(pinned, want)
        # a progressive call: the means over both calls' samples
        want2 = ctx.render(sc.camera, spp, first_sample=spp, max_depth=6, seed=3, reset=False)
        ctx.render(sc.camera, spp, max_depth=6, seed=3)
        ctx.render(sc.camera, spp, first_sample=spp, max_depth=6, seed=3, reset=False, out=pinned)
        assert np.array_equal(pinned, want2)
        assert ctx.stats().device_error == 0
