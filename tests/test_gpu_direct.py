"""direct_integrator on the GPU (RB_RENDER_DIRECT, the k_direct kernel):

- per sample: with spp = 1 the film sum of a pixel is one sample's radiance;
  against the reference's direct_integrator::trace (golden fixtures) nearly
  every sample agrees to float rounding (a few diverge where CUDA's
  sin/cos/log round differently from glibc's and a sample then picks another
  lobe or light);
- every pixel of one sample index against the host build of the same
  function;
- the sample counts reach the kernel (default 4 + 4, and explicit counts), and
  direct lighting refuses to combine with guiding or volumes.
"""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.helpers import HostPaths, scene_from_params

pytestmark = pytest.mark.gpu

SAMPLE_RTOL = 1e-3


def _agreement(gpu, ref):
    ok = np.abs(gpu - ref) <= SAMPLE_RTOL * np.maximum(1.0, np.abs(ref))
    return ok.all(axis=1).mean()


@pytest.mark.parametrize("name", ["direct_spheres", "direct_fog"])
def test_direct_samples_match_reference(name):
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    counts = (int(fx["emitter_samples"]), int(fx["bsdf_samples"]))
    px, sm, want = fx["pixels"], fx["samples"], fx["radiance"]
    got = np.zeros_like(want)
    idx = np.unique(sm)[:64]
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        for s in idx:
            ctx.render(scene.camera, spp=1, first_sample=int(s), want_image=False, direct=counts)
            sums, _, cnt = ctx.film()
            sel = sm == s
            got[sel] = sums.reshape(-1, 3)[px[sel]]
            assert (cnt.reshape(-1)[px[sel]] == 1).all()
        assert ctx.stats().device_error == 0
    used = np.isin(sm, idx)
    agree = _agreement(got[used], want[used])
    assert agree >= 0.97, f"{name}: only {agree:.4f} of samples agree with the reference"


def test_direct_whole_image_matches_host_build():
    fx = golden.load("direct_spheres")
    scene = scene_from_params(fx["params"])
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).direct_samples(scene.camera, px, np.full_like(px, 5), 4, 4)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=1, first_sample=5, want_image=False, direct=(4, 4), paths_per_wave=3000)
        sums, _, cnt = ctx.film()
        st = ctx.stats()
    assert (cnt == 1).all() and st.device_error == 0
    assert st.extend_rays >= W * H  # camera rays at least
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"only {agree:.4f} of pixels agree"


def test_direct_sample_counts_and_flags():
    scene = rb.generate_scene(rb.RB_SCENE_BOX, seed=0, width=32, height=32)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        default = ctx.render(scene.camera, 4, seed=2, direct=(0, 0))
        explicit = ctx.render(scene.camera, 4, seed=2, direct=(4, 4))
        assert np.array_equal(default, explicit)
        other = ctx.render(scene.camera, 4, seed=2, direct=(1, 2))
        assert not np.array_equal(other, explicit)
        for bad in (dict(direct=(0, 3)), dict(direct=(2, 0)), dict(direct=(4, 4), guide=True),
                    dict(direct=(4, 4), volume=True)):
            with pytest.raises(rb.RbError):
                ctx.render(scene.camera, 1, **bad)


@pytest.mark.parametrize("counts", [(9, 2), (8, 3), (1, 1)])
def test_direct_both_kernels_match_host_build(counts):
    """Up to 8 light samples the staged kernels run, beyond that one thread per
    sample: both against the host build of the same sample."""
    fx = golden.load("direct_fog")
    scene = scene_from_params(fx["params"])
    W, H = scene.camera.width, scene.camera.height
    px = np.arange(W * H, dtype=np.uint32)
    want = HostPaths(scene).direct_samples(scene.camera, px, np.full_like(px, 7), *counts)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=1, first_sample=7, want_image=False, direct=counts, paths_per_wave=1000)
        sums, _, cnt = ctx.film()
        assert ctx.stats().device_error == 0
    assert (cnt == 1).all()
    agree = _agreement(sums.reshape(-1, 3).astype(np.float32), want)
    assert agree >= 0.97, f"{counts}: only {agree:.4f} of pixels agree"


def test_direct_launch_shapes_tuned_and_image_unchanged():
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=2, width=64, height=48, num_spheres=20, subdivision=2)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        want = ctx.render(scene.camera, 3, seed=4, direct=(2, 2))
        t, ms = ctx.tune_render(scene.camera, probe_spp=2, direct=(2, 2))
        assert ms > 0 and t.block_trace in (64, 128, 256)
        got = ctx.render(scene.camera, 3, seed=4, direct=(2, 2))
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
