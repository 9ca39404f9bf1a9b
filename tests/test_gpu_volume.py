"""Volume path tracing (RB_RENDER_VOLUME) against the reference's
volume_path_integrator: per-sample radiance with the reference's random-number
order, per-pixel means of an independent render, bit-identity with plain
path tracing on a scene without media, and guided volume rendering (surface
and medium guides): plain bits before training, unbiased after it."""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.helpers import assert_disagreements_unbiased, per_sample_radiance, scene_from_params

pytestmark = pytest.mark.gpu

SAMPLE_RTOL = 1e-3


def test_volume_samples_match_reference():
    fx = golden.load("fog_samples")
    scene = scene_from_params(fx["params"])
    depth = int(fx["max_depth"])
    px, sm, want = fx["pixels"], fx["samples"], fx["radiance"]
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, px, sm, depth, volume=True)
        assert ctx.stats().device_error == 0
    ok = np.abs(got - want) <= SAMPLE_RTOL * np.maximum(1.0, np.abs(want))
    agree = ok.all(axis=1).mean()
    # samples that scatter in the medium draw several log / exp / sin / cos per
    # vertex, where CUDA and glibc may round differently and a path then diverges
    assert agree >= 0.9, f"only {agree:.4f} of volume samples agree with the reference"
    assert_disagreements_unbiased(scene, got, want, fx["first_entity"], "fog")


def test_volume_image_means_within_three_sigma():
    fx = golden.load("fog_image")
    scene = scene_from_params(fx["params"])
    n, depth = int(fx["spp"]), int(fx["max_depth"])
    ref_mean = fx["sum"] / n
    ref_var = np.maximum(fx["sum_sq"] / n - ref_mean ** 2, 0.0) / n
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        m = 4096
        ctx.render(scene.camera, spp=m, max_depth=depth, seed=3, volume=True, want_image=False)
        sums, sq, cnt = ctx.film()
        assert ctx.stats().device_error == 0
    assert (cnt == m).all()
    mean = sums / m
    var = np.maximum(sq / m - mean ** 2, 0.0) / m
    # Per-pixel z-scores of path-traced images are skewed by heavy tails (rare
    # bright paths leave the 256-spp reference's variance estimate low), so the
    # check is on 4 x 4 pixel blocks, plus the image mean.
    B, r = 4, mean.shape[0]
    blk = lambda a: a.reshape(r // B, B, r // B, B, 3).sum((1, 3)) / B ** 2
    blk_var = lambda v: v.reshape(r // B, B, r // B, B, 3).sum((1, 3)) / B ** 4
    zb = (blk(mean) - blk(ref_mean)) / np.sqrt(blk_var(var + ref_var) + 1e-30)
    ratio = mean.mean() / ref_mean.mean()
    stats = dict(block_out_3sigma=float((np.abs(zb) > 3).mean()), block_z_mean=float(zb.mean()), mean_ratio=float(ratio))
    assert stats["block_out_3sigma"] < 0.05, stats
    assert abs(stats["block_z_mean"]) < 0.5, stats
    assert abs(ratio - 1) < 0.02, stats


def test_volume_without_media_equals_plain():
    """volume_path_integrator on a scene without media draws the same random
    numbers and computes the same products as path_integrator."""
    fx = golden.load("spheres_samples")
    scene = scene_from_params(fx["params"])
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        plain = ctx.render(scene.camera, 4, max_depth=8, seed=2)
        vol = ctx.render(scene.camera, 4, max_depth=8, seed=2, volume=True)
        plain2 = ctx.render(scene.camera, 4, max_depth=8, seed=2)
    assert np.array_equal(plain, vol)
    assert np.array_equal(plain, plain2)


def _fog(res):
    return rb.generate_scene(rb.RB_SCENE_FOG, seed=4, width=res, height=res, num_spheres=12, subdivision=2)


def _mean_var(ctx):
    s, sq, c = ctx.film()
    m = s / c[..., None]
    return m, np.maximum(sq / c[..., None] - m ** 2, 0) / c[..., None]


@pytest.mark.parametrize("lanes", [1, 3])
def test_untrained_volume_guides_render_plain_bits(lanes):
    """Guided volume rendering before any training step samples the BSDF and
    the phase function with plain volume path tracing's random numbers (on
    one lane, and on three lanes of four waves)."""
    scene = _fog(24)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.set_tuning(lanes=lanes, paths_per_wave=24 * 24 * 2)
        ctx.guide_init(seed=0)
        plain = ctx.render(scene.camera, 8, max_depth=8, seed=5, volume=True)
        guided = ctx.render(scene.camera, 8, max_depth=8, seed=5, volume=True, guide=True)
        assert np.array_equal(plain, guided)


@pytest.mark.parametrize("lanes", [1, 3])
def test_guided_volume_render_is_unbiased(lanes):
    """Surface and medium guides trained online on the fog scene, then a guided
    volume render against a converged plain volume render: 4 x 4 block z-scores
    and the image mean (one-sample MIS keeps the estimator unbiased). On three
    lanes each wave samples both guides' weight snapshots of its lane."""
    res, B, depth = 32, 4, 8
    scene = _fog(res)
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.set_tuning(lanes=lanes)
        ctx.render(scene.camera, 16384, max_depth=depth, seed=100, volume=True, want_image=False)
        ref, ref_var = _mean_var(ctx)
        ctx.guide_init(seed=0, batch_size=16384, min_rows=1024, steps_per_wave=4)
        ctx.render(scene.camera, 1024, max_depth=depth, seed=7, volume=True, guide=True, train=True,
                   paths_per_wave=res * res * 64, want_image=False)
        ms = ctx.guide_medium_stats()
        assert ms.steps >= 32 and ms.device_error == 0 and ctx.guide_stats().steps >= 32
        ctx.render(scene.camera, 4096, max_depth=depth, seed=9, volume=True, guide=True, want_image=False)
        m, var = _mean_var(ctx)
    blk = lambda a: a.reshape(res // B, B, res // B, B, 3).mean((1, 3))
    zb = (blk(m) - blk(ref)) / np.sqrt((var + ref_var).reshape(res // B, B, res // B, B, 3).sum((1, 3)) / B ** 4 + 1e-12)
    # the block variances are sample variances of a heavy-tailed estimator (rare
    # bright paths through the slit), so the block z-scores lean negative and their
    # mean varies from run to run with the training order (-0.45 seen in one of many
    # runs whose image mean agreed within 0.5%); the image-mean ratio below is the
    # tight check of unbiasedness
    assert abs(zb.mean()) < 0.6, zb.mean()
    assert np.mean(np.abs(zb) > 4) < 0.02, np.mean(np.abs(zb) > 4)
    assert abs(m.mean() / ref.mean() - 1) < 0.01, m.mean() / ref.mean()
