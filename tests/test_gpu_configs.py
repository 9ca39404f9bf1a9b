"""Parity on the benchmark configurations themselves, against the reference
renderer compiled as the oracle (fixtures from tests/golden/make_golden.py):

- configuration 1 as specified (box room, 256 x 256, 16 spp, depth 5): pixel
  and block means within 3 sigma of the reference's 512-spp render;
- configuration 2's 1,024,010-triangle sphere field: 2^19 seeded camera rays
  and two generations of bounce rays, closest hits bit-equal to
  scene::intersect (entity, triangle and the bits of t for every ray);
- configuration 4's slit room and configuration 5's fog (8,192,046 triangles,
  volume_path_integrator) at reduced resolution: per-sample radiance with the
  reference's random-number order, the disagreeing few without bias, and image
  means within 3 sigma;
- relMSE of plain renders against a converged 8192-spp reference: it falls as
  1 / spp and matches the variance the render itself predicts (no bias).
"""
import numpy as np
import pytest

import rainbow_b200 as rb
from tests import golden
from tests.helpers import (assert_disagreements_unbiased, assert_hits_equal, block_z, hit_digests,
                           per_sample_radiance, ray_levels, sample_agreement, scene_from_params)

pytestmark = pytest.mark.gpu


def _render_mean_var(scene, spp, depth, seed, volume=False):
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        ctx.render(scene.camera, spp=spp, max_depth=depth, seed=seed, volume=volume, want_image=False)
        sums, sq, cnt = ctx.film()
        assert ctx.stats().device_error == 0
    assert (cnt == spp).all()
    mean = sums / spp
    return mean, np.maximum(sq / spp - mean ** 2, 0.0)


def test_config1_as_specified_within_three_sigma():
    fx = golden.load("config1_image")
    scene = scene_from_params(fx["params"])
    assert (scene.camera.width, scene.camera.height) == (256, 256) and scene.num_triangles == 32
    n_ref, depth = int(fx["spp"]), int(fx["max_depth"])
    ref_mean, ref_var = fx["mean"].astype(np.float64), fx["var"].astype(np.float64)
    # the configuration's own frame: 16 spp, compared on 4 x 4 pixel blocks
    mean, var = _render_mean_var(scene, 16, depth, seed=1)
    z = block_z(mean, ref_mean, ref_var, 16, n_ref, var=var)
    assert (np.abs(z) > 3).mean() < 0.01, f"{(np.abs(z) > 3).mean():.4f} of 16-spp block channels outside 3 sigma"
    assert abs(z.mean()) < 0.1, z.mean()
    # and per pixel at 256 spp
    mean, _ = _render_mean_var(scene, 256, depth, seed=2)
    se = np.sqrt(ref_var * (1.0 / 256 + 1.0 / n_ref))
    z = np.where(se > 0, (mean - ref_mean) / np.where(se > 0, se, 1), 0.0)
    assert (np.abs(z) > 3).mean() < 0.01, f"{(np.abs(z) > 3).mean():.4f} of pixel channels outside 3 sigma"
    assert abs(z.mean()) < 0.1, z.mean()


def test_config2_ray_levels_bit_equal_to_reference():
    fx = golden.load("c2_ray_levels")
    scene = scene_from_params(fx["params"])
    assert scene.num_triangles == 1024010
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        levels = ray_levels(scene.camera, ctx.trace_closest, int(fx["n0"]), int(fx["seed"]))
    total = 0
    for k, (rays, hits) in enumerate(levels):
        assert rays.shape[0] == int(fx[f"count{k}"]), f"level {k}: ray count differs (an earlier level's hits differ)"
        total += rays.shape[0]
        assert_hits_equal(hits[:4096], fx[f"head{k}"], f"level {k} head")
        assert int((hits["entity"] >= 0).sum()) == int(fx[f"hit_count{k}"])
        d = hit_digests(hits)
        bad = np.flatnonzero(d != fx[f"digests{k}"])
        assert bad.size == 0, f"level {k}: hits differ in chunks of 4096 rays starting at {bad[:8] * 4096}"
    assert total >= 1 << 20, total


@pytest.mark.parametrize("name,volume,min_agree", [("slit_samples", False, 0.97), ("fog5_samples", True, 0.9)])
def test_large_config_samples_match_reference(name, volume, min_agree):
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    depth = int(fx["max_depth"])
    px, sm, want = fx["pixels"], fx["samples"], fx["radiance"]
    with rb.Context(0) as ctx:
        ctx.upload(scene)
        got = per_sample_radiance(ctx, scene, px, sm, depth, volume=volume)
        assert ctx.stats().device_error == 0
    agree = sample_agreement(got, want).mean()
    # volume samples draw several log / exp / sin / cos per medium vertex, where
    # CUDA and glibc may round differently and a path then diverges
    assert agree >= min_agree, f"{name}: only {agree:.4f} of samples agree with the reference"
    assert_disagreements_unbiased(scene, got, want, fx["first_entity"], name)


@pytest.mark.parametrize("name,volume", [("slit_image", False), ("fog5_image", True)])
def test_large_config_images_within_three_sigma(name, volume):
    fx = golden.load(name)
    scene = scene_from_params(fx["params"])
    n_ref, depth = int(fx["spp"]), int(fx["max_depth"])
    n = 4096
    mean, var = _render_mean_var(scene, n, depth, seed=3, volume=volume)
    # heavy-tailed paths (the slit, scattering in the fog) leave per-pixel
    # variance estimates low, so the check is on 4 x 4 blocks, with each
    # render's own variance, plus the mean z
    z = block_z(mean, fx["mean"].astype(np.float64), fx["var"].astype(np.float64), n, n_ref, var=var)
    assert (np.abs(z) > 3).mean() < 0.02, f"{name}: {(np.abs(z) > 3).mean():.4f} of block channels outside 3 sigma"
    assert abs(z.mean()) < 0.15, z.mean()


def test_plain_relmse_against_converged_reference():
    """relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 1e-2), R the
    reference's 8192-spp FP64 render. An unbiased render's expected relMSE is
    the mean of (var / n + var / 8192) / (R^2 + 1e-2); the measured value must
    match it and fall as 1 / n."""
    fx = golden.load("box_converged")
    scene = scene_from_params(fx["params"])
    R, n_ref, depth = fx["mean"], int(fx["spp"]), int(fx["max_depth"])
    den = R ** 2 + 1e-2
    out = {}
    for n, seed in ((64, 11), (1024, 12)):
        mean, var = _render_mean_var(scene, n, depth, seed)
        rel = float(np.mean((mean - R) ** 2 / den))
        expected = float(np.mean(var * (1.0 / n + 1.0 / n_ref) / den))
        assert 0.6 < rel / expected < 1.6, f"{n} spp: relMSE {rel:.3g}, expected {expected:.3g} from the variance"
        out[n] = rel
    assert out[1024] < out[64] / 8, out
