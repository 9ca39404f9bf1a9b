"""GPU tests of the learned path guide: the tcgen05 forward pass, gradients and
Adam step against the FP64 oracle (oracle/guide_ref.py), the device sampler,
and guided rendering (unbiased against plain path tracing, identical to it
while the guide is untrained, and better than it once trained)."""
import numpy as np
import pytest

import rainbow_b200 as rb
from oracle import guide_ref as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = rb.Context(0)
    c.guide_init(seed=1)
    yield c
    c.close()


def _params(seed):
    rng = np.random.default_rng(seed)
    params = G.init_params(seed)
    w5, b5 = params[-1]
    w5[:41] = rng.normal(0.0, 0.15, size=w5[:41].shape).astype(np.float32)
    b5[:41] = rng.normal(0.0, 0.5, size=41).astype(np.float32)
    for w, b in params[:-1]:
        b[...] = rng.normal(0.0, 0.05, size=b.shape).astype(np.float32)
    return params


def _samples(seed, n):
    rng = np.random.default_rng(seed)
    s = np.zeros(n, dtype=rb.GUIDE_SAMPLE_DTYPE)
    s["inputs"] = rng.random((n, 9))
    d = rng.normal(size=(n, 3))
    s["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    s["bsdf_pdf"] = rng.random(n) * 0.5 + 0.02
    w = rng.random(n) * 2.0
    w[rng.random(n) < 0.2] = 0.0
    s["weight"] = w
    return s


def test_forward_matches_oracle(ctx):
    params = _params(3)
    ctx.guide_set_params(G.to_flat(params))
    x = np.random.default_rng(4).random((1000, 9)).astype(np.float32)  # 7 full tiles and a ragged one
    out = ctx.guide_forward(x)
    ref, _ = G.forward(params, x.astype(np.float64), emulate_bf16=True)
    scale = np.abs(ref[:, :41]).max()
    err = np.abs(out[:, :41] - ref[:, :41])
    assert np.isfinite(out).all()
    assert err.max() <= 2e-2 * scale, err.max()
    assert err.mean() <= 1e-3 * scale, err.mean()
    # the unused outputs stay at zero weights -> zero
    assert np.abs(out[:, 41:]).max() == 0.0


def test_forward_empty_and_single_row(ctx):
    params = _params(5)
    ctx.guide_set_params(G.to_flat(params))
    assert ctx.guide_forward(np.zeros((0, 9), np.float32)).shape == (0, 48)
    x = np.full((1, 9), 0.25, np.float32)
    ref, _ = G.forward(params, x.astype(np.float64), emulate_bf16=True)
    out = ctx.guide_forward(x)
    assert np.abs(out[0, :41] - ref[0, :41]).max() <= 2e-2 * np.abs(ref[0, :41]).max()


def test_gradient_matches_oracle(ctx):
    params = _params(6)
    ctx.guide_set_params(G.to_flat(params))
    s = _samples(7, 1100)
    grad, loss = ctx.guide_train(s, steps=1, sequential=True)
    x = s["inputs"].astype(np.float64)
    d = s["direction"].astype(np.float64)
    ref = G.gradients(params, x, d, s["weight"].astype(np.float64), s["bsdf_pdf"].astype(np.float64), emulate_bf16=True)
    ref_loss = G.loss(params, x, d, s["weight"].astype(np.float64), s["bsdf_pdf"].astype(np.float64), emulate_bf16=True)
    assert loss == pytest.approx(ref_loss, rel=2e-3)
    flat_ref = G.to_flat([(gw.astype(np.float32), gb.astype(np.float32)) for gw, gb in ref]).astype(np.float64)
    for li, (fi, fo) in enumerate(G.LAYERS):
        o0 = sum(i * o + o for i, o in G.LAYERS[:li])
        a = grad[o0:o0 + fi * fo + fo].astype(np.float64)
        b = flat_ref[o0:o0 + fi * fo + fo]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel < 2e-2 and cos > 0.9998, (li, rel, cos)


def test_adam_step_matches_oracle(ctx):
    params = _params(8)
    ctx.guide_set_params(G.to_flat(params))
    s = _samples(9, 512)
    m = [(np.zeros_like(w), np.zeros_like(b)) for w, b in params]
    v = [(np.zeros_like(w), np.zeros_like(b)) for w, b in params]
    ref = [(w.copy(), b.copy()) for w, b in params]
    for t in (1, 2):
        grad, _ = ctx.guide_train(s, steps=1, sequential=True)
        G.adam_step(ref, G.from_flat(grad), m, v, t, lr=1e-3)
        got = ctx.guide_params()
        want = G.to_flat(ref)
        ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
        assert ulp.max() <= 1, (t, ulp.max())


def test_sampler_matches_oracle(ctx):
    rng = np.random.default_rng(10)
    n = 4096
    raw = rng.normal(0.0, 1.0, size=(n, 48)).astype(np.float32)
    raw[:, 3:40:5] = rng.uniform(-5, 7, size=(n, 8))  # log-kappa over and beyond the clamp range
    u = rng.random((n, 3)).astype(np.float32)
    d, pdf = ctx.guide_sample(raw, u)
    mu, kappa, w, _ = G.decode(raw.astype(np.float64))
    dref = G.sample_guide(mu, kappa, w, u[:, 0].astype(np.float64), u[:, 1].astype(np.float64), u[:, 2].astype(np.float64))
    pref = G.guide_pdf(mu, kappa, w, dref)
    # rows whose lobe pick sits within float rounding of a boundary may pick a neighbour
    up = (u[:, 0] - G.EPS_UNIFORM) / (1 - G.EPS_UNIFORM)
    cdf = np.cumsum(w, axis=1)
    near = (np.abs(cdf - up[:, None]) < 1e-5).any(axis=1) | (np.abs(u[:, 0] - G.EPS_UNIFORM) < 1e-6)
    ok = ~near
    assert ok.sum() > 0.99 * n
    assert np.abs(np.linalg.norm(d, axis=1) - 1).max() < 1e-4
    derr = np.linalg.norm(d[ok] - dref[ok], axis=1)
    assert np.quantile(derr, 0.999) < 2e-3, np.quantile(derr, 0.999)
    rel = np.abs(pdf[ok] - pref[ok]) / pref[ok]
    assert np.quantile(rel, 0.99) < 1e-2, np.quantile(rel, 0.99)


def test_training_learns_a_direction_field(ctx):
    """Samples whose directions cluster around a position-dependent axis: the
    loss falls and the guide density at the axis rises well above uniform."""
    ctx.guide_init(seed=2, batch_size=8192, min_rows=1024)
    rng = np.random.default_rng(12)
    n = 65536
    x = rng.random((n, 9)).astype(np.float32)
    axis = np.stack([np.cos(2 * np.pi * x[:, 0]), np.sin(2 * np.pi * x[:, 0]), np.zeros(n)], axis=1)
    mu = np.repeat(axis[:, None, :], 8, axis=1)
    kap = np.full((n, 8), 30.0)
    wts = np.full((n, 8), 1 / 8.0)
    d = G.sample_guide(mu, kap, wts, np.ones(n), rng.random(n), rng.random(n))
    s = np.zeros(n, dtype=rb.GUIDE_SAMPLE_DTYPE)
    s["inputs"] = x
    s["direction"] = d
    s["bsdf_pdf"] = 1.0 / (4 * np.pi)
    s["weight"] = 1.0
    _, loss0 = ctx.guide_train(s, steps=1)
    _, loss1 = ctx.guide_train(s, steps=400)
    assert loss1 < loss0 - 2.0, (loss0, loss1)
    out = ctx.guide_forward(x[:512])
    mu_g, k_g, w_g, _ = G.decode(out.astype(np.float64))
    q = G.guide_pdf(mu_g, k_g, w_g, axis[:512])
    assert np.median(q) > 10 * (1 / (4 * np.pi)), np.median(q)
    st = ctx.guide_stats()
    assert st.steps == 401 and st.device_error == 0


def _slit(res, clutter=12):
    return rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=res, height=res, num_spheres=clutter, subdivision=2)


def test_untrained_guide_renders_plain_bits(ctx):
    scene = _slit(48)
    ctx.upload(scene)
    ctx.guide_init(seed=0)
    plain = ctx.render(scene.camera, 8, max_depth=6, seed=5)
    guided = ctx.render(scene.camera, 8, max_depth=6, seed=5, guide=True)
    assert np.array_equal(plain, guided)


def _film_mean_var(ctx):
    s, sq, c = ctx.film()
    m = s / c[..., None]
    return m, np.maximum(sq / c[..., None] - m ** 2, 0) / c[..., None]


def test_guided_render_is_unbiased(ctx):
    """Online-trained guided render against a converged plain render. Per-pixel
    z-scores of path-traced images are skewed by heavy tails at any spp, so the
    check is on 4 x 4 pixel blocks and on the image mean."""
    res, B = 32, 4
    scene = _slit(res)
    ctx.upload(scene)
    ctx.render(scene.camera, 65536, max_depth=6, seed=100)
    ref, ref_var = _film_mean_var(ctx)
    ctx.guide_init(seed=0, batch_size=16384, min_rows=1024, steps_per_wave=4)
    ctx.render(scene.camera, 2048, max_depth=6, seed=7, guide=True, train=True, paths_per_wave=res * res * 64)
    assert ctx.guide_stats().steps >= 64
    ctx.render(scene.camera, 8192, max_depth=6, seed=9, guide=True)
    m, var = _film_mean_var(ctx)
    blk = lambda a: a.reshape(res // B, B, res // B, B, 3).mean((1, 3))
    zb = (blk(m) - blk(ref)) / np.sqrt((var + ref_var).reshape(res // B, B, res // B, B, 3).sum((1, 3)) / B ** 4 + 1e-12)
    # the block variances are sample variances of a heavy-tailed estimator (rare
    # bright paths through the slit), so the block z-scores lean negative and their
    # mean varies from run to run with the training order (-0.45 seen in one of many
    # runs whose image mean agreed within 0.5%); the image-mean ratio below is the
    # tight check of unbiasedness
    assert abs(zb.mean()) < 0.6, zb.mean()
    assert np.mean(np.abs(zb) > 4) < 0.02, np.mean(np.abs(zb) > 4)
    assert abs(m.mean() / ref.mean() - 1) < 0.005, m.mean() / ref.mean()


def test_trained_guide_reduces_error(ctx):
    """What the network gains: after online training on the slit room, guided
    path tracing at equal spp has clearly lower relMSE than plain BSDF sampling
    (both against a converged plain render)."""
    res, depth = 64, 8
    scene = rb.generate_scene(rb.RB_SCENE_SLIT_ROOM, seed=3, width=res, height=res, num_spheres=60, subdivision=3)
    ctx.upload(scene)
    ctx.render(scene.camera, 32768, max_depth=depth, seed=100)
    ref, _ = _film_mean_var(ctx)
    relmse = lambda m: np.mean((m - ref) ** 2 / (ref ** 2 + 1e-2))
    plain = [relmse(ctx.render(scene.camera, 256, max_depth=depth, seed=s)) for s in (7, 8)]
    ctx.guide_init(seed=0, batch_size=1 << 16, min_rows=1024, steps_per_wave=8)
    ctx.render(scene.camera, 1024, max_depth=depth, seed=11, guide=True, train=True, paths_per_wave=res * res * 32)
    guided = [relmse(ctx.render(scene.camera, 256, max_depth=depth, seed=s, guide=True)) for s in (7, 8)]
    assert np.mean(guided) < 0.8 * np.mean(plain), (guided, plain)


def test_guided_lanes_unbiased_and_plain_before_training():
    """Guided rendering on wave lanes (each lane samples a snapshot of the
    weights taken after its previous wave trained): identical to plain before
    any training, unbiased after online training on lanes."""
    res, B = 32, 4
    scene = _slit(res)
    with rb.Context(0) as c:
        c.upload(scene)
        c.set_tuning(lanes=3, paths_per_wave=res * res * 4)
        c.guide_init(seed=0)
        plain = c.render(scene.camera, 16, max_depth=6, seed=5)
        assert np.array_equal(plain, c.render(scene.camera, 16, max_depth=6, seed=5, guide=True))
        c.render(scene.camera, 65536, max_depth=6, seed=100, want_image=False)
        ref, ref_var = _film_mean_var(c)
        c.guide_init(seed=0, batch_size=16384, min_rows=1024, steps_per_wave=4)
        c.set_tuning(lanes=2, paths_per_wave=res * res * 64)
        c.render(scene.camera, 2048, max_depth=6, seed=7, guide=True, train=True, want_image=False)
        assert c.guide_stats().steps >= 64 and c.guide_stats().device_error == 0
        c.render(scene.camera, 8192, max_depth=6, seed=9, guide=True, want_image=False)
        m, var = _film_mean_var(c)
    blk = lambda a: a.reshape(res // B, B, res // B, B, 3).mean((1, 3))
    zb = (blk(m) - blk(ref)) / np.sqrt((var + ref_var).reshape(res // B, B, res // B, B, 3).sum((1, 3)) / B ** 4 + 1e-12)
    # the block variances are sample variances of a heavy-tailed estimator (rare
    # bright paths through the slit), so the block z-scores lean negative and their
    # mean varies from run to run with the training order (-0.45 seen in one of many
    # runs whose image mean agreed within 0.5%); the image-mean ratio below is the
    # tight check of unbiasedness
    assert abs(zb.mean()) < 0.6, zb.mean()
    assert np.mean(np.abs(zb) > 4) < 0.02, np.mean(np.abs(zb) > 4)
    assert abs(m.mean() / ref.mean() - 1) < 0.005, m.mean() / ref.mean()
