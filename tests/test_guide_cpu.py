"""CPU checks of the guiding oracle: its analytic gradients against torch
autograd in float64, the normalisation of the guide density, and its sampler
against its density. These pin the oracle the GPU kernels are compared with."""
import numpy as np
import pytest
import torch

from oracle import guide_ref as G


def _random_case(seed, n=48):
    rng = np.random.default_rng(seed)
    params = G.init_params(seed)
    w5, b5 = params[-1]
    w5[:41] = rng.normal(0.0, 0.3, size=w5[:41].shape).astype(np.float32)
    b5[:41] = rng.normal(0.0, 0.5, size=41).astype(np.float32)
    for w, b in params[:-1]:
        b[...] = rng.normal(0.0, 0.1, size=b.shape).astype(np.float32)
    x = rng.random((n, 9))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    weight = rng.random(n) * 3.0
    weight[::7] = 0.0
    p_bsdf = rng.random(n) * 0.5 + 0.01
    return params, x, d, weight, p_bsdf


def _torch_loss(params, x, d, weight, p_bsdf):
    tp = [(torch.tensor(w.astype(np.float64), requires_grad=True), torch.tensor(b.astype(np.float64), requires_grad=True))
          for w, b in params]
    h = torch.tensor(G.encode(x))
    for li, (w, b) in enumerate(tp):
        z = h @ w.T + b
        h = torch.relu(z) if li < len(tp) - 1 else z
    out = h
    n = out.shape[0]
    o = out[:, :40].reshape(n, 8, 5)
    mu = o[:, :, :3] / o[:, :, :3].norm(dim=2, keepdim=True)
    kappa = torch.exp(torch.clamp(o[:, :, 3], G.KAPPA_MIN, G.KAPPA_MAX))
    wt = torch.softmax(o[:, :, 4], dim=1)
    alpha = G.ALPHA_LO + (G.ALPHA_HI - G.ALPHA_LO) * torch.sigmoid(out[:, 40])
    dt = torch.tensor(d)
    c = kappa / (2.0 * np.pi * (-torch.expm1(-2.0 * kappa)))
    comp = c * torch.exp(kappa * ((mu * dt[:, None, :]).sum(2) - 1.0))
    q = (1.0 - G.EPS_UNIFORM) * (wt * comp).sum(1) + G.EPS_UNIFORM / (4.0 * np.pi)
    mix = alpha * q + (1.0 - alpha) * torch.tensor(p_bsdf)
    loss = torch.mean(-torch.tensor(weight) * (torch.log(q) + torch.log(mix)))
    loss.backward()
    return loss.item(), [(w.grad.numpy(), b.grad.numpy()) for w, b in tp]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_gradients_match_autograd(seed):
    params, x, d, weight, p_bsdf = _random_case(seed)
    loss_t, grads_t = _torch_loss(params, x, d, weight, p_bsdf)
    assert G.loss(params, x, d, weight, p_bsdf) == pytest.approx(loss_t, rel=1e-12)
    grads = G.gradients(params, x, d, weight, p_bsdf)
    for (gw, gb), (tw, tb) in zip(grads, grads_t):
        scale = max(np.abs(tw).max(), 1e-12)
        assert np.abs(gw - tw).max() <= 1e-9 * scale
        assert np.abs(gb - tb).max() <= 1e-9 * max(np.abs(tb).max(), 1e-12)


def test_oracle_gradient_finite_difference():
    params, x, d, weight, p_bsdf = _random_case(5, n=16)
    grads = G.gradients(params, x, d, weight, p_bsdf)
    rng = np.random.default_rng(9)
    for li in range(len(params)):
        w, _ = params[li]
        for _ in range(4):
            o = rng.integers(0, 41 if li == 4 else w.shape[0])
            i = rng.integers(0, G.N_ENC if li == 0 else w.shape[1])
            p64 = [(a.astype(np.float64), b.astype(np.float64)) for a, b in params]
            h = 1e-6
            p64[li][0][o, i] += h
            lp = G.loss(p64, x, d, weight, p_bsdf)
            p64[li][0][o, i] -= 2 * h
            lm = G.loss(p64, x, d, weight, p_bsdf)
            fd = (lp - lm) / (2 * h)
            assert fd == pytest.approx(grads[li][0][o, i], rel=1e-4, abs=1e-8)


def test_flat_round_trip_and_size():
    params = G.init_params(3)
    flat = G.to_flat(params)
    assert flat.size == G.NUM_PARAMS == 30000
    back = G.from_flat(flat)
    for (a, b), (c, e) in zip(params, back):
        assert np.array_equal(a, c) and np.array_equal(b, e)


def _sphere_grid(n_theta=400, n_phi=800):
    th = (np.arange(n_theta) + 0.5) * np.pi / n_theta
    ph = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi
    T, P = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], axis=-1).reshape(-1, 3)
    dA = (np.sin(T) * (np.pi / n_theta) * (2 * np.pi / n_phi)).ravel()
    return d, dA


def test_guide_pdf_integrates_to_one():
    params, x, _, _, _ = _random_case(4, n=6)
    out, _ = G.forward(params, x)
    mu, kappa, w, _ = G.decode(out)
    d, dA = _sphere_grid()
    for r in range(x.shape[0]):
        n = d.shape[0]
        pdf = G.guide_pdf(np.repeat(mu[r:r + 1], n, 0), np.repeat(kappa[r:r + 1], n, 0), np.repeat(w[r:r + 1], n, 0), d)
        assert (pdf * dA).sum() == pytest.approx(1.0, abs=2e-3)


def test_sampler_matches_density():
    """Histogram of sample_guide over a coarse (cos theta, phi) grid against the
    density integrated over the same cells."""
    rng = np.random.default_rng(11)
    mu = np.array([[[0.0, 0.0, 1.0], [0.6, 0.0, 0.8], [0.0, -1.0, 0.0]] + [[1.0, 0.0, 0.0]] * 5])
    kappa = np.array([[20.0, 5.0, 1.0, 0.5, 0.5, 0.5, 0.5, 0.5]])
    w = np.array([[0.3, 0.3, 0.2, 0.04, 0.04, 0.04, 0.04, 0.04]])
    n = 200000
    u = rng.random((n, 3))
    dirs = G.sample_guide(np.repeat(mu, n, 0), np.repeat(kappa, n, 0), np.repeat(w, n, 0), u[:, 0], u[:, 1], u[:, 2])
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1.0, atol=1e-9)
    nz, nphi = 16, 16
    iz = np.minimum(((dirs[:, 2] + 1) / 2 * nz).astype(int), nz - 1)
    ip = np.minimum(((np.arctan2(dirs[:, 1], dirs[:, 0]) % (2 * np.pi)) / (2 * np.pi) * nphi).astype(int), nphi - 1)
    hist = np.bincount(iz * nphi + ip, minlength=nz * nphi) / n
    d, dA = _sphere_grid(800, 1600)
    pdf = G.guide_pdf(np.repeat(mu, d.shape[0], 0), np.repeat(kappa, d.shape[0], 0), np.repeat(w, d.shape[0], 0), d)
    jz = np.minimum(((d[:, 2] + 1) / 2 * nz).astype(int), nz - 1)
    jp = np.minimum(((np.arctan2(d[:, 1], d[:, 0]) % (2 * np.pi)) / (2 * np.pi) * nphi).astype(int), nphi - 1)
    expect = np.bincount(jz * nphi + jp, weights=pdf * dA, minlength=nz * nphi)
    sigma = np.sqrt(expect * (1 - expect) / n) + 1e-6
    assert np.max(np.abs(hist - expect) / sigma) < 6.0


def test_onb_is_orthonormal():
    rng = np.random.default_rng(2)
    n = rng.normal(size=(1000, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n[0] = [0, 0, -1]
    n[1] = [0, 0, 1]
    t, b = G.onb(n)
    for a, c in ((t, b), (t, n), (b, n)):
        assert np.abs((a * c).sum(1)).max() < 1e-12
    assert np.allclose(np.linalg.norm(t, axis=1), 1) and np.allclose(np.linalg.norm(b, axis=1), 1)


def test_training_weight():
    L_final = np.array([[1.0, 2.0, 3.0]])
    L_before = np.array([[0.5, 1.0, 3.0]])
    beta = np.array([[0.5, 0.0, 1.0]])
    assert G.training_weight(L_final, L_before, beta)[0] == pytest.approx(0.2126 * 1.0)
