"""FP64 CPU restatement of the guiding network (TEST INFRASTRUCTURE ONLY).

The reference renderer has no learned sampling, so there is no reference code
to follow here: this module is the project's own definition of the guide,
written once in numpy so that the GPU kernels' forward pass, gradients, Adam
step and vMF sampler can be checked against it. It is pinned against torch
autograd in float64 by the CPU tests.

Network: 9 inputs in [0, 1] (position normalised to the scene box, shading
normal and outgoing direction mapped from [-1, 1]) -> frequency encoding
sin(2^k pi v), cos(2^k pi v) for k = 0..11 (216 features, zero-padded to 224)
-> 4 hidden ReLU layers of width 64 -> 48 outputs. Outputs 0..39 are 8 von
Mises-Fisher lobes of 5 values each (mean direction 3, log-concentration 1,
weight logit 1), output 40 is the guide-vs-BSDF mixing logit, 41..47 are
unused. Weights are W[out][in] with a bias per output (30,000 parameters in
the flat order W1 b1 W2 b2 ... W5 b5).

Guide density: q(d) = (1 - EPS) * sum_i w_i vMF(d; mu_i, kappa_i) + EPS / (4 pi).
The uniform share keeps q > 0 everywhere, which bounds the loss gradient.
One-sample MIS with the BSDF: p(d) = alpha q(d) + (1 - alpha) p_bsdf(d).
"""
from __future__ import annotations

import numpy as np

N_IN = 9
N_FREQ = 12
N_ENC = N_IN * N_FREQ * 2  # 216
K1 = 224
HID = 64
N_OUT = 48
N_LOBES = 8
LAYERS = [(K1, HID), (HID, HID), (HID, HID), (HID, HID), (HID, N_OUT)]
NUM_PARAMS = sum(i * o + o for i, o in LAYERS)  # 30000
KAPPA_MIN, KAPPA_MAX = -4.0, 8.0  # clamp of the log-concentration
ALPHA_LO, ALPHA_HI = 0.1, 0.9      # range of the guide selection probability
EPS_UNIFORM = 0.02                 # share of the uniform sphere density in q
NORM_FLOOR = 1e-6                  # |m| floor in the mean-direction gradient
LUMINANCE = np.array([0.2126, 0.7152, 0.0722])


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even) and back to float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + ((u >> 16) & 1) + 0x7FFF) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def encode(x):
    """x: (n, 9) -> (n, 224); feature 24 j + 2 k + s is sin (s = 0) or cos (s = 1) of 2^k pi x_j."""
    x = np.asarray(x, dtype=np.float64)
    f = np.zeros((x.shape[0], K1), dtype=np.float64)
    for j in range(N_IN):
        for k in range(N_FREQ):
            a = np.pi * (2.0 ** k) * x[:, j]
            f[:, 24 * j + 2 * k] = np.sin(a)
            f[:, 24 * j + 2 * k + 1] = np.cos(a)
    return f


def init_params(seed=0):
    """He-uniform weights with zero biases; the output layer is scaled by 0.1
    so that the untrained guide is close to a uniform mixture."""
    rng = np.random.default_rng(seed)
    params = []
    for fan_in, fan_out in LAYERS:
        fan = N_ENC if fan_in == K1 else fan_in
        lim = np.sqrt(6.0 / fan)
        w = rng.uniform(-lim, lim, size=(fan_out, fan_in)).astype(np.float32)
        if fan_in == K1:
            w[:, N_ENC:] = 0.0
        params.append((w, np.zeros(fan_out, dtype=np.float32)))
    params[-1][0][...] *= np.float32(0.1)
    params[-1][0][41:] = 0.0
    return params


def to_flat(params):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in params]).astype(np.float32)


def from_flat(vec):
    vec = np.asarray(vec, dtype=np.float32)
    params, o = [], 0
    for fan_in, fan_out in LAYERS:
        w = vec[o:o + fan_in * fan_out].reshape(fan_out, fan_in).copy()
        o += fan_in * fan_out
        b = vec[o:o + fan_out].copy()
        o += fan_out
        params.append((w, b))
    return params


def forward(params, x, emulate_bf16=False):
    """Raw outputs (n, 48) and the list of layer inputs. With emulate_bf16 the
    weights, biases, features and hidden activations are rounded to bfloat16 as
    the tensor-core kernels store them (accumulation stays exact here)."""
    r = (lambda a: bf16(a).astype(np.float64)) if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    h = r(encode(x))
    cache = [h]
    for li, (w, b) in enumerate(params):
        z = h @ r(w).T + r(b)
        if li < len(params) - 1:
            h = r(np.maximum(z, 0.0))
            cache.append(h)
        else:
            h = z
    return h, cache


def decode(out):
    """Raw outputs -> (mu (n, 8, 3), kappa (n, 8), weights (n, 8), alpha (n,))."""
    o = out[:, :40].reshape(-1, N_LOBES, 5)
    m = o[:, :, :3]
    norm = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(norm > 1e-12, m / np.maximum(norm, 1e-30), np.array([0.0, 0.0, 1.0]))
    kappa = np.exp(np.clip(o[:, :, 3], KAPPA_MIN, KAPPA_MAX))
    logits = o[:, :, 4]
    e = np.exp(logits - logits.max(axis=1, keepdims=True))
    w = e / e.sum(axis=1, keepdims=True)
    alpha = ALPHA_LO + (ALPHA_HI - ALPHA_LO) / (1.0 + np.exp(-out[:, 40]))
    return mu, kappa, w, alpha


def vmf_norm(kappa):
    """vMF normalisation kappa / (2 pi (1 - exp(-2 kappa))), with the density written as c exp(kappa (mu.d - 1))."""
    return kappa / (2.0 * np.pi * (-np.expm1(-2.0 * kappa)))


def guide_pdf(mu, kappa, w, d):
    """Guide density q of unit directions d (n, 3)."""
    dots = np.einsum("nkc,nc->nk", mu, d)
    mix = (w * vmf_norm(kappa) * np.exp(kappa * (dots - 1.0))).sum(axis=1)
    return (1.0 - EPS_UNIFORM) * mix + EPS_UNIFORM / (4.0 * np.pi)


def onb(n):
    """Orthonormal basis (t, b) around unit n (Duff et al. 2017, 'Building an
    Orthonormal Basis, Revisited')."""
    sign = np.where(n[..., 2] >= 0.0, 1.0, -1.0)
    a = -1.0 / (sign + n[..., 2])
    b = n[..., 0] * n[..., 1] * a
    t = np.stack([1.0 + sign * n[..., 0] ** 2 * a, sign * b, -sign * n[..., 0]], axis=-1)
    bb = np.stack([b, sign + n[..., 1] ** 2 * a, -n[..., 1]], axis=-1)
    return t, bb


def sample_guide(mu, kappa, w, u_pick, u1, u2):
    """Direction from q: u_pick < EPS picks the uniform sphere (z = 1 - 2 u1,
    phi = 2 pi u2); otherwise (u_pick - EPS) / (1 - EPS) picks a lobe by its
    cumulative weight and (u1, u2) sample it with the numerically stable
    inversion of Jakob (2012, 'Numerically stable sampling of the von
    Mises-Fisher distribution on S^2'): w = 1 + log(u1 + (1 - u1) e^{-2 kappa}) / kappa."""
    n = mu.shape[0]
    out = np.zeros((n, 3))
    for r in range(n):
        if u_pick[r] < EPS_UNIFORM:
            z = 1.0 - 2.0 * u1[r]
            s = np.sqrt(max(0.0, 1.0 - z * z))
            ph = 2.0 * np.pi * u2[r]
            out[r] = [s * np.cos(ph), s * np.sin(ph), z]
            continue
        up = (u_pick[r] - EPS_UNIFORM) / (1.0 - EPS_UNIFORM)
        cdf = np.cumsum(w[r])
        j = int(np.searchsorted(cdf, up * cdf[-1], side="right"))
        j = min(j, N_LOBES - 1)
        k = kappa[r, j]
        e2 = np.exp(-2.0 * k)
        cz = 1.0 + np.log(e2 + u1[r] * (1.0 - e2)) / k
        cz = min(1.0, max(-1.0, cz))
        s = np.sqrt(max(0.0, 1.0 - cz * cz))
        ph = 2.0 * np.pi * u2[r]
        t, b = onb(mu[r, j])
        out[r] = cz * mu[r, j] + s * (np.cos(ph) * t + np.sin(ph) * b)
    return out


def loss(params, x, d, weight, p_bsdf, emulate_bf16=False):
    """Importance-weighted cross entropy of the guide and of the one-sample MIS
    mixture, averaged over the batch:
        L = -mean( weight * (log q(d) + log(alpha q(d) + (1 - alpha) p_bsdf(d))) )
    where weight = F(d) / p_sample(d) for the integrand F = luminance(f cos L_i)."""
    out, _ = forward(params, x, emulate_bf16)
    mu, kappa, w, alpha = decode(out)
    q = guide_pdf(mu, kappa, w, d)
    mix = alpha * q + (1.0 - alpha) * p_bsdf
    return float(np.mean(-weight * (np.log(q) + np.log(mix))))


def output_grad(out, d, weight, p_bsdf):
    """dL/d(raw outputs) (n, 48) of loss(); every per-sample term is divided by n."""
    n = out.shape[0]
    o = out[:, :40].reshape(-1, N_LOBES, 5)
    m = o[:, :, :3]
    nrm = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(nrm > 1e-12, m / np.maximum(nrm, 1e-30), np.array([0.0, 0.0, 1.0]))
    lk_raw = o[:, :, 3]
    kappa = np.exp(np.clip(lk_raw, KAPPA_MIN, KAPPA_MAX))
    logits = o[:, :, 4]
    e = np.exp(logits - logits.max(axis=1, keepdims=True))
    w = e / e.sum(axis=1, keepdims=True)
    s = 1.0 / (1.0 + np.exp(-out[:, 40]))
    alpha = ALPHA_LO + (ALPHA_HI - ALPHA_LO) * s

    dots = np.einsum("nkc,nc->nk", mu, d)
    comp = vmf_norm(kappa) * np.exp(kappa * (dots - 1.0))
    q = (1.0 - EPS_UNIFORM) * (w * comp).sum(axis=1) + EPS_UNIFORM / (4.0 * np.pi)
    mix = alpha * q + (1.0 - alpha) * p_bsdf
    g_q = -weight * (1.0 / q + alpha / mix) / n
    g_alpha = -weight * ((q - p_bsdf) / mix) / n
    g_comp = (1.0 - EPS_UNIFORM) * g_q[:, None] * w
    g_w = (1.0 - EPS_UNIFORM) * g_q[:, None] * comp
    g_logits = w * (g_w - (g_w * w).sum(axis=1, keepdims=True))
    # d log c / d kappa = 1 / kappa - 2 e^{-2 kappa} / (1 - e^{-2 kappa})
    dlogc = 1.0 / kappa - 2.0 * np.exp(-2.0 * kappa) / (-np.expm1(-2.0 * kappa))
    g_kappa = g_comp * comp * (dlogc + (dots - 1.0))
    g_lk = g_kappa * kappa * ((lk_raw > KAPPA_MIN) & (lk_raw < KAPPA_MAX))
    g_mu = (g_comp * comp * kappa)[:, :, None] * d[:, None, :]
    g_m = (g_mu - (g_mu * mu).sum(axis=2, keepdims=True) * mu) / np.maximum(nrm, NORM_FLOOR)
    g = np.zeros_like(out)
    go = g[:, :40].reshape(-1, N_LOBES, 5)
    go[:, :, :3] = g_m
    go[:, :, 3] = g_lk
    go[:, :, 4] = g_logits
    g[:, 40] = g_alpha * (ALPHA_HI - ALPHA_LO) * s * (1.0 - s)
    return g


def gradients(params, x, d, weight, p_bsdf, emulate_bf16=False):
    """Weight and bias gradients of loss() by back-propagation. With
    emulate_bf16 the back-propagated signals are rounded to bfloat16 before
    each product, as the tensor-core kernels store them (the bias gradient is
    then the column sum of the rounded signal, as a product with a ones column)."""
    r = (lambda a: bf16(a).astype(np.float64)) if emulate_bf16 else (lambda a: a)
    rw = (lambda a: bf16(a).astype(np.float64)) if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    out, cache = forward(params, x, emulate_bf16)
    g = output_grad(out, d, weight, p_bsdf)
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        w, _ = params[li]
        g = r(g)
        grads[li] = (g.T @ cache[li], g.sum(axis=0))
        if li > 0:
            g = (g @ rw(w)) * (cache[li] > 0.0)
    return grads


def adam_step(params, grads, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update in place on the FP32 master weights; t is the 1-based step."""
    for li in range(len(params)):
        for pi in range(2):
            p = params[li][pi]
            g = np.asarray(grads[li][pi], dtype=np.float32)
            m[li][pi][...] = np.float32(b1) * m[li][pi] + np.float32(1 - b1) * g
            v[li][pi][...] = np.float32(b2) * v[li][pi] + np.float32(1 - b2) * g * g
            mh = m[li][pi] / np.float32(1 - b1 ** t)
            vh = v[li][pi] / np.float32(1 - b2 ** t)
            p[...] = p - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))


def training_weight(L_final, L_before, beta):
    """Weight of one recorded path vertex: the luminance of the radiance its
    continuation brought back, divided per channel by the path throughput at
    the vertex (an estimate of F(d) / p_sample(d)); channels with zero
    throughput add nothing."""
    dl = np.asarray(L_final, dtype=np.float64) - np.asarray(L_before, dtype=np.float64)
    b = np.asarray(beta, dtype=np.float64)
    ratio = np.where(b > 0.0, dl / np.where(b > 0.0, b, 1.0), 0.0)
    return ratio @ LUMINANCE
