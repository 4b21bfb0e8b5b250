"""CPU oracle of the learned guider (test infrastructure only: tests, smoke and the bench's
CPU baseline import it; the product path never does).

Restates, in numpy, what the GPU guider computes so its forward pass, loss and parameter
gradients can be checked number by number:

* the directional density is a mixture of von Mises-Fisher lobes.  Density
  k / (2 pi (1 - exp(-2k))) exp(k (mu.x - 1)) and the inversion sampler
  w = 1 + log(r + (1 - r) exp(-2k)) / k follow distribution_mixture_models.cxx:93-152;
* the guided direction and the BSDF sample are combined by one-sample MIS with selection
  probability c, density (1 - c) p_bsdf + c p_guide, as SampleWithBinaryMixtureDensity /
  EvaluateWithBinaryMixtureDensity do (renderingalgorithms_pathtracing_guided.cxx:474-544);
* where the reference fits a mixture per spatial cell by EM from radiance records
  (path_guiding.cxx), the mixture here comes from an MLP over the encoded surface point,
  trained on the same kind of record with the KL objective of neural importance sampling:
  minimise -(F / q) log p(wi), p the one-sample-MIS density above.

`forward(..., bf16_round=True)` rounds to bfloat16 where the GPU stores bfloat16
(features, weights, hidden activations, output gradients) so that a difference from the
GPU is only accumulation order; with `bf16_round=False` everything is float64 (for finite
differences).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT, N_LOBES, N_FREQ, N_LAYERS = 96, 64, 48, 8, 12, 5
C_MIN, C_SPAN = 0.05, 0.9                      # c = C_MIN + C_SPAN sigmoid(o)
LOGK_MID = (np.log(0.05) + np.log(40.0)) / 2   # log kappa = MID + HALF tanh((o - MID) / HALF)
LOGK_HALF = (np.log(40.0) - np.log(0.05)) / 2
RECORD_FLOATS = 14  # pos[3] n[3] wo[3] wi[3] p_bsdf f_over_q


def layer_in(l: int) -> int:
    return N_IN if l == 0 else N_HID


def layer_out(l: int) -> int:
    return N_OUT if l == N_LAYERS - 1 else N_HID


def w_offset(l: int) -> int:
    return sum(layer_in(i) * layer_out(i) + layer_out(i) for i in range(l))


def b_offset(l: int) -> int:
    return w_offset(l) + layer_in(l) * layer_out(l)


N_PARAMS = w_offset(N_LAYERS)


def bf16(x) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(a.shape)


def init_params(seed: int = 1) -> np.ndarray:
    """He-uniform weights (the last layer scaled by 0.1), zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for l in range(N_LAYERS):
        lim = np.sqrt(6.0 / layer_in(l)) * (0.1 if l == N_LAYERS - 1 else 1.0)
        n = layer_in(l) * layer_out(l)
        p[w_offset(l):w_offset(l) + n] = rng.uniform(-lim, lim, n)
    return p


def unpack(params):
    """[(W_l [out, in], b_l [out])] views of the flat parameter vector."""
    out = []
    for l in range(N_LAYERS):
        i, o = layer_in(l), layer_out(l)
        W = params[w_offset(l):w_offset(l) + i * o].reshape(o, i)
        b = params[b_offset(l):b_offset(l) + o]
        out.append((W, b))
    return out


_EIGHTH = [np.float32(v) for v in (1.0, 1.09050773, 1.18920712, 1.29683955, 1.41421356, 1.54221083,
                                    1.68179283, 1.83400809)]


def freq(j: int) -> np.float32:
    """Band multiplier 2^(j/8), as the float32 the device computes."""
    return np.float32(_EIGHTH[j & 7] * np.float32(1 << (j >> 3)))


def features(p01, n, wo, round_bf16: bool = True) -> np.ndarray:
    """Encoded surface points (rows of 96): sin/cos of pi 2^(j/8) x for 12 bands j of each
    normalised coordinate x, the coordinates, the normal, the outgoing direction and a
    constant 1, zero padded."""
    p01 = np.asarray(p01, np.float32).reshape(-1, 3)
    n = np.asarray(n, np.float32).reshape(-1, 3)
    wo = np.asarray(wo, np.float32).reshape(-1, 3)
    m = p01.shape[0]
    x = np.zeros((m, N_IN), np.float32)
    k = 0
    for a in range(3):
        f = (np.float32(np.pi) * p01[:, a]).astype(np.float32)
        for j in range(N_FREQ):
            fj = (f * freq(j)).astype(np.float32).astype(np.float64)
            x[:, k] = np.sin(fj)
            x[:, k + 1] = np.cos(fj)
            k += 2
    x[:, k:k + 3] = p01
    x[:, k + 3:k + 6] = n
    x[:, k + 6:k + 9] = wo
    x[:, k + 9] = 1.0
    return bf16(x) if round_bf16 else x


def record_features(rec: np.ndarray, round_bf16: bool = True) -> np.ndarray:
    rec = np.asarray(rec, np.float32).reshape(-1, RECORD_FLOATS)
    return features(rec[:, 0:3], rec[:, 3:6], rec[:, 6:9], round_bf16)


def forward(params, x, bf16_round: bool = True):
    """Returns (outputs [n, 48], hidden activations [4 x (n, 64)], effective weights)."""
    layers = unpack(np.asarray(params, np.float32 if bf16_round else np.float64))
    rnd = bf16 if bf16_round else (lambda v: np.asarray(v, np.float64))
    h = rnd(x).astype(np.float64)
    hidden, weights = [], []
    out = None
    for l, (W, b) in enumerate(layers):
        Wl = rnd(W).astype(np.float64)
        weights.append(Wl)
        z = h @ Wl.T + b.astype(np.float64)
        if l < N_LAYERS - 1:
            h = np.maximum(z, 0.0)
            if bf16_round:
                h = bf16(h).astype(np.float64)
            hidden.append(h)
        else:
            out = z.astype(np.float32) if bf16_round else z
    return out, hidden, weights


def decode(out):
    """Lobe weights, unit means, concentrations and the selection probability c."""
    o = np.asarray(out, np.float64)
    a = o[:, 0:5 * N_LOBES:5]
    a = a - a.max(axis=1, keepdims=True)
    w = np.exp(a)
    w /= w.sum(axis=1, keepdims=True)
    m = np.stack([o[:, 5 * k + 1:5 * k + 4] for k in range(N_LOBES)], axis=1)
    ln = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(ln > 1e-12, m / np.maximum(ln, 1e-300), np.array([0.0, 0.0, 1.0]))
    kap = np.exp(LOGK_MID + LOGK_HALF * np.tanh((o[:, 4:5 * N_LOBES:5] - LOGK_MID) / LOGK_HALF))
    c = C_MIN + C_SPAN / (1.0 + np.exp(-o[:, 5 * N_LOBES]))
    return w, mu, kap, c


def vmf_pdf(mu, kappa, x):
    """distribution_mixture_models.cxx:93-117 (per-lobe density)."""
    cosv = np.einsum("...k,...k->...", mu, x)
    return kappa / (2 * np.pi * (1 - np.exp(-2 * kappa))) * np.exp(kappa * (cosv - 1))


def mixture_pdf(out, wi):
    w, mu, kap, _ = decode(out)
    wi = np.asarray(wi, np.float64).reshape(-1, 1, 3)
    return (w * vmf_pdf(mu, kap, wi)).sum(axis=1)


def vmf_sample(mu, kappa, r1, r2):
    """distribution_mixture_models.cxx:120-145: inversion of the vMF cosine marginal."""
    w = 1 + np.log(r2 + (1 - r2) * np.exp(-2 * kappa)) / kappa
    rho = np.sqrt(np.maximum(0.0, 1 - w * w))
    local = np.stack([rho * np.cos(2 * np.pi * r1), rho * np.sin(2 * np.pi * r1), w], axis=-1)
    mu = np.asarray(mu, np.float64)
    # Any orthonormal frame around mu gives the same distribution.
    t = np.where(np.abs(mu[..., :1]) > 0.9, np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    b1 = np.cross(mu, t)
    b1 /= np.linalg.norm(b1, axis=-1, keepdims=True)
    b2 = np.cross(mu, b1)
    return local[..., :1] * b1 + local[..., 1:2] * b2 + local[..., 2:3] * mu


def mis_pdf(c, p_bsdf, p_guide):
    """One-sample MIS density (renderingalgorithms_pathtracing_guided.cxx:474-544)."""
    return (1 - c) * p_bsdf + c * p_guide


def loss_and_output_grad(out, rec):
    """Mean of -(F/q) log p(wi) and its gradient with respect to the 41 outputs (float64)."""
    o = np.asarray(out, np.float64)
    rec = np.asarray(rec, np.float64).reshape(-1, RECORD_FLOATS)
    n = o.shape[0]
    x = rec[:, 9:12]
    pb = rec[:, 12]
    wgt = rec[:, 13]
    a = o[:, 0:5 * N_LOBES:5]
    a = a - a.max(axis=1, keepdims=True)
    pi = np.exp(a)
    pi /= pi.sum(axis=1, keepdims=True)
    m = np.stack([o[:, 5 * k + 1:5 * k + 4] for k in range(N_LOBES)], axis=1)
    ln = np.linalg.norm(m, axis=2)
    ok = ln > 1e-12
    mu = np.where(ok[..., None], m / np.maximum(ln, 1e-300)[..., None], np.array([0.0, 0.0, 1.0]))
    th = np.tanh((o[:, 4:5 * N_LOBES:5] - LOGK_MID) / LOGK_HALF)
    kap = np.exp(LOGK_MID + LOGK_HALF * th)
    cosv = np.einsum("nkj,nj->nk", mu, x)
    v = kap / (2 * np.pi * (1 - np.exp(-2 * kap))) * np.exp(kap * (cosv - 1))
    pv = (pi * v).sum(axis=1)
    sg = 1 / (1 + np.exp(-o[:, 5 * N_LOBES]))
    c = C_MIN + C_SPAN * sg
    p = np.maximum((1 - c) * pb + c * pv, 1e-20)
    pos = wgt > 0
    loss = np.where(pos, -wgt * np.log(p), 0.0).sum() / n
    dLdp = np.where(pos, -wgt / p, 0.0)
    dLdpv = dLdp * c
    g = np.zeros((n, N_OUT))
    g[:, 0:5 * N_LOBES:5] = dLdpv[:, None] * pi * (v - pv[:, None])
    s = dLdpv[:, None] * pi * v * kap
    gx = x[:, None, :] * s[..., None]
    proj = gx - mu * np.einsum("nkj,nkj->nk", mu, gx)[..., None]
    dm = np.where(ok[..., None], proj / np.maximum(ln, 1e-300)[..., None], 0.0)
    for k in range(N_LOBES):
        g[:, 5 * k + 1:5 * k + 4] = dm[:, k]
    e2 = np.exp(-2 * kap)
    dlogv = 1 / kap - 2 * e2 / (1 - e2) + (cosv - 1)
    g[:, 4:5 * N_LOBES:5] = dLdpv[:, None] * pi * v * dlogv * kap * (1 - th * th)
    g[:, 5 * N_LOBES] = dLdp * (pv - pb) * C_SPAN * sg * (1 - sg)
    return loss, g / n


def loss(params, rec, bf16_round: bool = False) -> float:
    x = record_features(rec, bf16_round)
    out, _, _ = forward(params, x, bf16_round)
    return loss_and_output_grad(out, rec)[0]


def gradient(params, rec, bf16_round: bool = True):
    """Mean loss and its gradient with respect to the flat parameter vector (backprop through
    the ReLU MLP; bfloat16 rounding of the output and hidden gradients when bf16_round)."""
    x = record_features(rec, bf16_round).astype(np.float64)
    out, hidden, weights = forward(params, x, bf16_round)
    L, dy = loss_and_output_grad(out, rec)
    if bf16_round:
        dy = bf16(dy).astype(np.float64)
    grad = np.zeros(N_PARAMS, np.float64)
    for l in range(N_LAYERS - 1, -1, -1):
        xin = x if l == 0 else hidden[l - 1]
        i, o = layer_in(l), layer_out(l)
        grad[w_offset(l):w_offset(l) + i * o] = (dy.T @ xin).reshape(-1)
        grad[b_offset(l):b_offset(l) + o] = dy.sum(axis=0)
        if l > 0:
            dh = (dy @ weights[l]) * (hidden[l - 1] > 0)
            dy = bf16(dh).astype(np.float64) if bf16_round else dh
    return L, grad


def adam(params, m, v, grad, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba 2015), as the GPU applies it; returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    bc1 = 1 - b1 ** step
    bc2 = 1 - b2 ** step
    p = params - lr * (m / bc1) / (np.sqrt(v / bc2) + eps)
    return p, m, v


def random_records(n: int, seed: int = 0, sharp=(0.3, 0.5, 0.8)) -> np.ndarray:
    """Synthetic training records: points in the unit box, normals and outgoing directions
    on the sphere, incident directions concentrated near `sharp` (a fixed bright direction)
    with a cosine-lobe density as p_bsdf and positive F/q weights."""
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, RECORD_FLOATS), np.float32)
    rec[:, 0:3] = rng.random((n, 3))
    nn = rng.normal(size=(n, 3))
    rec[:, 3:6] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    rec[:, 6:9] = wo / np.linalg.norm(wo, axis=1, keepdims=True)
    mu = np.asarray(sharp, np.float64)
    mu /= np.linalg.norm(mu)
    wi = vmf_sample(np.broadcast_to(mu, (n, 3)), 20.0, rng.random(n), rng.random(n))
    rec[:, 9:12] = wi
    rec[:, 12] = np.maximum(0.0, (wi * rec[:, 3:6]).sum(1)) / np.pi + 0.02
    rec[:, 13] = rng.uniform(0.1, 2.0, n)
    return rec
