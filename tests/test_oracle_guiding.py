"""The CPU oracle of the learned guider against analytic facts: the loss gradient against
central finite differences, the vMF sampler against its density's moments
(tests_guiding.cxx:639-676 checks the same sampler's sanity), normalisation of the mixture,
unbiasedness of the one-sample MIS estimator, bfloat16 rounding, Adam, and that training
on synthetic records lowers the loss."""
import numpy as np
import pytest

from oracle import guiding as G


def _params(seed=3, bias=0.05):
    p = G.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed + 100)
    for l in range(G.N_LAYERS):
        o = G.layer_out(l)
        p[G.b_offset(l):G.b_offset(l) + o] = rng.normal(0, bias, o)
    return p


def test_layout():
    assert G.N_PARAMS == 96 * 64 + 64 + 3 * (64 * 64 + 64) + 64 * 48 + 48
    assert G.w_offset(1) == 96 * 64 + 64


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -2.5, 0.0], np.float32)
    r = G.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                        # tie to even
    assert r[2] == np.float32(1.0 + 2 ** -6)  # tie to even (upwards)
    assert r[3] == np.float32(1.0 + 2 ** -7)
    assert r[4] == -2.5 and r[5] == 0.0


def test_features_layout():
    p = np.array([[0.25, 0.5, 0.75]])
    n = np.array([[0.0, 1.0, 0.0]])
    wo = np.array([[0.6, 0.0, 0.8]])
    x = G.features(p, n, wo, round_bf16=False)[0]
    assert x.shape == (96,)
    assert np.isclose(x[0], np.sin(np.pi * 0.25), atol=1e-6) and np.isclose(x[1], np.cos(np.pi * 0.25), atol=1e-6)
    assert np.isclose(x[2], np.sin(2 ** 0.125 * np.pi * 0.25), atol=1e-6)
    assert np.isclose(x[16], np.sin(2 * np.pi * 0.25), atol=1e-6)
    assert np.allclose(x[72:75], p[0]) and np.allclose(x[75:78], n[0]) and np.allclose(x[78:81], wo[0])
    assert x[81] == 1.0 and np.all(x[82:] == 0)


def test_gradient_matches_finite_differences():
    rec = G.random_records(48, seed=5)
    p = _params()
    L, g = G.gradient(p, rec, bf16_round=False)
    assert np.isfinite(L) and L > 0
    rng = np.random.default_rng(7)
    # Parameters of every layer, weights and biases.
    idx = []
    for l in range(G.N_LAYERS):
        n = G.layer_in(l) * G.layer_out(l)
        idx += list(G.w_offset(l) + rng.choice(n, 6, replace=False))
        idx += list(G.b_offset(l) + rng.choice(G.layer_out(l), 2, replace=False))
    eps = 1e-5
    fd = []
    for i in idx:
        a = p.copy()
        a[i] += eps
        b = p.copy()
        b[i] -= eps
        fd.append((G.loss(a, rec) - G.loss(b, rec)) / (2 * eps))
    fd = np.array(fd)
    an = g[idx]
    err = np.linalg.norm(fd - an) / np.linalg.norm(fd)
    assert err < 1e-4, (err, np.c_[fd, an][:10])


def test_output_gradient_matches_finite_differences():
    """The loss gradient with respect to the 41 outputs alone, also where the smooth output
    maps saturate."""
    rec = G.random_records(16, seed=9)
    rng = np.random.default_rng(2)
    out = rng.normal(0, 0.7, (16, G.N_OUT))
    out[:, 4:40:5] = rng.uniform(-1, 3, (16, 8))       # concentrations in range
    out[0, 4] = 9.0                                     # kappa near its upper limit
    out[1, 40] = 5.0                                    # c near its upper limit
    L, g = G.loss_and_output_grad(out, rec)
    eps = 1e-6
    for r in range(4):
        for j in range(41):
            a = out.copy()
            a[r, j] += eps
            b = out.copy()
            b[r, j] -= eps
            fd = (G.loss_and_output_grad(a, rec)[0] - G.loss_and_output_grad(b, rec)[0]) / (2 * eps)
            assert abs(fd - g[r, j]) <= 1e-5 * max(1.0, abs(fd)), (r, j, fd, g[r, j])
    # Saturated outputs keep a (small) gradient instead of a dead zone.
    assert g[0, 4] != 0.0 and g[1, 40] != 0.0


@pytest.mark.parametrize("kappa", [0.5, 5.0, 40.0])
def test_vmf_sampler_moments(kappa):
    rng = np.random.default_rng(int(kappa * 10))
    n = 200_000
    mu = np.array([0.3, -0.5, 0.81])
    mu /= np.linalg.norm(mu)
    x = G.vmf_sample(np.broadcast_to(mu, (n, 3)), kappa, rng.random(n), rng.random(n))
    assert np.allclose(np.linalg.norm(x, axis=1), 1.0, atol=1e-9)
    c = x @ mu
    # E[mu.x] = coth(k) - 1/k for the vMF on the sphere.
    expect = 1 / np.tanh(kappa) - 1 / kappa
    assert abs(c.mean() - expect) < 4 * c.std() / np.sqrt(n)
    # Importance-sampled integral of 1 with the density: E[1 / p] = 4 pi.
    w = 1 / G.vmf_pdf(mu, kappa, x)
    if kappa <= 5:
        assert abs(w.mean() - 4 * np.pi) < 4 * w.std() / np.sqrt(n)


def test_mixture_pdf_normalised():
    rng = np.random.default_rng(4)
    out = rng.normal(0, 1, (1, G.N_OUT))
    out[:, 4:40:5] = rng.uniform(-1, 2.5, (1, 8))
    n = 400_000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pdf = G.mixture_pdf(np.repeat(out, n, axis=0), d)
    est = pdf.mean() * 4 * np.pi
    err = pdf.std() * 4 * np.pi / np.sqrt(n)
    assert abs(est - 1.0) < 4 * err + 1e-3


def test_one_sample_mis_unbiased():
    """E[f / ((1-c) p_bsdf + c p_guide)] with the one-sample mixture = integral of f."""
    rng = np.random.default_rng(11)
    n = 400_000
    nrm = np.array([0.0, 0.0, 1.0])
    c = 0.6
    mu = np.array([0.0, 0.6, 0.8])
    kap = 8.0
    # Cosine-weighted hemisphere sampler as the BSDF part.
    u1, u2 = rng.random(n), rng.random(n)
    r = np.sqrt(u1)
    bs = np.stack([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2), np.sqrt(1 - u1)], 1)
    gs = G.vmf_sample(np.broadcast_to(mu, (n, 3)), kap, rng.random(n), rng.random(n))
    pick = rng.random(n) < c
    x = np.where(pick[:, None], gs, bs)
    p_b = np.maximum(x @ nrm, 0) / np.pi
    p = G.mis_pdf(c, p_b, G.vmf_pdf(mu, kap, x))
    f = np.maximum(x @ nrm, 0) * (1 + 4 * np.maximum(x @ mu, 0) ** 8)   # cosine times a lobe
    est = f / p
    # Reference integral by a plain uniform-sphere estimate with many samples.
    d = rng.normal(size=(2_000_000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    fr = np.maximum(d @ nrm, 0) * (1 + 4 * np.maximum(d @ mu, 0) ** 8) * 4 * np.pi
    ref, ref_err = fr.mean(), fr.std() / np.sqrt(len(fr))
    assert abs(est.mean() - ref) < 4 * np.hypot(est.std() / np.sqrt(n), ref_err)


def test_adam_step():
    p = np.array([1.0, -2.0])
    g = np.array([0.5, -0.1])
    p1, m, v = G.adam(p, np.zeros(2), np.zeros(2), g, 1, 0.01)
    # First bias-corrected step moves each parameter by lr against its gradient's sign.
    assert np.allclose(p1, p - 0.01 * np.sign(g), atol=1e-7)


def test_training_lowers_loss():
    rec = G.random_records(1024, seed=1)
    # Eight distinct surface points share the records, so the network must learn the
    # directional distribution rather than memorise single directions.
    rec[:, 0:9] = rec[np.arange(1024) % 8, 0:9]
    p = G.init_params(2).astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    L0 = G.loss(p, rec)
    for step in range(1, 121):
        L, g = G.gradient(p, rec, bf16_round=False)
        p, m, v = G.adam(p, m, v, g, step, 5e-3)
    L1 = G.loss(p, rec)
    assert L1 < L0 - 0.5, (L0, L1)
    # The learned mixture concentrates on the records' bright direction.
    mu = np.array([0.3, 0.5, 0.8]) / np.linalg.norm([0.3, 0.5, 0.8])
    x = G.record_features(rec[:64], False)
    out, _, _ = G.forward(p, x, False)
    assert np.median(G.mixture_pdf(out, np.broadcast_to(mu, (64, 3)))) > 1.0
