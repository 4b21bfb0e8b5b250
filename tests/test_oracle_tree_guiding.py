"""The tree guider's CPU pieces: the library's host kd-tree builder against the oracle's
(the reference's Builder, path_guiding_tree.hxx:306-440), and the oracle's incremental vMF
EM (distribution_mixture_models.cxx:279-388) against analytic facts: it recovers the mean
and concentration of a single von Mises-Fisher distribution, keeps a normalised mixture, and
the prior dominates while few records have been seen."""
import numpy as np
import pytest

from oracle import tree_guiding as T


def _vmf_samples(mu, kappa, n, rng):
    from oracle import guiding as G
    return G.vmf_sample(np.broadcast_to(mu, (n, 3)), kappa, rng.random(n), rng.random(n))


@pytest.mark.parametrize("n,min_points", [(5000, 100), (1999, 100), (150, 100), (4096, 7)])
def test_kdtree_build_matches_oracle(n, min_points):
    from naivetrace_b200.algo import kdtree_build_batch
    rng = np.random.default_rng(n)
    pts = rng.random((n, 3)).astype(np.float32)
    pts[:, 1] *= 0.3                       # anisotropic: splits favour x and z
    cells, nc = kdtree_build_batch(pts, min_points)
    nodes, ref = T.build_kdtree(pts, min_points)
    assert nc == ref.max() + 1
    np.testing.assert_array_equal(cells, ref)
    counts = np.bincount(cells)
    if nc > 1:
        assert counts.min() >= min_points and counts.max() < 2 * min_points + 2
    # Lookup agrees with the build for the points themselves.
    look = np.array([T.lookup(nodes, p) for p in pts[:300]])
    np.testing.assert_array_equal(look, ref[:300])


def test_em_recovers_a_single_vmf():
    rng = np.random.default_rng(3)
    mu = np.array([0.2, -0.5, 0.84])
    mu /= np.linalg.norm(mu)
    x = _vmf_samples(mu, 12.0, 20000, rng)
    c = T.CellFit().fit(x, np.ones(len(x)))
    assert abs(c.w.sum() - 1) < 1e-12
    # The weighted mean direction and its concentration: the mixture's mean resultant.
    m = (c.w[:, None] * c.mu * (1 / np.tanh(c.k) - 1 / c.k)[:, None]).sum(axis=0)
    assert np.linalg.norm(m / np.linalg.norm(m) - mu) < 0.05
    # Concentrated, though less than the data (mean cosine 0.92): the prior keeps a share of
    # every lobe and pulls the concentrations towards 2.
    assert 0.75 < np.linalg.norm(m) < np.mean(x @ mu)
    p = T.mixture_pdf(c.w, c.mu, c.k, np.array([mu, -mu]))
    assert p[0] > 50 * p[1]
    # The fitted mixture is a density on the sphere.
    d = rng.normal(size=(200000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    integral = T.mixture_pdf(c.w, c.mu, c.k, d).mean() * 4 * np.pi
    assert abs(integral - 1) < 0.02


def test_em_prior_and_pending_statistics():
    rng = np.random.default_rng(5)
    x = _vmf_samples(np.array([0, 0, 1.0]), 20.0, 95, rng)
    c = T.CellFit().fit(x, np.ones(95))
    # 95 records with strength 1: chunks of 10, nine maximisation steps, five records pending.
    assert c.pend_n == 5 and c.n_w == 95
    c2 = T.CellFit().fit(x[:50], np.ones(50)).fit(x[50:], np.ones(45))
    np.testing.assert_allclose(c2.w, c.w, rtol=1e-12)
    np.testing.assert_allclose(c2.mu, c.mu, rtol=1e-12)
    assert np.all((c.k >= T.KAPPA_MIN) & (c.k <= T.KAPPA_MAX))
    # Fewer than one chunk: the prior stays untouched.
    c3 = T.CellFit().fit(x[:7], np.ones(7))
    w0, mu0, k0 = T.prior_mixture()
    np.testing.assert_array_equal(c3.mu, mu0)
    np.testing.assert_array_equal(c3.k, k0)
