"""Quadtree radiance distribution of the tree guider, on the CPU.

The oracle (oracle/tree_guiding.py) is pinned by the reference's own quadtree tests
(tests_guiding.cxx:515-635, 695-707: QuadTreeBuilderTrivial, QuadTreeDivideIntoChildRanges,
QuadTreeBuilderConsistency, TreeAdaptor, PolarMap) and by the distribution's analytic
facts (the density integrates to one, sampling follows it); the library's host fit
(tt_quadtree_fit_batch, no GPU needed) must equal the oracle bit for bit.
"""
import numpy as np
import pytest
from scipy import stats

from oracle.tree_guiding import (Quad, adapt_tree, dir_to_square, quad_leaf, quad_pdf, quad_sample,
                                 square_to_dir)


def _leaf_mask(child):
    return np.array([c[0] < 0 for c in child])


def _squares(child):
    """Square (lo, hi) of every node, depth first."""
    out = [None] * len(child)

    def rec(k, lo, hi):
        out[k] = (lo, hi)
        if child[k][0] >= 0:
            c0, c1 = 0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])
            for q in range(4):
                clo = [c0 if q & 1 else lo[0], c1 if q & 2 else lo[1]]
                chi = [hi[0] if q & 1 else c0, hi[1] if q & 2 else c1]
                rec(child[k][q], clo, chi)

    rec(0, [0.0, 0.0], [1.0, 1.0])
    return out


def test_reference_builder_trivial():
    """QuadTreeBuilderTrivial: no records, one leaf."""
    q = Quad()
    q.initial_fit(np.zeros((0, 2)), np.zeros(0), fraction=1.0)
    assert len(q.child) == 1 and q.child[0][0] < 0


def test_reference_divide_into_child_ranges():
    """QuadTreeDivideIntoChildRanges: one, two, three and four records at the centres of the
    four quadrants land in children 0..3 in that order."""
    pts = [(0.25, 0.25)] + [(0.75, 0.25)] * 2 + [(0.25, 0.75)] * 3 + [(0.75, 0.75)] * 4
    rng = np.random.default_rng(3)
    pts = np.array(pts, np.float32)[rng.permutation(len(pts))]
    q = Quad()
    q.initial_fit(pts, np.ones(len(pts)), fraction=0.05)
    assert q.child[0][0] >= 0
    assert [q.stats[c][2] for c in q.child[0]] == [1, 2, 3, 4]


def test_reference_builder_consistency():
    """QuadTreeBuilderConsistency: 100 uniform records of weight 1, threshold 1.00001/100 of
    the total: the root splits, every node counts the records inside its square, nodes are
    numbered depth first (a parent before its children)."""
    rng = np.random.default_rng(11)
    pts = rng.random((100, 2)).astype(np.float32)
    q = Quad()
    q.initial_fit(pts, np.ones(100), fraction=1.00001 / 100)
    assert q.child[0][0] >= 0
    for k, (lo, hi) in enumerate(_squares(q.child)):
        inside = np.sum((pts[:, 0] >= lo[0]) & (pts[:, 0] < hi[0]) & (pts[:, 1] >= lo[1]) & (pts[:, 1] < hi[1]))
        assert q.stats[k][2] == inside
        if q.child[k][0] >= 0:
            assert all(c > k for c in q.child[k])
            assert q.stats[k][2] == sum(q.stats[c][2] for c in q.child[k])
        elif q.stats[k][2] > 1:
            depth = int(round(-np.log2(hi[0] - lo[0])))
            assert depth == 7  # MAX_DEPTH 8 counts the root as depth 1


def test_reference_tree_adaptor():
    """TreeAdaptor: a leaf of weight 16 adapted with threshold fraction 5/16 gives 1 + 4
    nodes; adapted again with 2/16 gives 1 + 4 + 16; a weight of 10 pushed at (0.75, 0.75)
    adds to the root."""
    child = [[-1, -1, -1, -1]]
    w = [16.0]
    child, _, w = adapt_tree(child, w, 5.0 / 16.0)
    assert len(child) == 1 + 4 and len(w) == len(child)
    child, _, w = adapt_tree(child, w, 2.0 / 16.0)
    assert len(child) == 1 + 4 + 16 and len(w) == len(child)
    w = [float(x) for x in w]
    k, lo, hi = 0, [0.0, 0.0], [1.0, 1.0]
    while True:
        w[k] += 10.0
        if child[k][0] < 0:
            break
        c0, c1 = 0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])
        qd = (0 if 0.75 < c0 else 1) | (0 if 0.75 < c1 else 2)
        lo = [c0 if qd & 1 else lo[0], c1 if qd & 2 else lo[1]]
        hi = [hi[0] if qd & 1 else c0, hi[1] if qd & 2 else c1]
        k = child[k][qd]
    assert abs(w[0] - (16.0 + 10.0)) < 1e-3


def test_reference_polar_map():
    """PolarMap: square -> sphere -> square round trip (the reference checks 1e-3)."""
    rng = np.random.default_rng(2)
    x = rng.random((1000, 2)).astype(np.float32)
    y = dir_to_square(square_to_dir(x).astype(np.float32))
    assert np.abs(x - y).max() < 1e-5
    d = square_to_dir(x)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0)


def _records(seed, n, concentrated=0.5):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    m = int(concentrated * n)
    d[:m] = d[:m] * 0.15 + np.array([0.3, -0.2, 0.9])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d.astype(np.float32), rng.exponential(1.0, n).astype(np.float32)


def _oracle_fit(da, wa, db, wb, stage):
    q = Quad()
    q.initial_fit(dir_to_square(da), wa)
    q.bake()
    if stage >= 1:
        q.incremental_fit(dir_to_square(db), wb)
    if stage >= 2:
        q.update_and_bake()
    return q


@pytest.mark.parametrize("seed,n,conc", [(1, 2000, 0.5), (7, 300, 0.9), (9, 5000, 0.1)])
def test_library_quadtree_fit_matches_oracle(seed, n, conc):
    from naivetrace_b200.algo import quadtree_fit_batch
    da, wa = _records(seed, n, conc)
    db, wb = _records(seed + 100, n // 2, conc)
    for stage in range(3):
        ch, w, pr = quadtree_fit_batch(da, wa, db, wb, stage=stage)
        q = _oracle_fit(da, wa, db, wb, stage)
        assert np.array_equal(ch, np.array(q.child, np.int32)), stage
        assert np.array_equal(w, q.probs), stage
        assert np.array_equal(pr, q.prior), stage


def test_fit_invariants():
    """The initial tree splits exactly the nodes whose weight exceeds 0.1 of the total (below
    depth 8), inner sampling weights are the sums of their children, and the adaptation
    keeps them so."""
    da, wa = _records(4, 3000)
    q = _oracle_fit(da, wa, None, None, 0)
    uv = dir_to_square(da)
    thr = 0.1 * float(np.sum(wa.astype(np.float64)))
    for k, (lo, hi) in enumerate(_squares(q.child)):
        inside = (uv[:, 0] >= lo[0]) & (uv[:, 0] < hi[0]) & (uv[:, 1] >= lo[1]) & (uv[:, 1] < hi[1])
        wsum = float(np.sum(wa[inside].astype(np.float64)))
        depth = int(round(-np.log2(hi[0] - lo[0])))
        if q.child[k][0] >= 0:
            assert wsum > thr
            assert q.probs[k] == pytest.approx(sum(float(q.probs[c]) for c in q.child[k]), rel=1e-5)
        elif depth < 7:
            assert wsum <= thr * (1 + 1e-9)
    db, wb = _records(5, 1500)
    q.incremental_fit(dir_to_square(db), wb)
    assert q.update_and_bake()
    for k in range(len(q.child)):
        if q.child[k][0] >= 0:
            assert q.probs[k] == pytest.approx(sum(float(q.probs[c]) for c in q.child[k]), rel=1e-5)


def test_density_integrates_to_one():
    da, wa = _records(6, 4000)
    q = _oracle_fit(da, wa, None, None, 0)
    rng = np.random.default_rng(8)
    d = rng.normal(size=(200000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    est = float(np.mean(quad_pdf(q.child, q.probs, d.astype(np.float32)))) * 4 * np.pi
    assert abs(est - 1.0) < 0.02, est
    leaves = _leaf_mask(q.child)
    assert float(np.sum(q.probs[leaves].astype(np.float64))) == pytest.approx(float(q.probs[0]), rel=1e-5)


def test_oracle_sampling_follows_leaf_weights():
    """Hierarchical warping picks leaf k with probability weight_k / weight_root and lands
    uniformly inside its square (the density it reports equals the tree's density there)."""
    da, wa = _records(12, 3000)
    q = _oracle_fit(da, wa, None, None, 0)
    leaves = np.flatnonzero(_leaf_mask(q.child))
    rng = np.random.default_rng(13)
    n = 40000
    counts = np.zeros(len(q.child))
    for u0, u1 in rng.random((n, 2)):
        (pu, pv), pdf, k = quad_sample(q.child, q.probs, u0, u1)
        counts[k] += 1
        kk, area = quad_leaf(q.child, (pu, pv))
        assert kk == k
        assert float(pdf) == pytest.approx(float(q.probs[k]) / (float(q.probs[0]) * area), rel=1e-5)
    exp = q.probs[leaves].astype(np.float64) / float(q.probs[0]) * n
    keep = exp > 5
    obs = counts[leaves][keep]
    e = exp[keep] * obs.sum() / exp[keep].sum()
    p = stats.chisquare(obs, e).pvalue
    assert p > 1e-3, p
