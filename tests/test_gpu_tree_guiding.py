"""The tree guider (method TT_GUIDE_TREE) on the GPU against the CPU oracle
(oracle/tree_guiding.py), and tree-guided rendering against plain rendering.

1. The device fit of one cell (one warp running the EM) against the float64 oracle:
   incremental EM as the reference runs it, split over two calls so that the pending
   statistics carry over, and batch EM.
2. Rounds build and adapt the kd-tree: cells multiply, every mixture stays a normalised
   8-lobe vMF mixture within the concentration limits, lookups land in valid cells.
3. Tree-guided rendering is unbiased (tile z-tests against plain renders, training between
   passes and frozen, with and without media) and lowers relMSE at equal samples on the
   gap-lit room.
"""
import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext, vmf_fit_batch
from naivetrace_b200.scene import make_params
from oracle import guiding as G
from oracle import tree_guiding as T
from oracle.oracle import combine
from test_gpu_guiding import assert_tiles_agree, tile_means

pytestmark = pytest.mark.gpu


def _records(n, seed):
    rng = np.random.default_rng(seed)
    mu1, mu2 = np.array([0, 0, 1.0]), np.array([0.6, 0.8, 0])
    a = n * 4 // 7
    x = np.concatenate([G.vmf_sample(np.broadcast_to(mu1, (a, 3)), 8.0, rng.random(a), rng.random(a)),
                        G.vmf_sample(np.broadcast_to(mu2, (n - a, 3)), 30.0, rng.random(n - a), rng.random(n - a))])
    x = x[rng.permutation(n)]
    return np.c_[x, rng.lognormal(0, 1, n)].astype(np.float32)


def _compare(mix, fit, cell):
    w, mu, k = T.unpack(mix)
    np.testing.assert_allclose(w, cell.w, atol=2e-5)
    np.testing.assert_allclose(mu, cell.mu, atol=2e-5)
    np.testing.assert_allclose(k, cell.k, rtol=2e-4)
    assert int(fit[3]) == cell.pend_n
    np.testing.assert_allclose(fit[0], cell.avg_w, rtol=1e-5)
    np.testing.assert_allclose(fit[12:36].reshape(8, 3), cell.pend_wrx, rtol=1e-4, atol=1e-3)


def test_vmf_fit_matches_oracle(gpu_lib):
    rec = _records(1234, 1)
    x, w = rec[:, :3].astype(np.float64), rec[:, 3].astype(np.float64)
    # Incremental: 1234 records, prior strength 12.34, chunks of 120: ten maximisation
    # steps and 34 records pending; then 700 more with the state carried over.
    m1, f1 = vmf_fit_batch(rec[:1234])
    c = T.CellFit().fit(x, w)
    _compare(m1, f1, c)
    rec2 = _records(700, 2)
    m2, f2 = vmf_fit_batch(rec2, m1, f1)
    c.fit(rec2[:, :3].astype(np.float64), rec2[:, 3].astype(np.float64))
    _compare(m2, f2, c)
    # Batch EM: six iterations over all records.
    m3, f3 = vmf_fit_batch(rec, batch_iters=6)
    c3 = T.CellFit().fit(x, w, batch_iters=6)
    _compare(m3, f3, c3)


def test_tree_rounds_and_cells(gpu_lib):
    scene = scenes.guiding_room(96, 54)
    g = GpuContext(scene, make_params(max_ray_depth=12))
    g.set_guiding(True, 1, method=abi.GUIDE_TREE, tree_subdivision=100, tree_em_iters=4, seed=3)
    for k in range(4):
        g.render(8, seed=1 + k)
    info = g.tree_info()
    assert info["rounds"] == 4 and info["cells"] > 1 and info["nodes"] == info["cells"] - 1
    assert info["records"] == g.stats()["guide_records"] > 0
    mix = g.tree_mixtures().astype(np.float64)
    np.testing.assert_allclose(mix[:, :8].sum(axis=1), 1.0, atol=1e-5)
    np.testing.assert_allclose(np.linalg.norm(mix[:, 8:32].reshape(-1, 8, 3), axis=2), 1.0, atol=1e-5)
    assert np.all((mix[:, 32:] >= 1e-4 - 1e-9) & (mix[:, 32:] <= 40 + 1e-5))
    cells = g.tree_lookup(np.random.default_rng(0).random((1000, 3)))
    assert cells.min() >= 0 and cells.max() < info["cells"]
    assert g.stats()["error_flags"] == 0


def _batches(ctx, K, spp, seed0, xres, yres, tile):
    out = []
    for k in range(K):
        ctx.clear()
        ctx.render(spp, seed=seed0 + k)
        acc, light, sppc, splat = ctx.accumulators()
        out.append(tile_means(combine(acc, light, spp, splat, ctx.npix), xres, yres, tile))
    return np.array(out)


@pytest.mark.parametrize("name,train_during,em_iters", [("cornell_box", True, 4), ("cornell_box_medium", False, 4),
                                                        ("guiding_room", True, 0), ("guiding_room", False, 4)])
def test_tree_guided_render_unbiased(gpu_lib, name, train_during, em_iters):
    """Tile means of tree-guided and plain renders agree within the Bonferroni bound of
    assert_tiles_agree (as for the learned guider)."""
    xres, yres, tile = (64, 64, 16) if name != "guiding_room" else (96, 54, 18)
    scene = getattr(scenes, name)(xres, yres)
    p = make_params(max_ray_depth=10 if name != "guiding_room" else 12)
    plain = GpuContext(scene, p)
    guided = GpuContext(scene, p)
    kw = dict(method=abi.GUIDE_TREE, tree_subdivision=100, tree_em_iters=em_iters, seed=5)
    guided.set_guiding(True, 1, **kw)
    for k in range(6):
        guided.render(4, seed=900 + k)
    rounds_before = guided.tree_info()["rounds"]
    assert rounds_before == 6
    if not train_during:
        guided.set_guiding(True, 0, **kw)
    K = 32  # batches per side: the room's batch means are skewed, and 16 left the t tails too light
    spp = 16 if name != "guiding_room" else 64
    tp = _batches(plain, K, spp, 100, xres, yres, tile)
    tg = _batches(guided, K, spp, 300, xres, yres, tile)
    assert (guided.tree_info()["rounds"] > rounds_before) == train_during
    assert_tiles_agree(tp, tg)
    assert guided.stats()["error_flags"] == 0


def test_tree_guiding_gain(gpu_lib):
    """Gap-lit room, 64 spp after eight 4-spp training rounds (batch EM, 200 records per
    initial cell): relMSE against a 4096-spp plain render below plain's by > 1.25x
    (measured about 1.5x)."""
    xres, yres = 160, 90
    scene = scenes.guiding_room(xres, yres)
    p = make_params(max_ray_depth=12)
    ref = GpuContext(scene, p)
    for k in range(16):
        ref.render(256, seed=10_000 + k)
    R = ref.framebuffer().astype(np.float64)

    def relmse(g):
        I = g.framebuffer().astype(np.float64)
        return float(np.mean((I - R) ** 2 / (R * R + 1e-2)))

    e_plain = []
    for k in range(3):
        g = GpuContext(scene, p)
        g.render(64, seed=100 + k)
        e_plain.append(relmse(g))
    g = GpuContext(scene, p)
    kw = dict(method=abi.GUIDE_TREE, tree_subdivision=200, tree_em_iters=4, seed=7)
    g.set_guiding(True, 1, **kw)
    for k in range(8):
        g.render(4, seed=200 + k)
    g.set_guiding(True, 0, **kw)
    e_tree = []
    for k in range(3):
        g.clear()
        g.render(64, seed=300 + k)
        e_tree.append(relmse(g))
    gain = np.mean(e_plain) / np.mean(e_tree)
    assert gain > 1.25, (e_plain, e_tree)


# ---- Quadtree distribution (tree_distribution = TREE_QUADTREE) -------------------------

def _quad_fixture(seed=21, n=4000):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    m = n // 2
    d[:m] = d[:m] * 0.1 + np.array([0.5, 0.5, 0.7])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.exponential(1.0, n).astype(np.float32)
    from naivetrace_b200.algo import quadtree_fit_batch
    ch, wt, _ = quadtree_fit_batch(d.astype(np.float32), w, d[::3].astype(np.float32), w[::3], stage=2)
    return ch, wt


def test_quadtree_device_sampler_matches_oracle(gpu_lib):
    """The tree-guided kernel's quadtree sampler (hierarchical warping in float32) against
    the oracle's on the same uniforms: the same leaf and point, directions within float
    rounding, densities equal; the density evaluated at the returned direction equals the
    sampled one except where the direction sits on a leaf boundary."""
    from naivetrace_b200.algo import quadtree_sample_batch
    ch, wt = _quad_fixture()
    rng = np.random.default_rng(5)
    u = rng.random((20000, 2)).astype(np.float32)
    d, pdf, pdf_eval = quadtree_sample_batch(ch, wt, u)
    pts, pdo = [], []
    for u0, u1 in u:
        (pu, pv), pd, _ = T.quad_sample(ch.tolist(), wt, u0, u1)
        pts.append((pu, pv))
        pdo.append(float(pd) / (4 * np.pi))
    do = T.square_to_dir(np.array(pts, np.float32))
    np.testing.assert_allclose(d, do, atol=2e-6)
    np.testing.assert_allclose(pdf, pdo, rtol=2e-6)
    assert np.mean(np.isclose(pdf_eval, pdf, rtol=1e-5)) >= 0.999
    np.testing.assert_allclose(pdf, T.quad_pdf(ch.tolist(), wt, d), rtol=1e-4)


def test_quadtree_device_chi_square(gpu_lib):
    """2^20 device samples binned by the leaves of the tree: chi-square against the leaf
    weights, p >= 0.01 (the quadtree sampling check of the reference's sampling tests)."""
    from scipy import stats
    from naivetrace_b200.algo import quadtree_sample_batch
    ch, wt = _quad_fixture(seed=31)
    n = 1 << 20
    u = np.random.default_rng(6).random((n, 2)).astype(np.float32)
    d, _, _ = quadtree_sample_batch(ch, wt, u)
    child = ch.tolist()
    leaves = [k for k in range(len(child)) if child[k][0] < 0]
    index = {k: i for i, k in enumerate(leaves)}
    uv = T.dir_to_square(d)
    counts = np.zeros(len(leaves))
    for p in uv:
        counts[index[T.quad_leaf(child, p)[0]]] += 1
    exp = wt[leaves].astype(np.float64) / float(wt[0]) * n
    keep = exp > 5
    e = exp[keep] * counts[keep].sum() / exp[keep].sum()
    assert stats.chisquare(counts[keep], e).pvalue >= 0.01


def test_quadtree_rounds_and_cells(gpu_lib):
    """Training rounds with quadtrees: cells multiply, every cell's tree is well formed
    (children after parents, inner weights the sums of their children, positive root)."""
    scene = scenes.guiding_room(96, 54)
    g = GpuContext(scene, make_params(max_ray_depth=12))
    g.set_guiding(True, 1, method=abi.GUIDE_TREE, tree_subdivision=100, seed=3,
                  tree_distribution=abi.TREE_QUADTREE)
    for k in range(4):
        g.render(8, seed=1 + k)
    info = g.tree_info()
    assert info["rounds"] == 4 and info["cells"] > 1
    for c in range(info["cells"]):
        ch, w = g.tree_quadtree(c)
        assert len(ch) >= 1 and w[0] > 0 and np.all(np.isfinite(w))
        for k in range(len(ch)):
            if ch[k, 0] >= 0:
                assert np.all(ch[k] > k) and np.all(ch[k] < len(ch))
                assert w[k] == pytest.approx(float(w[ch[k]].astype(np.float64).sum()), rel=1e-5)
    assert g.stats()["error_flags"] == 0


@pytest.mark.parametrize("name,train_during", [("cornell_box", True), ("guiding_room", False),
                                               ("cornell_box_medium", False)])
def test_quadtree_guided_render_unbiased(gpu_lib, name, train_during):
    """Quadtree-guided against plain renders: tile means within the Bonferroni bound of
    assert_tiles_agree, with the trees trained between the passes or frozen."""
    xres, yres, tile = (64, 64, 16) if name != "guiding_room" else (96, 54, 18)
    scene = getattr(scenes, name)(xres, yres)
    p = make_params(max_ray_depth=10 if name != "guiding_room" else 12)
    plain = GpuContext(scene, p)
    guided = GpuContext(scene, p)
    kw = dict(method=abi.GUIDE_TREE, tree_subdivision=100, seed=5, tree_distribution=abi.TREE_QUADTREE)
    guided.set_guiding(True, 1, **kw)
    for k in range(6):
        guided.render(4, seed=900 + k)
    if not train_during:
        guided.set_guiding(True, 0, **kw)
    K = 32  # batches per side: the room's batch means are skewed, and 16 left the t tails too light
    spp = 16 if name != "guiding_room" else 64
    tp = _batches(plain, K, spp, 100, xres, yres, tile)
    tg = _batches(guided, K, spp, 300, xres, yres, tile)
    assert_tiles_agree(tp, tg)
    assert guided.stats()["error_flags"] == 0
