"""The learned guider on the GPU against the CPU oracle (oracle/guiding.py), and guided
rendering against plain rendering.

1. Feature encoding, forward pass and loss gradient through the C ABI against the oracle
   that rounds to bfloat16 where the GPU stores bfloat16 (differences: accumulation order
   only), and against the float64 oracle (the size of the bfloat16 error).
2. One Adam step of the device optimiser against the oracle's Adam on the same gradient.
3. Training on synthetic records lowers the loss and concentrates the mixture.
4. Training records collected by a render: layout, positivity, the fraction that carries
   light.
5. Guided rendering is unbiased: tile means of guided renders (network training between
   passes, and frozen) agree with plain renders within a z-test, with and without media.
6. The guided RenderingAlgo schedule (training sweeps, then frozen passes).
"""
import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext, GpuGuidedPathTracer
from naivetrace_b200.scene import make_params
from oracle import guiding as G
from oracle.oracle import combine

pytestmark = pytest.mark.gpu


def _ctx(scene=None):
    scene = scene if scene is not None else scenes.cornell_box(16, 16)
    return GpuContext(scene, make_params(max_ray_depth=10))


def _params(seed=3, bias=0.05):
    p = G.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    for l in range(G.N_LAYERS):
        o = G.layer_out(l)
        p[G.b_offset(l):G.b_offset(l) + o] = rng.normal(0, bias, o)
    return p.astype(np.float32)


def test_num_params(gpu_lib):
    assert gpu_lib.tt_guide_num_params() == G.N_PARAMS


def test_features_match_oracle(gpu_lib):
    g = _ctx()
    rec = G.random_records(4096, seed=2)
    xg = g.guide_features(rec[:, 0:9])
    xo = G.record_features(rec)
    diff = xg != xo
    # The device's hardware sine (absolute error about 1e-6) may round to a neighbouring
    # bfloat16 value.
    assert diff.mean() < 2e-3, diff.mean()
    # At most one bfloat16 step apart (8 significant bits), or within the sine's error.
    assert np.all(np.abs(xg - xo)[diff] <= 2 ** -7 * np.abs(xo)[diff] + 4e-6)


def test_forward_matches_oracle(gpu_lib):
    g = _ctx()
    p = _params()
    g.guide_set_params(p)
    assert np.array_equal(g.guide_params(), p)
    rec = G.random_records(3000, seed=4)       # not a multiple of the 16-row tile
    x = G.record_features(rec)
    og = g.guide_forward(x)
    oo, _, _ = G.forward(p, x, True)
    err = np.linalg.norm(og - oo) / np.linalg.norm(oo)
    assert err < 5e-3, err
    assert np.abs(og - oo).max() < 0.05 * np.abs(oo).max()
    of, _, _ = G.forward(p, x, False)
    assert np.linalg.norm(og - of) / np.linalg.norm(of) < 3e-2


@pytest.mark.parametrize("n", [3000, 100000])
def test_forward_tcgen05_matches(gpu_lib, n):
    """The tensor-core forward (128-row tiles, ragged last tile; 100000 rows give more tiles
    than the resident chains) against the mma.sync forward and the oracle: both round the hidden
    activations to bfloat16 and sum in FP32, so they agree to the summation order."""
    g = _ctx()
    p = _params()
    g.guide_set_params(p)
    x = G.record_features(G.random_records(n, seed=11))
    ot = g.guide_forward(x, tcgen05=True)
    om = g.guide_forward(x)
    assert np.all(np.isfinite(ot))
    assert np.linalg.norm(ot - om) / np.linalg.norm(om) < 2e-3
    oo, _, _ = G.forward(p, x, True)
    assert np.linalg.norm(ot - oo) / np.linalg.norm(oo) < 5e-3
    assert g.stats()["error_flags"] == 0


@pytest.mark.parametrize("n", [777, 9000])
def test_gradient_matches_oracle(gpu_lib, n):
    """9000 records span 71 tiles of 128 records of the tcgen05 training kernel, the last
    one ragged."""
    g = _ctx()
    p = _params()
    g.guide_set_params(p)
    rec = G.random_records(n, seed=n)
    loss_g, grad_g = g.guide_gradient(rec)
    loss_o, grad_o = G.gradient(p, rec, bf16_round=True)
    assert abs(loss_g - loss_o) <= 2e-3 * abs(loss_o), (loss_g, loss_o)
    err = np.linalg.norm(grad_g - grad_o) / np.linalg.norm(grad_o)
    cos = grad_g @ grad_o / (np.linalg.norm(grad_g) * np.linalg.norm(grad_o))
    assert err < 3e-2 and cos > 0.999, (err, cos)
    # Per layer, so that no layer hides behind a larger one.
    for l in range(G.N_LAYERS):
        a, b = G.w_offset(l), G.b_offset(l) + G.layer_out(l)
        e = np.linalg.norm(grad_g[a:b] - grad_o[a:b]) / np.linalg.norm(grad_o[a:b])
        assert e < 5e-2, (l, e)
    # The bfloat16 network stays close to the exact float64 gradient.
    _, grad_f = G.gradient(p, rec, bf16_round=False)
    cos_f = grad_g @ grad_f / (np.linalg.norm(grad_g) * np.linalg.norm(grad_f))
    assert cos_f > 0.99, cos_f


@pytest.mark.parametrize("n", [100, 5000, 70000])
def test_weight_gradient_tcgen05_matches_mma(gpu_lib, n):
    """The training step on the tcgen05 tensor cores (one kernel: forward, backward and the
    weight and bias gradients accumulated in tensor memory, the bias gradient from a column
    of ones) against the warp-level mma.sync kernels on the same records: the same BF16
    products, summed in FP32 in another order.  Where the two sums of a hidden gradient round
    to neighbouring BF16 values (one step is 2^-8 relative) the difference travels back
    through the layers, so the bound is 2e-3 relative per layer."""
    g = _ctx()
    g.guide_set_params(_params())
    rec = G.random_records(n, seed=n + 1)
    loss_t, grad_t = g.guide_gradient(rec)
    g.set_guiding(True, 0, network=abi.GUIDE_NET_MMA)
    loss_m, grad_m = g.guide_gradient(rec)
    assert abs(loss_t - loss_m) <= 1e-5 * abs(loss_m)
    for l in range(G.N_LAYERS):
        a, b = G.w_offset(l), G.b_offset(l) + G.layer_out(l)
        e = np.linalg.norm(grad_t[a:b] - grad_m[a:b]) / np.linalg.norm(grad_m[a:b])
        assert e < 2e-3, (l, e)
    assert g.stats()["error_flags"] == 0


def _splitmix64(z):
    m = (1 << 64) - 1
    z = (z + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


@pytest.mark.parametrize("n,pool_n", [(3000, 5000), (9000, 700)])
def test_gradient_of_pool_minibatch(gpu_lib, n, pool_n):
    """The training step draws its mini-batch inside the gradient kernel: record i of the
    batch is pool[h(seed ^ h(i)) mod pool_n].  The same records gathered on the host with
    that hash give the same gradient bit for bit (the loss sum uses float atomics)."""
    g = _ctx()
    g.guide_set_params(_params())
    pool = G.random_records(pool_n, seed=pool_n)
    seed = 0x1234ABCD5678 + n
    loss_p, grad_p = g.guide_gradient_pool(pool, n, seed)
    idx = [_splitmix64(seed ^ _splitmix64(i)) % pool_n for i in range(n)]
    loss_h, grad_h = g.guide_gradient(pool[idx])
    np.testing.assert_array_equal(grad_p, grad_h)
    assert abs(loss_p - loss_h) <= 1e-5 * abs(loss_h)


def test_adam_step_matches_oracle(gpu_lib):
    g = _ctx()
    p = _params(seed=8)
    g.guide_set_params(p)
    rec = G.random_records(2048, seed=8)
    _, grad = g.guide_gradient(rec)
    g.guide_train(rec, steps=1, learning_rate=1e-3)
    p1 = g.guide_params()
    e, _, _ = G.adam(p.astype(np.float64), 0.0, 0.0, grad.astype(np.float64), 1, 1e-3)
    np.testing.assert_allclose(p1, e, atol=2e-6)


def test_training_on_gpu_lowers_loss(gpu_lib):
    g = _ctx()
    g.guide_set_params(G.init_params(2))
    rec = G.random_records(1024, seed=1)
    rec[:, 0:9] = rec[np.arange(1024) % 8, 0:9]
    L0 = G.loss(G.init_params(2).astype(np.float64), rec)
    L1 = g.guide_train(rec, steps=120, learning_rate=5e-3)
    assert L1 < L0 - 0.5, (L0, L1)
    mu = np.array([0.3, 0.5, 0.8]) / np.linalg.norm([0.3, 0.5, 0.8])
    out = g.guide_forward(G.record_features(rec[:64]))
    assert np.median(G.mixture_pdf(out, np.broadcast_to(mu, (64, 3)))) > 1.0


def test_render_records(gpu_lib):
    """Records of guided passes in the gap-lit room: normalised positions, unit vectors,
    positive finite weights (only records that carry light are kept), at most one per path;
    the pool is a ring that keeps the newest records."""
    scene = scenes.guiding_room(64, 36)
    g = GpuContext(scene, make_params(max_ray_depth=12))
    g.set_guiding(True, 2, record_pool=1 << 16, seed=3)
    g.render(16, seed=1)
    r = g.guide_records()
    assert 0 < len(r) <= 64 * 36 * 16
    assert np.all((r[:, 0:3] >= -1e-4) & (r[:, 0:3] <= 1 + 1e-4))
    for a in (3, 6, 9):
        np.testing.assert_allclose(np.linalg.norm(r[:, a:a + 3], axis=1), 1.0, atol=1e-3)
    assert np.all(r[:, 12] >= 0) and np.all(r[:, 13] > 0) and np.all(np.isfinite(r[:, 13]))
    assert len(g.guide_records()) == 0            # reading empties the pool
    # A pool smaller than one pass's yield holds exactly its capacity.
    g.set_guiding(True, 2, record_pool=64, seed=3)
    g.render(16, seed=2)
    assert len(g.guide_records()) == 64


def assert_tiles_agree(ta, tb, alpha=0.01):
    """Tile means of two sets of K independent renders (K, tiles..., 3) agree (Welch's t-test
    with a Bonferroni bound): z = |difference of the means| / sqrt(se_a^2 + se_b^2) follows
    Student's t with the Welch-Satterthwaite degrees of freedom of its tile-channel (between
    K - 1 and 2K - 2: fewer when one side's variance dominates); every tile-channel stays
    below the two-sided t quantile at alpha / T for the family of T = tiles x 3 tests, and
    the tiles with a channel beyond 3 sigma stay within the 99.9 % binomial quantile of
    their count (each tile's chance bounded by three channels' tail sum at the smallest
    degrees of freedom)."""
    from scipy import stats
    K = len(ta)
    va, vb = ta.var(0, ddof=1) / K, tb.var(0, ddof=1) / K
    se = np.sqrt(va + vb)
    z = np.abs(tb.mean(0) - ta.mean(0)) / np.maximum(se, 1e-12)
    df = np.clip((va + vb) ** 2 / np.maximum((va * va + vb * vb) / (K - 1), 1e-300), K - 1, 2 * K - 2)
    T = z.size
    bound = stats.t.isf(alpha / (2 * T), df)
    assert np.all(z < bound), (z.max(), bound.min())
    tiles = z.reshape(-1, z.shape[-1])
    p_tile = min(1.0, 3 * 2 * stats.t.sf(3.0, float(df.min())))
    kmax = stats.binom.ppf(0.999, len(tiles), p_tile)
    beyond = int(np.sum(tiles.max(axis=1) >= 3.0))
    assert beyond <= kmax, (beyond, kmax)
    return z


def tile_means(rgb, xres, yres, tile):
    a = rgb.reshape(yres, xres, 3)
    ty, tx = yres // tile, xres // tile
    return a[: ty * tile, : tx * tile].reshape(ty, tile, tx, tile, 3).mean(axis=(1, 3))


def _batches(ctx, K, spp, seed0, xres, yres, tile):
    out = []
    for k in range(K):
        ctx.clear()
        ctx.render(spp, seed=seed0 + k)
        acc, light, sppc, splat = ctx.accumulators()
        out.append(tile_means(combine(acc, light, spp, splat, ctx.npix), xres, yres, tile))
    return np.array(out)


@pytest.mark.parametrize("name,train_during", [("cornell_box", True), ("cornell_box", False),
                                               ("cornell_box_medium", False), ("guiding_room", True)])
def test_guided_render_unbiased(gpu_lib, name, train_during):
    """Tile means of guided and plain renders, K independent renders per side, agree within
    the Bonferroni bound of assert_tiles_agree."""
    xres, yres, tile = (64, 64, 16) if name != "guiding_room" else (96, 54, 18)
    scene = getattr(scenes, name)(xres, yres)
    p = make_params(max_ray_depth=10 if name != "guiding_room" else 12)
    plain = GpuContext(scene, p)
    guided = GpuContext(scene, p)
    guided.set_guiding(True, 1, learning_rate=1e-2, steps_per_pass=4, seed=5)
    for k in range(8):                       # train before the measured batches
        guided.render(4, seed=900 + k)
    st = guided.stats()
    steps_before = st["guide_steps"]
    assert st["guide_records"] > 0 and 0 < steps_before <= 32 and steps_before % 4 == 0
    assert np.isfinite(st["guide_loss"])
    if not train_during:
        guided.set_guiding(True, 0, learning_rate=1e-2, steps_per_pass=4, seed=5)
    K = 32  # batches per side: the room's batch means are skewed, and 16 left the t tails too light
    spp = 16 if name != "guiding_room" else 64
    tp = _batches(plain, K, spp, 100, xres, yres, tile)
    tg = _batches(guided, K, spp, 300, xres, yres, tile)
    steps_after = guided.stats()["guide_steps"]
    assert (steps_after > steps_before) == train_during
    assert_tiles_agree(tp, tg)
    assert guided.stats()["error_flags"] == 0


def test_guiding_gain(gpu_lib):
    """What the trained network gains: on the gap-lit room, relMSE against a 4096-spp plain
    render at 64 spp, guided (after 32 two-sample training passes) against plain.  The
    same network switched off must render like plain (no gain from anything else)."""
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

    plain = GpuContext(scene, p)
    e_plain = []
    for k in range(3):
        plain.clear()
        plain.render(64, seed=100 + k)
        e_plain.append(relmse(plain))
    g = GpuContext(scene, p)
    g.set_guiding(True, 1, learning_rate=1e-3, steps_per_pass=16, seed=7)
    for k in range(32):
        g.render(2, seed=200 + k)
    g.set_guiding(True, 0, learning_rate=1e-3, steps_per_pass=16, seed=7)
    e_guided = []
    for k in range(3):
        g.clear()
        g.render(64, seed=300 + k)
        e_guided.append(relmse(g))
    gain = np.mean(e_plain) / np.mean(e_guided)
    assert gain > 1.5, (e_plain, e_guided)
    g.set_guiding(False)
    g.clear()
    g.render(64, seed=400)
    assert 0.6 < np.mean(e_plain) / relmse(g) < 1.6


def test_guided_algo_schedule(gpu_lib):
    scene = scenes.cornell_box(32, 32)
    algo = GpuGuidedPathTracer(scene, make_params(max_ray_depth=8, max_spp=12), guide_max_spp=4,
                               steps_per_pass=2)
    calls = []
    algo.set_interrupt_callback(lambda complete: calls.append(complete))
    algo.run()
    # One initial pass, sweeps of 2 and 4 passes, then the schedule 1 + 2 + 4 + 5 = 12.
    assert calls == [True] * 7, calls
    acc, light, spp, splat = algo.ctx.accumulators()
    assert np.all(spp == 12)
    st = algo.ctx.stats()
    assert 0 < st["guide_steps"] <= 2 * (1 + 2 + 4) and st["guide_steps"] % 2 == 0
    img = algo.generate_image()
    assert img.shape == (32, 32, 3) and img.mean() > 5


def test_guided_render_tcgen05_matches_mma(gpu_lib):
    """Guided renders with the network on the tcgen05 kernel and on the mma.sync kernel,
    same weights and seeds: the two kernels give the same network outputs, so the images
    agree to the order of the floating-point accumulation."""
    scene = scenes.guiding_room(96, 54)
    g = GpuContext(scene, make_params(max_ray_depth=12))
    g.set_guiding(True, 1, seed=3, network=abi.GUIDE_NET_MMA)
    for k in range(3):
        g.render(4, seed=50 + k)
    imgs = []
    for net in (abi.GUIDE_NET_MMA, abi.GUIDE_NET_TCGEN05):
        g.set_guiding(True, 0, seed=3, network=net)
        g.clear()
        g.render(8, seed=77)
        imgs.append(g.framebuffer().astype(np.float64))
    assert g.stats()["error_flags"] == 0
    a, b = imgs
    assert np.abs(a - b).max() <= 1e-5 * max(np.abs(a).max(), 1e-6), np.abs(a - b).max()
