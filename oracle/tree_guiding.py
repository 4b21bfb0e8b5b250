"""CPU oracle of the tree guider (test infrastructure only): the initial kd-tree build and
the incremental EM of one cell's 8-lobe vMF mixture, in float64.

- Builder (path_guiding_tree.hxx:306-440): recursive; a leaf when fewer than 2 x min_points
  remain or the depth reaches 20; otherwise split at the median (the element at index n/2 in
  sorted order) along the axis of largest extent, unless a side would keep fewer than
  min_points.  Cells are numbered in the order leaves are created (left first).
- Lookup (Tree::Lookup, :129-150): left when the coordinate is below the split.
- Incremental fit (vmf_fitting::incremental::Fit / UpdateStatistics / MaximizationStep,
  distribution_mixture_models.cxx:279-388) with the parameters of
  RadianceDistributionLearned::Parameters (path_guiding.cxx:60-76): prior strength
  max(1, 0.01 x max record count), a maximisation step every 10 x strength records, the
  fixed prior InitializeForUnitSphere<8> (distribution_mixture_models.cxx:174-189).
"""
import math

import numpy as np

LOBES = 8
PRIOR_MU = np.array([
    [0.66778004, 0.73539025, 0.11519922], [-0.9836298, -0.008926501, 0.1799797],
    [-0.14629413, -0.7809748, 0.60718733], [0.49043104, 0.04368747, -0.87038434],
    [-0.10088497, 0.42765132, 0.8982965], [-0.35999632, -0.6945797, -0.62286574],
    [-0.43178025, 0.7588791, -0.48751223], [0.860208, -0.47938251, 0.17388113]], np.float64)
PRIOR_KAPPA = 2.0
KAPPA_MIN, KAPPA_MAX = 1e-4, 40.0
EPS = 1e-38
MAX_DEPTH = 20


def prior_mixture():
    """(weights[8], means[8, 3], concentrations[8])."""
    return np.full(LOBES, 1.0 / LOBES), PRIOR_MU.copy(), np.full(LOBES, PRIOR_KAPPA)


def pack(w, mu, k):
    return np.concatenate([w, mu.reshape(-1), k]).astype(np.float64)


def unpack(m40):
    m40 = np.asarray(m40, np.float64)
    return m40[:8].copy(), m40[8:32].reshape(8, 3).copy(), m40[32:40].copy()


def vmf_pdf(mu, k, x):
    """Density of each lobe at directions x: (n, 8)."""
    c = k / (2 * np.pi * (1 - np.exp(-2 * k)))
    return c[None, :] * np.exp(k[None, :] * (x @ mu.T - 1.0))


def mixture_pdf(w, mu, k, x):
    return vmf_pdf(mu, k, x) @ w


def mean_cosine_to_conc(r):
    r = np.minimum(r, 1.0 - 1e-6)
    return r * (3 - r * r) / (1 - r * r)


class CellFit:
    """Mixture and fit state of one cell (the accumulators of incremental::Data)."""

    def __init__(self):
        self.w, self.mu, self.k = prior_mixture()
        self.avg_w = 0.0
        self.n_w = 0
        self.max_samples = 0
        self.pend_n = 0
        self.pend_wr = np.zeros(LOBES)
        self.pend_wrx = np.zeros((LOBES, 3))

    def fit(self, dirs, weights, batch_iters=0):
        """Fits records in the order given (one round).  batch_iters > 0: that many
        maximisation steps, each over all the records (the incremental statistics unused)."""
        dirs = np.asarray(dirs, np.float64).reshape(-1, 3)
        weights = np.asarray(weights, np.float64)
        n = len(dirs)
        self.max_samples = max(self.max_samples, n)
        ps = max(1.0, 0.01 * self.max_samples)
        batch = batch_iters > 0
        if batch:
            self.pend_n = 0
            self.pend_wr = np.zeros(LOBES)
            self.pend_wrx = np.zeros((LOBES, 3))
        chunk = n if batch else max(1, int(ps)) * 10
        i = 0
        it = 0
        while i < n:
            seg = min(chunk - self.pend_n, n - i)
            x, wt = dirs[i:i + seg], weights[i:i + seg]
            resp = self.w[None, :] * vmf_pdf(self.mu, self.k, x) + EPS
            resp /= resp.sum(axis=1, keepdims=True)
            wr = wt[:, None] * resp
            self.pend_wr += wr.sum(axis=0)
            self.pend_wrx += wr.T @ x
            if it == 0 or not batch:
                self.avg_w = (self.avg_w * self.n_w + wt.sum()) / (self.n_w + seg)
                self.n_w += seg
            self.pend_n += seg
            i += seg
            if self.pend_n < chunk:
                break
            N = float(chunk)
            mwr = self.pend_wr / N
            mwrx = self.pend_wrx / N
            w = (ps - 1) / N * (1.0 / LOBES) + mwr / (self.avg_w + EPS) + EPS
            dim = self.avg_w * ps / N
            mu = (dim * PRIOR_MU + mwrx) / (dim + mwr + EPS)[:, None]
            nrm = np.linalg.norm(mu, axis=1)
            mu = np.where((nrm > EPS)[:, None], mu / np.maximum(nrm, 1e-300)[:, None], np.array([1.0, 0.0, 0.0]))
            mcos = np.linalg.norm(mwrx, axis=1) / (mwr + EPS)
            da = ps / N
            k = (PRIOR_KAPPA * da + mean_cosine_to_conc(mcos)) / (da + 1)
            self.w = w / w.sum()
            self.mu = mu
            self.k = np.clip(k, KAPPA_MIN, KAPPA_MAX)
            self.pend_n = 0
            self.pend_wr = np.zeros(LOBES)
            self.pend_wrx = np.zeros((LOBES, 3))
            it += 1
            if batch and it < batch_iters:
                i = 0
        return self


def build_kdtree(points, min_points=100, max_depth=MAX_DEPTH):
    """Returns (nodes, cell_of_point); a node is (split, axis, left, right) with a child < 0
    meaning leaf ~cell."""
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    nodes = []
    cell_of = np.zeros(len(pts), np.int64)
    ncells = [0]

    def leaf(idx):
        c = ncells[0]
        ncells[0] += 1
        cell_of[idx] = c
        return ~c

    def rec(idx, depth):
        n = len(idx)
        if n < 2 * min_points or depth >= max_depth:
            return leaf(idx)
        p = pts[idx]
        axis = int(np.argmax(p.max(axis=0) - p.min(axis=0)))
        order = np.argsort(p[:, axis], kind="stable")
        mid = n // 2
        pos = float(p[order[mid], axis])
        if mid < min_points or n - mid < min_points:
            return leaf(idx)
        node = len(nodes)
        nodes.append([pos, axis, 0, 0])
        left = rec(idx[order[:mid]], depth + 1)
        right = rec(idx[order[mid:]], depth + 1)
        nodes[node][2], nodes[node][3] = left, right
        return node

    rec(np.arange(len(pts)), 1)
    return nodes, cell_of


def lookup(nodes, p):
    ref = 0 if nodes else ~0
    while ref >= 0:
        split, axis, left, right = nodes[ref]
        ref = left if p[axis] < np.float32(split) else right
    return ~ref


# ---- Quadtree radiance distribution ---------------------------------------------------
# The reference's active directional distribution (quadtree_radiance_distribution,
# path_guiding.hxx:190-340, path_guiding.cxx:108-310; tree, builder, adaptor and sampler in
# path_guiding_quadtree.hxx / .cxx), restated with the arithmetic types the library uses:
# record weights and statistics in float64 (Welford updates in record order), sampling
# weights in float32 (inner nodes the float32 sums of their children in quadrant order).
# Quadrants: 0 = (u < c, v < c), 1 = (u >= c, v < c), 2 = (u < c, v >= c), 3 = (u >= c, v >= c);
# nodes numbered depth first, a parent before its children.

QUAD_MAX_DEPTH = 8                     # path_guiding_quadtree.hxx:22
MIN_SAMPLE_COUNT, GOOD_SAMPLE_COUNT = 2.0, 100.0   # path_guiding.hxx:313-314
LARGE_FLOAT = float(np.finfo(np.float32).max / np.float32(16.0))   # vec3f.hxx:23
SAFE_ERROR = 0.01 * LARGE_FLOAT * 0.25 ** QUAD_MAX_DEPTH           # path_guiding.hxx:199
F32 = np.float32


def dir_to_square(d):
    """MapSphereToTree (path_guiding.cxx:112-118): float32 (n, 2) from unit directions."""
    d = np.asarray(d, np.float32).astype(np.float64).reshape(-1, 3)
    v = (d[:, 2] + 1.0) * 0.5
    u = (np.arctan2(d[:, 1], d[:, 0]) / np.pi + 1.0) * 0.5
    return np.stack([u, v], axis=1).astype(np.float32)


def square_to_dir(uv):
    """MapTreeToSphere (path_guiding.cxx:120-128), float64."""
    uv = np.asarray(uv, np.float64).reshape(-1, 2)
    z = uv[:, 1] * 2.0 - 1.0
    rho = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = (uv[:, 0] * 2.0 - 1.0) * np.pi
    return np.stack([rho * np.cos(phi), rho * np.sin(phi), z], axis=1)


def _quadrant(u, v, lo, hi):
    c0, c1 = 0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])   # dyadic: exact in float32 too
    return (0 if u < c0 else 1) | (0 if v < c1 else 2)


def _child_square(lo, hi, q):
    c0, c1 = 0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])
    lo, hi = list(lo), list(hi)
    if q & 1:
        lo[0] = c0
    else:
        hi[0] = c0
    if q & 2:
        lo[1] = c1
    else:
        hi[1] = c1
    return lo, hi


def adapt_tree(child, weights, fraction):
    """TreeAdaptor (path_guiding_quadtree.hxx:200-300) over node weights (float32): a node
    whose weight exceeds fraction x the root's stays split, a leaf above it is split with its
    weight shared evenly by the quadrants (SplitLeaf stops below the threshold), a node at or
    below it becomes a leaf; depth at most 8.  Returns the new children, per new node (old
    node, edge length relative to it) and the new nodes' weights."""
    weights = [F32(x) for x in weights]
    thr = F32(F32(fraction) * weights[0])
    nchild, mp, nw = [], [], []

    def alloc(old, frac, weight):
        nchild.append([-1, -1, -1, -1])
        mp.append((old, frac))
        nw.append(weight)
        return len(nchild) - 1

    def split_leaf(weight, depth, old, frac):
        if weight < thr or depth >= QUAD_MAX_DEPTH:
            return alloc(old, frac, weight)
        b = alloc(old, frac, weight)
        nchild[b] = [split_leaf(F32(weight * F32(0.25)), depth + 1, old, F32(F32(0.5) * frac)) for _ in range(4)]
        return b

    def adapt(k, depth):
        weight = weights[k]
        if depth < QUAD_MAX_DEPTH and weight > thr:
            if child[k][0] < 0:
                return split_leaf(weight, depth, k, F32(1.0))
            b = alloc(k, F32(1.0), weight)
            nchild[b] = [adapt(c, depth + 1) for c in child[k]]
            return b
        return alloc(k, F32(1.0), weight)

    adapt(0, 1)
    return nchild, mp, nw


class Quad:
    """One cell's quadtree: children, learned statistics (mean, sqdev, n), sampling weights
    and prior."""

    def __init__(self):
        self.child = [[-1, -1, -1, -1]]
        self.stats = [[0.0, 0.0, 0]]
        self.probs = np.ones(1, np.float32)
        self.prior = np.ones(1, np.float32)

    def leaf(self, k):
        return self.child[k][0] < 0

    def _push(self, u, v, w):
        k, lo, hi = 0, [0.0, 0.0], [1.0, 1.0]
        while True:
            s = self.stats[k]
            s[2] += 1
            dlt = w - s[0]
            s[0] += dlt / s[2]
            s[1] += dlt * (w - s[0])
            if self.leaf(k):
                return
            q = _quadrant(u, v, lo, hi)
            k = self.child[k][q]
            lo, hi = _child_square(lo, hi, q)

    def _propagate(self, k):
        if self.leaf(k):
            return
        s = F32(0.0)
        for c in self.child[k]:
            self._propagate(c)
            s = F32(s + self.probs[c])
        self.probs[k] = s

    def initial_fit(self, uv, w, fraction=0.1):
        """InitialFit (path_guiding.cxx:203-217): Builder (path_guiding_quadtree.cxx:31-60)
        splitting while a node's weight exceeds `fraction` (InitialFit: 0.1) of the total
        and the depth is below 8, then every record pushed."""
        uv = np.asarray(uv, np.float32).reshape(-1, 2)
        w = np.asarray(w, np.float32).reshape(-1)
        thr = fraction * sum(float(x) for x in w)
        self.child = []

        def build(ids, lo, hi, depth):
            tot = 0.0
            for i in ids:
                tot += float(w[i])
            k = len(self.child)
            self.child.append([-1, -1, -1, -1])
            if tot > thr and depth < QUAD_MAX_DEPTH:
                parts = [[], [], [], []]
                for i in ids:
                    parts[_quadrant(uv[i, 0], uv[i, 1], lo, hi)].append(i)
                kids = []
                for q in range(4):
                    clo, chi = _child_square(lo, hi, q)
                    kids.append(build(parts[q], clo, chi, depth + 1))
                self.child[k] = kids
            return k

        build(list(range(len(w))), [0.0, 0.0], [1.0, 1.0], 1)
        n = len(self.child)
        self.stats = [[0.0, 0.0, 0] for _ in range(n)]
        self.probs = np.zeros(n, np.float32)
        self.prior = np.zeros(n, np.float32)
        for i in range(len(w)):
            self._push(uv[i, 0], uv[i, 1], float(w[i]))

    def bake(self):
        """Bake (path_guiding.cxx:274-288)."""
        rn = float(self.stats[0][2])
        if not rn > 0:
            return
        for k, (m, _, c) in enumerate(self.stats):
            self.probs[k] = F32(c / rn * m)
        self.prior = self.probs.copy()
        self._propagate(0)

    @staticmethod
    def _mean_err(s, fill):
        return math.sqrt(s[1]) / (s[2] - 1) if s[2] >= MIN_SAMPLE_COUNT else fill

    def incremental_fit(self, uv, w, sub_round=1):
        """IncrementalFit (path_guiding.cxx:172-200)."""
        uv = np.asarray(uv, np.float32)
        w = np.asarray(w, np.float32)
        for i in range(len(w)):
            self._push(uv[i, 0], uv[i, 1], float(w[i]))
        rn = float(self.stats[0][2])
        if not rn > 0:
            return
        flux = self.stats[0][0]
        explore = math.log(max(1, sub_round))
        for k, s in enumerate(self.stats):
            rel = s[2] / rn
            mean, err = rel * s[0], rel * self._mean_err(s, LARGE_FLOAT)
            mix = GOOD_SAMPLE_COUNT / (GOOD_SAMPLE_COUNT + max(0.0, s[2] - MIN_SAMPLE_COUNT))
            p = float(self.prior[k]) * mix + ((mean + err) * (1.0 - mix) if mix < 1.0 else 0.0)
            self.probs[k] = F32(F32(p) + F32(flux * math.sqrt(explore / (s[2] + 1.0))))
        self._propagate(0)

    def update_and_bake(self):
        """IterationUpdateAndBake (path_guiding.cxx:221-271) with TreeAdaptor
        (path_guiding_quadtree.hxx:200-300)."""
        if self.stats[0][2] <= 10:
            return False
        rn = float(self.stats[0][2])
        old_rel = [s[2] / rn for s in self.stats]
        old_flux = [F32(r * s[0]) for r, s in zip(old_rel, self.stats)]
        nchild, mp, _ = adapt_tree(self.child, old_flux, F32(0.05))
        nn = len(nchild)
        nstats, nprior, rel = [], np.zeros(nn, np.float32), []
        for i, (old, frac) in enumerate(mp):
            scale = F32(frac * frac)
            m, sq, c = self.stats[old]
            nstats.append([m, sq * float(scale), int(F32(c) * scale)])
            nprior[i] = F32(scale * self.probs[old])
            rel.append(float(scale) * old_rel[old])
        probs = np.zeros(nn, np.float32)
        for i, s in enumerate(nstats):
            mix = GOOD_SAMPLE_COUNT / (GOOD_SAMPLE_COUNT + max(0.0, s[2] - MIN_SAMPLE_COUNT))
            mean, err = rel[i] * s[0], rel[i] * self._mean_err(s, SAFE_ERROR)
            probs[i] = F32(float(nprior[i]) * mix + (mean + err) * (1.0 - mix))
        self.child = nchild
        self.probs = probs
        self._propagate(0)
        self.prior = self.probs.copy()
        self.stats = [[0.0, 0.0, 0] for _ in range(nn)]
        return True


def quad_sample(child, probs, u0, u1):
    """quadtree::Sample (path_guiding_quadtree.cxx:178-244) in float32 as the device does it:
    returns the point in the unit square, the density per unit square and the leaf."""
    lt1, eps = F32(np.nextafter(F32(1), F32(0))), F32(np.finfo(np.float32).eps)
    u0, u1 = min(F32(u0), lt1), min(F32(u1), lt1)
    lo, hi, k = [F32(0), F32(0)], [F32(1), F32(1)], 0
    for _ in range(16):
        c = child[k]
        if c[0] < 0:
            break
        w = [F32(probs[x]) for x in c]
        wl, wr = F32(w[0] + w[2]), F32(w[1] + w[3])
        s0 = F32(u0 * F32(wl + wr))
        q = 0 if s0 < wl else 1
        u0 = F32(s0 / F32(wl + eps)) if s0 < wl else F32(F32(s0 - wl) / F32(wr + eps))
        wb, wt = (w[1], w[3]) if q else (w[0], w[2])
        s1 = F32(u1 * F32(wb + wt))
        q |= 0 if s1 < wb else 2
        u1 = F32(s1 / F32(wb + eps)) if s1 < wb else F32(F32(s1 - wb) / F32(wt + eps))
        u0, u1 = min(u0, lt1), min(u1, lt1)
        lo, hi = _child_square(lo, hi, q)
        lo, hi = [F32(x) for x in lo], [F32(x) for x in hi]
        k = c[q]
    a0, a1 = F32(hi[0] - lo[0]), F32(hi[1] - lo[1])
    pdf = F32(F32(probs[k]) / F32(F32(F32(probs[0]) * a0) * a1))
    pu = max(min(F32(F32(a0 * u0) + lo[0]), F32(hi[0] * lt1)), lo[0])
    pv = max(min(F32(F32(a1 * u1) + lo[1]), F32(hi[1] * lt1)), lo[1])
    return (pu, pv), pdf, k


def quad_leaf(child, uv):
    """The leaf holding a point of the unit square and its area."""
    k, lo, hi = 0, [0.0, 0.0], [1.0, 1.0]
    while child[k][0] >= 0:
        q = _quadrant(uv[0], uv[1], lo, hi)
        lo, hi = _child_square(lo, hi, q)
        k = child[k][q]
    return k, (hi[0] - lo[0]) * (hi[1] - lo[1])


def quad_pdf(child, probs, d):
    """Density per unit solid angle of unit directions d under the quadtree (Pdf,
    path_guiding_quadtree.cxx:247-261, over the map's Jacobian 4 pi)."""
    out = []
    for uv in dir_to_square(d):
        k, area = quad_leaf(child, uv)
        out.append(float(probs[k]) / (float(probs[0]) * area) / (4.0 * np.pi))
    return np.array(out)
