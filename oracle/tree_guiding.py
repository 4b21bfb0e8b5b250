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
