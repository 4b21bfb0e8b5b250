// Quadtree directional distribution of the tree guider (layout and operations in
// tt_quadtree.h).  Host code: the trees are refitted once per training round, per cell.
#include "tt_quadtree.h"

#include <cmath>
#include <limits>
#include <numeric>

namespace tt {

namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kMinSampleCount = 2.0;    // min_sample_count (path_guiding.hxx:313)
constexpr double kGoodSampleCount = 100.0; // good_sample_count (:314)
// LargeFloat (vec3f.hxx:23) and safe_error_number (path_guiding.hxx:199): the error of a
// node with fewer than two records.
constexpr double kLargeFloat = (double)(std::numeric_limits<float>::max() / 16.f);
constexpr double kSafeError = 0.01 * kLargeFloat * 1.52587890625e-05;  // 0.25^8

struct Square {
  float lo[2] = {0.f, 0.f}, hi[2] = {1.f, 1.f};
  float cu() const { return 0.5f * (lo[0] + hi[0]); }
  float cv() const { return 0.5f * (lo[1] + hi[1]); }
  int quadrant(float u, float v) const { return (u < cu() ? 0 : 1) | (v < cv() ? 0 : 2); }
  Square child(int q) const {
    Square s = *this;
    const float c0 = cu(), c1 = cv();
    if (q & 1) s.lo[0] = c0; else s.hi[0] = c0;
    if (q & 2) s.lo[1] = c1; else s.hi[1] = c1;
    return s;
  }
};

// The error of a node's mean weight: sqrt(sum of squared deviations) / (count - 1), or
// `fill` below `min_count` records (SoaOnlineVariance::MeanErr, sampler.hxx:510-514).
double mean_err(const QuadStats& s, double fill, double min_count) {
  return (double)s.n >= min_count ? std::sqrt(s.sqdev) / (double)(s.n - 1) : fill;
}

}  // namespace

void dir_to_square(const float d[3], float uv[2]) {
  const double v = ((double)d[2] + 1.0) * 0.5;
  const double phi = std::atan2((double)d[1], (double)d[0]);
  uv[0] = (float)((phi / kPiD + 1.0) * 0.5);
  uv[1] = (float)v;
}

void square_to_dir(const float uv[2], float d[3]) {
  const double z = (double)uv[1] * 2.0 - 1.0;
  const double rho = std::sqrt(std::max(0.0, 1.0 - z * z));
  const double phi = ((double)uv[0] * 2.0 - 1.0) * kPiD;
  d[0] = (float)(rho * std::cos(phi));
  d[1] = (float)(rho * std::sin(phi));
  d[2] = (float)z;
}

void QuadDist::push(float u, float v, float w) {
  int node = 0;
  Square sq;
  for (;;) {
    stats[node].add((double)w);
    if (is_leaf(node)) break;
    const int q = sq.quadrant(u, v);
    node = child[node][q];
    sq = sq.child(q);
  }
}

void QuadDist::propagate(int node) {
  if (is_leaf(node)) return;
  float s = 0.f;
  for (int q = 0; q < 4; ++q) {
    propagate(child[node][q]);
    s += probs[child[node][q]];
  }
  probs[node] = s;
}

int QuadDist::leaf_depth(float u, float v) const {
  int node = 0, depth = 0;
  Square sq;
  while (!is_leaf(node)) {
    const int q = sq.quadrant(u, v);
    node = child[node][q];
    sq = sq.child(q);
    ++depth;
  }
  return depth;
}

void QuadDist::initial_fit(const float* uv, const float* w, int n) {
  double total = 0.0;
  for (int i = 0; i < n; ++i) total += (double)w[i];
  const double threshold = 0.1 * total;
  child.clear();
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  // Depth-first: a node is allocated before its children, children in quadrant order.
  struct Builder {
    QuadDist* q;
    const float* uv;
    const float* w;
    double threshold;
    int build(const std::vector<int>& ids, const Square& sq, int depth) {
      double sum = 0.0;
      for (int i : ids) sum += (double)w[i];
      const int node = (int)q->child.size();
      q->child.push_back({-1, -1, -1, -1});
      if (sum > threshold && depth < kQuadMaxDepth) {
        std::vector<int> part[4];
        for (int i : ids) part[sq.quadrant(uv[2 * i], uv[2 * i + 1])].push_back(i);
        std::array<int, 4> c;
        for (int k = 0; k < 4; ++k) c[k] = build(part[k], sq.child(k), depth + 1);
        q->child[node] = c;
      }
      return node;
    }
  } b{this, uv, w, threshold};
  b.build(idx, Square{}, 1);
  stats.assign(child.size(), QuadStats{});
  probs.assign(child.size(), 0.f);
  prior.assign(child.size(), 0.f);
  for (int i = 0; i < n; ++i) push(uv[2 * i], uv[2 * i + 1], w[i]);
}

void QuadDist::bake() {
  const double root_n = (double)stats[0].n;
  if (!(root_n > 0.0)) return;
  for (int i = 0; i < num_nodes(); ++i) probs[i] = (float)((double)stats[i].n / root_n * stats[i].mean);
  prior = probs;
  propagate(0);
}

void QuadDist::incremental_fit(const float* uv, const float* w, int n, int sub_round) {
  for (int i = 0; i < n; ++i) push(uv[2 * i], uv[2 * i + 1], w[i]);
  const double root_n = (double)stats[0].n;
  if (!(root_n > 0.0)) return;
  const double total_flux = stats[0].mean;  // relative count 1 at the root
  const double explore = std::log((double)std::max(1, sub_round));
  for (int i = 0; i < num_nodes(); ++i) {
    const QuadStats& s = stats[i];
    const double rel = (double)s.n / root_n;
    const double mean = rel * s.mean, err = rel * mean_err(s, kLargeFloat, kMinSampleCount);
    const double mix = kGoodSampleCount / (kGoodSampleCount + std::max(0.0, (double)s.n - kMinSampleCount));
    const double p = (double)prior[i] * mix + (mix < 1.0 ? (mean + err) * (1.0 - mix) : 0.0);
    probs[i] = (float)p + (float)(total_flux * std::sqrt(explore / ((double)s.n + 1.0)));
  }
  propagate(0);
}

bool QuadDist::update_and_bake() {
  if (stats[0].n <= 10) return false;
  const double root_n = (double)stats[0].n;
  const int old_n = num_nodes();
  std::vector<double> old_rel(old_n);
  std::vector<float> old_flux(old_n);
  for (int i = 0; i < old_n; ++i) {
    old_rel[i] = (double)stats[i].n / root_n;
    old_flux[i] = (float)(old_rel[i] * stats[i].mean);
  }
  const float threshold = 0.05f * old_flux[0];
  // TreeAdaptor (path_guiding_quadtree.hxx:200-300): a node whose flux exceeds the threshold
  // is kept split (or a leaf split, its flux shared evenly by the quadrants, down to the
  // threshold); a node at or below it becomes a leaf.
  struct Map {
    int old;
    float frac;  // edge length relative to the old node
  };
  std::vector<std::array<int, 4>> nchild;
  std::vector<Map> map;
  struct Adaptor {
    const QuadDist* q;
    const std::vector<float>* flux;
    float threshold;
    std::vector<std::array<int, 4>>* nchild;
    std::vector<Map>* map;
    int alloc(Map m) {
      nchild->push_back({-1, -1, -1, -1});
      map->push_back(m);
      return (int)nchild->size() - 1;
    }
    int split_leaf(float weight, int depth, Map m) {
      if (weight < threshold || depth >= kQuadMaxDepth) return alloc(m);
      const int b = alloc(m);
      std::array<int, 4> c;
      for (int k = 0; k < 4; ++k) c[k] = split_leaf(weight * 0.25f, depth + 1, Map{m.old, 0.5f * m.frac});
      (*nchild)[b] = c;
      return b;
    }
    int adapt(int node, int depth) {
      const float weight = (*flux)[node];
      if (depth < kQuadMaxDepth && weight > threshold) {
        if (q->is_leaf(node)) return split_leaf(weight, depth, Map{node, 1.f});
        const int b = alloc(Map{node, 1.f});
        std::array<int, 4> c;
        for (int k = 0; k < 4; ++k) c[k] = adapt(q->child[node][k], depth + 1);
        (*nchild)[b] = c;
        return b;
      }
      return alloc(Map{node, 1.f});
    }
  } ad{this, &old_flux, threshold, &nchild, &map};
  ad.adapt(0, 1);
  const int nn = (int)nchild.size();
  std::vector<QuadStats> nstats(nn);
  std::vector<float> nprior(nn), nprobs(nn);
  std::vector<double> rel(nn);
  for (int i = 0; i < nn; ++i) {
    const float scale = map[i].frac * map[i].frac;
    QuadStats s = stats[map[i].old];
    s.n = (int64_t)((float)s.n * scale);  // CountsMultiplied: a long scaled by a float
    s.sqdev *= (double)scale;
    nstats[i] = s;
    nprior[i] = scale * probs[map[i].old];
    rel[i] = (double)scale * old_rel[map[i].old];
  }
  for (int i = 0; i < nn; ++i) {
    const QuadStats& s = nstats[i];
    const double mix = kGoodSampleCount / (kGoodSampleCount + std::max(0.0, (double)s.n - kMinSampleCount));
    const double mean = rel[i] * s.mean, err = rel[i] * mean_err(s, kSafeError, kMinSampleCount);
    nprobs[i] = (float)((double)nprior[i] * mix + (mean + err) * (1.0 - mix));
  }
  child = std::move(nchild);
  probs = std::move(nprobs);
  propagate(0);
  prior = probs;
  stats.assign(child.size(), QuadStats{});
  return true;
}

void PointCov::add(const float p[3]) {
  n += 1.0;
  double d[3], e[3];
  for (int a = 0; a < 3; ++a) {
    d[a] = (double)p[a] - mean[a];
    mean[a] += d[a] / n;
    e[a] = (double)p[a] - mean[a];
  }
  m2[0] += d[0] * e[0];
  m2[1] += d[1] * e[1];
  m2[2] += d[2] * e[2];
  m2[3] += d[0] * e[1];
  m2[4] += d[0] * e[2];
  m2[5] += d[1] * e[2];
}

void PointCov::frame(double F[9]) const {
  // Covariance (divided by n, as OnlineCovariance::Cov), then cyclic Jacobi rotations until
  // the off-diagonal part vanishes.
  double A[3][3] = {{m2[0], m2[3], m2[4]}, {m2[3], m2[1], m2[5]}, {m2[4], m2[5], m2[2]}};
  const double inv = n > 0.0 ? 1.0 / n : 0.0;
  for (auto& row : A)
    for (double& x : row) x *= inv;
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    if (off < 1e-30) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (std::fabs(A[p][q]) < 1e-300) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A := A J (columns p, q)
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {  // A := J^T A (rows p, q)
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {  // V := V J
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  for (int k = 0; k < 3; ++k) {
    const double sd = std::sqrt(std::max(A[k][k], 1e-12));
    for (int a = 0; a < 3; ++a) F[3 * a + k] = V[a][k] * sd;
  }
}

void filter_record(const QuadDist& q, const double F[9], const double r[5], const float pos[3], const float wi[3],
                   float pos_out[3], float wi_out[3]) {
  for (int a = 0; a < 3; ++a) {
    double d = 0.0;
    for (int k = 0; k < 3; ++k) d += F[3 * a + k] * (2.0 * r[k] - 1.0);
    pos_out[a] = (float)((double)pos[a] + 3.0 * d);
  }
  float uv[2];
  dir_to_square(wi, uv);
  const double footprint = 0.5 * std::ldexp(1.0, -q.leaf_depth(uv[0], uv[1])) * 3.5449077018110318;
  // ToUniformSphereSection (sampler.cxx:55-65) about +z, then turned onto wi.
  const double z = 1.0 - r[4] * (1.0 - std::cos(footprint));
  const double sr = std::sqrt(std::max(0.0, 1.0 - z * z)), phi = 2.0 * kPiD * r[3];
  const double lx = std::cos(phi) * sr, ly = std::sin(phi) * sr;
  // Orthonormal frame with wi as its third axis (Duff et al. 2017).
  const double nx = wi[0], ny = wi[1], nz = wi[2];
  const double sign = std::copysign(1.0, nz);
  const double a = -1.0 / (sign + nz), b = nx * ny * a;
  const double t[3] = {1.0 + sign * nx * nx * a, sign * b, -sign * nx};
  const double bt[3] = {b, sign + ny * ny * a, -ny};
  double o[3];
  for (int k = 0; k < 3; ++k) o[k] = t[k] * lx + bt[k] * ly + (k == 0 ? nx : (k == 1 ? ny : nz)) * z;
  const double l = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
  for (int k = 0; k < 3; ++k) wi_out[k] = (float)(o[k] / l);
}

}  // namespace tt
