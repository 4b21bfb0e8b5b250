// Quadtree directional distribution of the tree guider: the reference's active radiance
// distribution (quadtree_radiance_distribution, path_guiding.hxx:190-340,
// path_guiding.cxx:108-310, tree and sampling in path_guiding_quadtree.{hxx,cxx}).
//
// Directions map to the unit square by the equal-area cylindrical map (u = phi / 2 pi + 1/2,
// v = (z + 1) / 2; MapSphereToTree, path_guiding.cxx:112-128), whose Jacobian is 4 pi.  A
// node covers a square of the unit square; its four children are the quadrants
// 0 = (u < centre, v < centre), 1 = (u >= centre, v < centre), 2 = (u < centre, v >= centre),
// 3 = (u >= centre, v >= centre).  The learned part keeps online mean / variance / count of
// the record weights pushed through every node on a record's path from the root; the
// sampled part holds per-node sampling weights (leaves; inner nodes the sums of their
// children), sampled by hierarchical warping (Clarberg et al. 2005, section 5.1).
#pragma once

#include <array>
#include <cstdint>
#include <vector>

namespace tt {

constexpr int kQuadMaxDepth = 8;  // MAX_DEPTH (path_guiding_quadtree.hxx:22)

// Running mean and sum of squared deviations (Welford), as the reference's OnlineVariance.
struct QuadStats {
  double mean = 0.0, sqdev = 0.0;
  int64_t n = 0;
  void add(double x) {
    ++n;
    const double d = x - mean;
    mean += d / (double)n;
    sqdev += d * (x - mean);
  }
};

class QuadDist {
 public:
  // Per node: the four children (all -1 for a leaf); node 0 is the root, every parent comes
  // before its children (depth-first, children in quadrant order).
  std::vector<std::array<int, 4>> child{{{-1, -1, -1, -1}}};
  std::vector<QuadStats> stats{QuadStats{}};  // learned statistics per node
  std::vector<float> probs{1.f};              // sampling weights per node
  std::vector<float> prior{1.f};              // the previous bake's weights

  int num_nodes() const { return (int)child.size(); }
  bool is_leaf(int node) const { return child[node][0] < 0; }
  // InitialFit (path_guiding.cxx:203-217): a tree whose nodes are split while their record
  // weight exceeds 0.1 of the total (Builder, path_guiding_quadtree.cxx:31-60), then every
  // record pushed through it.
  void initial_fit(const float* uv, const float* w, int n);
  // Bake (path_guiding.cxx:274-288): sampling weights = relative counts x mean weight.
  void bake();
  // IncrementalFit (path_guiding.cxx:172-200): records pushed, sampling weights mixed from
  // the prior and the mean plus its error by the node's count, plus an exploration term
  // sqrt(log(sub_round) / (count + 1)) x total flux.
  void incremental_fit(const float* uv, const float* w, int n, int sub_round);
  // IterationUpdateAndBake (path_guiding.cxx:221-271): with more than 10 records, the tree
  // is adapted to the learned flux (TreeAdaptor with 0.05 of the root's flux), the counts
  // scaled to the new nodes' areas, the sampling weights baked from them and the prior, and
  // the learned statistics restarted.  Returns false (nothing changed) otherwise.
  bool update_and_bake();
  // Depth of the leaf holding (u, v) (root = 0).
  int leaf_depth(float u, float v) const;

 private:
  void push(float u, float v, float w);
  void propagate(int node);  // inner nodes := sum of their children's weights
};

// The equal-area cylindrical map between unit directions and the unit square.
void dir_to_square(const float d[3], float uv[2]);
void square_to_dir(const float uv[2], float d[3]);

// Running mean and covariance of a cell's record positions (the cell's leaf_stats,
// OnlineCovariance, sampler.hxx:377-420) and the frame the stochastic filter scatters
// positions with: the covariance's eigenvectors scaled by the square roots of their
// eigenvalues (InitializePcaFrame, path_guiding.cxx:593-608).
struct PointCov {
  double n = 0.0;
  double mean[3] = {0.0, 0.0, 0.0};
  double m2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // xx, yy, zz, xy, xz, yz sums of products of deviations
  void add(const float p[3]);
  // Columns: eigenvector k times sqrt(max(eigenvalue k, 1e-12)).
  void frame(double F[9]) const;
};

// The stochastic filter (PathGuiding::ComputeStochasticFilterPosition, path_guiding.cxx:
// 361-377; RadianceDistributionSampled::ComputeStochasticFilteredDirection, :131-149): a
// copy of a record whose position moves by F (2 r - 1) x 3 (r uniform in the unit cube) and
// whose direction turns by a uniform direction in the cone of half-angle
// 0.5 x 0.5^depth x sqrt(4 pi) about it, depth being that of the quadtree leaf holding it.
void filter_record(const QuadDist& q, const double F[9], const double r[5], const float pos[3], const float wi[3],
                   float pos_out[3], float wi_out[3]);

}  // namespace tt
