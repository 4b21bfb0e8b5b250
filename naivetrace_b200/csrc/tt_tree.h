// Tree guider (tt_tree.cu): the reference's kd-tree guiding with per-cell von Mises-Fisher
// mixtures (PathGuiding, path_guiding.cxx:347-813, with the MoVmf radiance distribution of
// path_guiding.hxx:63-190 and the incremental EM of distribution_mixture_models.cxx:279-388),
// as a fallback beside the learned guider.  The tree lives on the host (a few thousand
// nodes, rebuilt or adapted once per training round); the EM fit of every cell runs on the
// GPU, one warp per cell; sampling looks the cell up on the device (k_guide_tree).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "tt_internal.h"
#include "tt_quadtree.h"

namespace tt {

constexpr int kTreeLobes = 8;
constexpr int kTreeMixFloats = 40;  // per cell: weights[8], means[8][3], concentrations[8]
constexpr int kTreeFitFloats = 36;  // per cell: mean weight, its count, max sample count,
                                    // pending count, pending sums w r_k [8] and w r_k x [8][3]
constexpr int kTreeMaxDepth = 20;   // kdtree::MAX_DEPTH (path_guiding_tree.hxx:20)

struct TreeNodeHost {
  float split;
  int axis;
  int child[2];  // >= 0: node index; < 0: ~cell
};

// The kd-tree over normalised positions ([0,1]^3 of the scene box) and the cells' state.
class TreeGuide {
 public:
  int subdivision = 100;   // guiding_tree_subdivision_factor (scene.hxx:39)
  int em_iters = 0;        // 0: the reference's incremental EM; k > 0: k batch EM iterations per round
  int distribution = 0;    // TT_TREE_VMF or TT_TREE_QUADTREE
  int round = 0;           // fitted rounds
  int ncells = 1;
  std::vector<TreeNodeHost> nodes;        // empty: the root is leaf cell 0
  std::vector<int> cell_depth{0};
  std::vector<int> cell_parent{-1};       // node holding the cell's leaf reference (-1: root)
  std::vector<int> cell_side{0};
  double prev_max_samples = 100.0, prev_total_samples = 0.0;
  long long records_fitted = 0;
  // Quadtree distribution: per cell its quadtree (learned statistics and sampling weights),
  // the positions of the round's records and the stochastic filter's frame.
  std::vector<QuadDist> quads;
  std::vector<PointCov> pstats;
  std::vector<std::array<double, 9>> frames;
  // Device state.
  float4* d_nodes = nullptr;   // split, axis, child0, child1 (int bits)
  int4* d_qchild = nullptr;    // quadtree nodes of all cells (absolute child indices, -1: leaf)
  float* d_qprob = nullptr;    // their sampling weights
  int* d_qroot = nullptr;      // root node of every cell
  int qchild_cap = 0, qprob_cap = 0, qroot_cap = 0;
  float* d_mix = nullptr;      // ncells x kTreeMixFloats
  float* d_fit = nullptr;      // ncells x kTreeFitFloats
  float4* d_recs = nullptr;    // records of a round sorted by cell: direction xyz, weight
  int* d_offsets = nullptr;    // ncells + 1
  int* d_copy = nullptr;       // (dst, src) cell pairs of a split
  int node_cap = 0, mix_cap = 0, fit_cap = 0, rec_cap = 0, off_cap = 0, copy_cap = 0;  // elements

  ~TreeGuide();
  void release();
  bool init(int subdivision_factor, cudaStream_t st, std::string* err);
  // One round (FinalizeRound + PrepareAdaptedStructures): the first round builds the tree
  // from the records (AdaptInitial), later rounds fit the records into the current cells
  // (FitTheSamples) and then split cells that received too many (AdaptIncremental).
  bool fit_round(const GuideRecord* recs, int n, uint64_t seed, cudaStream_t st, std::string* err);
  int lookup(float x, float y, float z) const;
  int root_ref() const { return nodes.empty() ? ~0 : 0; }

 private:
  bool ensure(int cells, int nodes_n, int recs, cudaStream_t st, std::string* err);
  bool upload_quads(cudaStream_t st, std::string* err);
  void fit_quads(const GuideRecord* recs, const std::vector<int>& cell_of, bool initial, uint64_t seed);
  int build(std::vector<int>& idx, int lo, int hi, int depth, const GuideRecord* recs, std::vector<int>& cell_of,
            int parent, int side);
};

// Builds the initial kd-tree of the reference's Builder (path_guiding_tree.hxx:306-440) over
// n points: split at the median along the axis of largest extent while both halves keep at
// least min_points and the depth stays below 20.  Writes each point's cell; returns the
// number of cells.  Host only (also behind tt_kdtree_build_batch).
int kdtree_build(const float* pts, int n, int min_points, std::vector<TreeNodeHost>* nodes, int32_t* cell_of_point);

// Incremental EM of one cell's mixture on the device (the fit kernel on one cell); for tests.
bool vmf_fit_one(const float* recs4, int n, const float* mix_in, const float* fit_in, int batch_iters, float* mix_out,
                 float* fit_out, std::string* err);

// The reference's fixed prior / initial mixture (InitializeForUnitSphere<8>,
// distribution_mixture_models.cxx:174-189).
void tree_prior_mixture(float* mix40);

void launch_tree_fit(const float4* recs, const int* offsets, float* mix, float* fit, int ncells, int batch_iters,
                     cudaStream_t st);

}  // namespace tt
