// Tree guider: kd-tree cells over the scene box with per-cell 8-lobe vMF mixtures, fitted
// once per training round from the records the guided passes collect.
//
// Round structure (PathGuiding::FinalizeRound / PrepareAdaptedStructures,
// path_guiding.cxx:520-547, 613-621):
//   first round   AdaptInitial (:623-674): a kd-tree built from the round's record positions
//                 (median splits along the axis of largest extent, leaves of at least
//                 `subdivision` records), every cell fitted from the prior;
//   later rounds  FitTheSamples (:433-475): records looked up into the current cells and fitted
//                 incrementally; then AdaptIncremental (:676-790): a cell that received more
//                 than sqrt(N) * previous_max / sqrt(previous_N) records splits at the mean of
//                 its records along the axis of largest variance, both children inheriting the
//                 fitted mixture.
// The fit of one cell (vmf_fitting::incremental::Fit, distribution_mixture_models.cxx:279-388)
// walks the cell's records in a shuffled order, accumulating responsibility-weighted
// statistics, and runs a maximisation step with the prior every `10 x prior strength`
// records; statistics of an unfinished chunk carry over to the next round.  Here one warp
// runs one cell: each chunk's statistics are a warp reduction, and every lane runs the same
// maximisation step.
//
// Deviations: the records are this renderer's training records (one reservoir-sampled
// guided vertex per path, weight F/q = contribution after the vertex over throughput before
// it, i.e. the product of BSDF, cosine and incident radiance over the sampling density)
// rather than incident-radiance records; the stochastic filter that duplicates records with
// jittered positions and directions (path_guiding.cxx:361-431) is not applied.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "tt_device.cuh"
#include "tt_tree.h"

namespace tt {

namespace {

// InitializeForUnitSphere<8> (distribution_mixture_models.cxx:174-189): the prior mode and
// the starting mixture of every cell.  Kept identical to the reference (these eight means
// are its choice of a near-uniform covering of the sphere).
constexpr float kPriorMu[24] = {0.66778004f,  0.73539025f,  0.11519922f,  -0.9836298f, -0.008926501f, 0.1799797f,
                                -0.14629413f, -0.7809748f,  0.60718733f,  0.49043104f, 0.04368747f,   -0.87038434f,
                                -0.10088497f, 0.42765132f,  0.8982965f,   -0.35999632f, -0.6945797f,  -0.62286574f,
                                -0.43178025f, 0.7588791f,   -0.48751223f, 0.860208f,   -0.47938251f,  0.17388113f};
constexpr float kPriorKappa = 2.f;
constexpr float kKappaMin = 1.e-4f;  // K_THRESHOLD, distribution_mixture_models.hxx:12
constexpr float kKappaMax = 40.f;    // K_THRESHOLD_MAX, :14
constexpr float kFitEps = 1.e-38f;   // incremental::eps, distribution_mixture_models.hxx:104

__device__ __constant__ float c_prior_mu[24];

__device__ __forceinline__ float tree_vmf_pdf(float mx, float my, float mz, float k, float3 x) {
  return k / (2.f * kPi * (1.f - expf(-2.f * k))) * expf(k * (mx * x.x + my * x.y + mz * x.z - 1.f));
}

// MeanCosineToConc (distribution_mixture_models.hxx:47-55).
__device__ __forceinline__ float mean_cosine_to_conc(float r) {
  r = fminf(r, 1.f - 1.e-6f);
  return r * (3.f - r * r) / (1.f - r * r);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

// One warp per cell.  mix: weights[8], means[8][3], concentrations[8]; fit: mean weight, its
// count, max record count over the rounds, pending count, pending sums (8 + 24).
__global__ void __launch_bounds__(128) k_tree_fit(const float4* __restrict__ recs, const int* __restrict__ offsets,
                                                  float* mix, float* fit, int ncells, int batch_iters) {
  const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (cell >= ncells) return;
  const int b = offsets[cell], e = offsets[cell + 1];
  if (b >= e) return;
  float* M = mix + (size_t)kTreeMixFloats * cell;
  float* F = fit + (size_t)kTreeFitFloats * cell;
  float w[kTreeLobes], mu[kTreeLobes][3], ka[kTreeLobes];
#pragma unroll
  for (int k = 0; k < kTreeLobes; ++k) {
    w[k] = M[k];
    mu[k][0] = M[8 + 3 * k];
    mu[k][1] = M[9 + 3 * k];
    mu[k][2] = M[10 + 3 * k];
    ka[k] = M[32 + k];
  }
  float avg_w = F[0], n_w = F[1];
  const float max_s = fmaxf(F[2], (float)(e - b));
  int pend_n = (int)F[3];
  float pwr[kTreeLobes], pwrx[3 * kTreeLobes];
#pragma unroll
  for (int k = 0; k < kTreeLobes; ++k) pwr[k] = F[4 + k];
#pragma unroll
  for (int k = 0; k < 3 * kTreeLobes; ++k) pwrx[k] = F[12 + k];
  // RadianceDistributionLearned::Parameters (path_guiding.cxx:60-76): prior strength from the
  // cell's largest record count, a maximisation step every 10 x strength records.
  const float ps = fmaxf(1.f, 0.01f * max_s);
  // Batch mode (batch_iters > 0): every maximisation step uses all of the round's records
  // of the cell, batch_iters times; the incremental statistics are not used.
  const bool batch = batch_iters > 0;
  if (batch) {
    pend_n = 0;
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) pwr[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 3 * kTreeLobes; ++k) pwrx[k] = 0.f;
  }
  const int chunk = batch ? e - b : max(1, (int)ps) * 10;
  int iter = 0;
  for (int i = b; i < e;) {
    const int seg = min(chunk - pend_n, e - i);
    float swr[kTreeLobes], swrx[3 * kTreeLobes], sw = 0.f;
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) swr[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 3 * kTreeLobes; ++k) swrx[k] = 0.f;
    // UpdateStatistics (:301-336) of the segment's records, responsibilities under the
    // current mixture.
    for (int j = i + lane; j < i + seg; j += 32) {
      const float4 r = recs[j];
      const float3 x = xyz(r);
      float resp[kTreeLobes], tot = 0.f;
#pragma unroll
      for (int k = 0; k < kTreeLobes; ++k) {
        resp[k] = w[k] * tree_vmf_pdf(mu[k][0], mu[k][1], mu[k][2], ka[k], x) + kFitEps;
        tot += resp[k];
      }
      const float inv = 1.f / tot;
#pragma unroll
      for (int k = 0; k < kTreeLobes; ++k) {
        const float wr = r.w * resp[k] * inv;
        swr[k] += wr;
        swrx[3 * k] += wr * x.x;
        swrx[3 * k + 1] += wr * x.y;
        swrx[3 * k + 2] += wr * x.z;
      }
      sw += r.w;
    }
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) pwr[k] += warp_sum(swr[k]);
#pragma unroll
    for (int k = 0; k < 3 * kTreeLobes; ++k) pwrx[k] += warp_sum(swrx[k]);
    sw = warp_sum(sw);
    if (iter == 0 || !batch) {
      avg_w = (avg_w * n_w + sw) / (n_w + (float)seg);
      n_w += (float)seg;
    }
    pend_n += seg;
    i += seg;
    if (pend_n < chunk) break;
    // MaximizationStep (:339-388) with the fixed prior mode (path_guiding.cxx:72-75).
    const float N = (float)chunk;
    float wsum = 0.f;
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) {
      const float mwr = pwr[k] / N;
      const float m0 = pwrx[3 * k] / N, m1 = pwrx[3 * k + 1] / N, m2 = pwrx[3 * k + 2] / N;
      w[k] = (ps - 1.f) / N * (1.f / kTreeLobes) + mwr / (avg_w + kFitEps) + kFitEps;
      const float dim = avg_w * ps / N;
      const float den = dim + mwr + kFitEps;
      float a0 = (dim * c_prior_mu[3 * k] + m0) / den, a1 = (dim * c_prior_mu[3 * k + 1] + m1) / den,
            a2 = (dim * c_prior_mu[3 * k + 2] + m2) / den;
      const float nrm = sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
      if (nrm > kFitEps) {
        a0 /= nrm;
        a1 /= nrm;
        a2 /= nrm;
      } else {
        a0 = 1.f;
        a1 = a2 = 0.f;
      }
      mu[k][0] = a0;
      mu[k][1] = a1;
      mu[k][2] = a2;
      const float mcos = sqrtf(m0 * m0 + m1 * m1 + m2 * m2) / (mwr + kFitEps);
      const float da = ps / N;
      const float kk = (kPriorKappa * da + mean_cosine_to_conc(mcos)) / (da + 1.f);
      ka[k] = fminf(fmaxf(kk, kKappaMin), kKappaMax);
      wsum += w[k];
    }
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) w[k] /= wsum;
    pend_n = 0;
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) pwr[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 3 * kTreeLobes; ++k) pwrx[k] = 0.f;
    if (batch && ++iter < batch_iters) i = b;
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) {
      M[k] = w[k];
      M[8 + 3 * k] = mu[k][0];
      M[9 + 3 * k] = mu[k][1];
      M[10 + 3 * k] = mu[k][2];
      M[32 + k] = ka[k];
    }
    F[0] = avg_w;
    F[1] = n_w;
    F[2] = max_s;
    F[3] = (float)pend_n;
#pragma unroll
    for (int k = 0; k < kTreeLobes; ++k) F[4 + k] = pwr[k];
#pragma unroll
    for (int k = 0; k < 3 * kTreeLobes; ++k) F[12 + k] = pwrx[k];
  }
}

// Children of split cells inherit the parent's state: cells[pairs[2i]] = cells[pairs[2i+1]].
__global__ void k_tree_copy(const int* pairs, int n, float* mix, float* fit) {
  const int i = blockIdx.x;
  if (i >= n) return;
  const int dst = pairs[2 * i], src = pairs[2 * i + 1];
  for (int k = threadIdx.x; k < kTreeMixFloats; k += blockDim.x)
    mix[(size_t)kTreeMixFloats * dst + k] = mix[(size_t)kTreeMixFloats * src + k];
  for (int k = threadIdx.x; k < kTreeFitFloats; k += blockDim.x)
    fit[(size_t)kTreeFitFloats * dst + k] = fit[(size_t)kTreeFitFloats * src + k];
}

bool g_prior_uploaded[64] = {false};

cudaError_t upload_prior() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && g_prior_uploaded[dev]) return cudaSuccess;
  const cudaError_t e = cudaMemcpyToSymbol(c_prior_mu, kPriorMu, sizeof(kPriorMu));
  if (e == cudaSuccess && dev >= 0 && dev < 64) g_prior_uploaded[dev] = true;
  return e;
}

// Median splits along the axis of largest extent (Builder::TryBuildBranchRecursive,
// path_guiding_tree.hxx:388-420); a leaf when fewer than 2 x min_points remain or the depth
// reaches the limit, or when a split would leave a side with fewer than min_points.
template <class Coord, class Leaf>
int build_rec(std::vector<int>& idx, int lo, int hi, int depth, int min_points, const Coord& coord,
              std::vector<TreeNodeHost>* nodes, const Leaf& leaf, int parent, int side) {
  const int n = hi - lo;
  if (n < 2 * min_points || depth >= kTreeMaxDepth) return ~leaf(lo, hi, depth, parent, side);
  float bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = lo; i < hi; ++i)
    for (int a = 0; a < 3; ++a) {
      bmin[a] = std::min(bmin[a], coord(idx[i], a));
      bmax[a] = std::max(bmax[a], coord(idx[i], a));
    }
  int axis = 0;
  for (int a = 1; a < 3; ++a)
    if (bmax[a] - bmin[a] > bmax[axis] - bmin[axis]) axis = a;
  const int mid = lo + n / 2;
  std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi,
                   [&](int p, int q) { return coord(p, axis) < coord(q, axis); });
  const float pos = coord(idx[mid], axis);
  if (n / 2 < min_points || n - n / 2 < min_points) return ~leaf(lo, hi, depth, parent, side);
  const int node = (int)nodes->size();
  nodes->push_back(TreeNodeHost{pos, axis, {0, 0}});
  const int l = build_rec(idx, lo, mid, depth + 1, min_points, coord, nodes, leaf, node, 0);
  const int r = build_rec(idx, mid, hi, depth + 1, min_points, coord, nodes, leaf, node, 1);
  (*nodes)[node].child[0] = l;
  (*nodes)[node].child[1] = r;
  return node;
}

template <class T>
bool grow(T** p, int* cap, int need, cudaStream_t st, bool keep, std::string* err) {
  if (need <= *cap) return true;
  const int ncap = std::max(need, 2 * *cap + 64);
  T* np = nullptr;
  if (cudaMalloc(&np, (size_t)ncap * sizeof(T)) != cudaSuccess) {
    *err = "tree guider: device allocation failed";
    return false;
  }
  if (*p) {
    if (keep) cudaMemcpyAsync(np, *p, (size_t)*cap * sizeof(T), cudaMemcpyDeviceToDevice, st);
    cudaStreamSynchronize(st);
    cudaFree(*p);
  }
  *p = np;
  *cap = ncap;
  return true;
}

}  // namespace

void tree_prior_mixture(float* mix40) {
  for (int k = 0; k < kTreeLobes; ++k) {
    mix40[k] = 1.f / kTreeLobes;
    for (int a = 0; a < 3; ++a) mix40[8 + 3 * k + a] = kPriorMu[3 * k + a];
    mix40[32 + k] = kPriorKappa;
  }
}

void launch_tree_fit(const float4* recs, const int* offsets, float* mix, float* fit, int ncells, int batch_iters,
                     cudaStream_t st) {
  if (ncells <= 0) return;
  const int blocks = (ncells * 32 + 127) / 128;
  k_tree_fit<<<blocks, 128, 0, st>>>(recs, offsets, mix, fit, ncells, batch_iters);
}

int kdtree_build(const float* pts, int n, int min_points, std::vector<TreeNodeHost>* nodes, int32_t* cell_of_point) {
  nodes->clear();
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  int ncells = 0;
  auto coord = [pts](int i, int a) { return pts[3 * (size_t)i + a]; };
  auto leaf = [&](int lo, int hi, int, int, int) {
    const int c = ncells++;
    for (int i = lo; i < hi; ++i) cell_of_point[idx[i]] = c;
    return c;
  };
  build_rec(idx, 0, n, 1, std::max(1, min_points), coord, nodes, leaf, -1, 0);
  return ncells;
}

TreeGuide::~TreeGuide() { release(); }

void TreeGuide::release() {
  for (void* p : {(void*)d_nodes, (void*)d_mix, (void*)d_fit, (void*)d_recs, (void*)d_offsets, (void*)d_copy,
                  (void*)d_qchild, (void*)d_qprob, (void*)d_qroot})
    if (p) cudaFree(p);
  d_nodes = nullptr;
  d_mix = d_fit = nullptr;
  d_recs = nullptr;
  d_offsets = d_copy = nullptr;
  d_qchild = nullptr;
  d_qprob = nullptr;
  d_qroot = nullptr;
  node_cap = mix_cap = fit_cap = rec_cap = off_cap = copy_cap = 0;
  qchild_cap = qprob_cap = qroot_cap = 0;
}

bool TreeGuide::ensure(int cells, int nodes_n, int recs, cudaStream_t st, std::string* err) {
  if (!grow(&d_mix, &mix_cap, cells * kTreeMixFloats, st, true, err)) return false;
  if (!grow(&d_fit, &fit_cap, cells * kTreeFitFloats, st, true, err)) return false;
  return grow(&d_nodes, &node_cap, std::max(1, nodes_n), st, false, err) &&
         grow(&d_recs, &rec_cap, std::max(1, recs), st, false, err) &&
         grow(&d_offsets, &off_cap, cells + 1, st, false, err) && grow(&d_copy, &copy_cap, 2 * cells, st, false, err);
}

bool TreeGuide::init(int subdivision_factor, cudaStream_t st, std::string* err) {
  release();
  subdivision = subdivision_factor > 0 ? subdivision_factor : 100;
  round = 0;
  ncells = 1;
  nodes.clear();
  cell_depth.assign(1, 1);
  cell_parent.assign(1, -1);
  cell_side.assign(1, 0);
  prev_max_samples = subdivision;
  prev_total_samples = 0;
  records_fitted = 0;
  // Before the first round the single cell's quadtree is one leaf: uniform over the sphere.
  quads.assign(1, QuadDist{});
  frames.assign(1, std::array<double, 9>{1, 0, 0, 0, 1, 0, 0, 0, 1});
  if (upload_prior() != cudaSuccess) {
    *err = "tree guider: constant upload failed";
    return false;
  }
  if (!ensure(1, 1, 1, st, err) || !upload_quads(st, err)) return false;
  std::vector<float> mix(kTreeMixFloats), fit(kTreeFitFloats, 0.f);
  tree_prior_mixture(mix.data());
  cudaMemcpyAsync(d_mix, mix.data(), mix.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_fit, fit.data(), fit.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    *err = std::string("tree guider: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

int TreeGuide::lookup(float x, float y, float z) const {
  int ref = root_ref();
  for (int d = 0; d < 64 && ref >= 0; ++d) {
    const TreeNodeHost& nd = nodes[ref];
    const float c = nd.axis == 0 ? x : (nd.axis == 1 ? y : z);
    ref = c < nd.split ? nd.child[0] : nd.child[1];
  }
  return ref < 0 ? ~ref : 0;
}

bool TreeGuide::fit_round(const GuideRecord* recs, int n, uint64_t seed, cudaStream_t st, std::string* err) {
  if (n <= 0) return true;
  std::vector<int> cell_of(n);
  const bool initial = round == 0;
  if (initial) {
    // AdaptInitial: a tree built from this round's records, every cell starting from the prior.
    nodes.clear();
    cell_depth.clear();
    cell_parent.clear();
    cell_side.clear();
    ncells = 0;
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    auto coord = [recs](int i, int a) { return recs[i].pos[a]; };
    auto leaf = [&](int lo, int hi, int depth, int parent, int side) {
      const int c = ncells++;
      cell_depth.push_back(depth);
      cell_parent.push_back(parent);
      cell_side.push_back(side);
      for (int i = lo; i < hi; ++i) cell_of[idx[i]] = c;
      return c;
    };
    build_rec(idx, 0, n, 1, subdivision, coord, &nodes, leaf, -1, 0);
    prev_max_samples = subdivision;
    prev_total_samples = n;
  } else {
    for (int i = 0; i < n; ++i) cell_of[i] = lookup(recs[i].pos[0], recs[i].pos[1], recs[i].pos[2]);
  }
  // Records sorted by cell, shuffled within each cell (FitTheSamples shuffles before fitting).
  std::vector<int> offsets(ncells + 1, 0);
  for (int c : cell_of) offsets[c + 1]++;
  for (int c = 0; c < ncells; ++c) offsets[c + 1] += offsets[c];
  std::vector<int> order(n), fill(offsets.begin(), offsets.end() - 1);
  for (int i = 0; i < n; ++i) order[fill[cell_of[i]]++] = i;
  std::mt19937_64 rng(seed * 0x9e3779b97f4a7c15ull + (uint64_t)round);
  for (int c = 0; c < ncells; ++c) std::shuffle(order.begin() + offsets[c], order.begin() + offsets[c + 1], rng);
  std::vector<float4> sorted(n);
  for (int i = 0; i < n; ++i) {
    const GuideRecord& r = recs[order[i]];
    sorted[i] = make_float4(r.wi[0], r.wi[1], r.wi[2], r.f_over_q);
  }
  if (!ensure(ncells, (int)nodes.size(), n, st, err)) return false;
  const bool quad = distribution == TT_TREE_QUADTREE;
  if (quad) fit_quads(recs, cell_of, initial, seed);
  if (quad) {
    // The vMF state is not used.
  } else if (initial) {
    std::vector<float> mix((size_t)ncells * kTreeMixFloats), fit((size_t)ncells * kTreeFitFloats, 0.f);
    for (int c = 0; c < ncells; ++c) tree_prior_mixture(&mix[(size_t)c * kTreeMixFloats]);
    cudaMemcpyAsync(d_mix, mix.data(), mix.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_fit, fit.data(), fit.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  }
  if (!quad) {
    cudaMemcpyAsync(d_recs, sorted.data(), (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_offsets, offsets.data(), offsets.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    launch_tree_fit(d_recs, d_offsets, d_mix, d_fit, ncells, em_iters, st);
  }
  if (!initial) {
    // AdaptIncremental: split cells that received too many records this round.
    const double max_per_cell = std::sqrt((double)n) * prev_max_samples / std::sqrt(std::max(1.0, prev_total_samples));
    std::vector<int> pairs;
    const int before = ncells;
    for (int c = 0; c < before; ++c) {
      const int cnt = offsets[c + 1] - offsets[c];
      if (cnt <= max_per_cell || cell_depth[c] >= kTreeMaxDepth) continue;
      double mean[3] = {0, 0, 0}, sq[3] = {0, 0, 0};
      for (int i = offsets[c]; i < offsets[c + 1]; ++i)
        for (int a = 0; a < 3; ++a) mean[a] += recs[order[i]].pos[a];
      for (int a = 0; a < 3; ++a) mean[a] /= cnt;
      for (int i = offsets[c]; i < offsets[c + 1]; ++i)
        for (int a = 0; a < 3; ++a) {
          const double d = recs[order[i]].pos[a] - mean[a];
          sq[a] += d * d;
        }
      int axis = 0;
      for (int a = 1; a < 3; ++a)
        if (sq[a] > sq[axis]) axis = a;
      const int nc = ncells++;
      const int node = (int)nodes.size();
      nodes.push_back(TreeNodeHost{(float)mean[axis], axis, {~c, ~nc}});
      if (cell_parent[c] >= 0) nodes[cell_parent[c]].child[cell_side[c]] = node;
      cell_parent[c] = node;
      cell_side[c] = 0;
      cell_parent.push_back(node);
      cell_side.push_back(1);
      cell_depth[c] += 1;
      cell_depth.push_back(cell_depth[c]);
      pairs.push_back(nc);
      pairs.push_back(c);
      if (quad) {
        // Both halves start from the cell's distribution (AdaptIncremental's CopyCell).
        quads.push_back(quads[c]);
        frames.push_back(frames[c]);
      }
    }
    prev_max_samples = max_per_cell;
    prev_total_samples = n;
    if (!pairs.empty() && !quad) {
      if (!ensure(ncells, (int)nodes.size(), n, st, err)) return false;
      cudaMemcpyAsync(d_copy, pairs.data(), pairs.size() * sizeof(int), cudaMemcpyHostToDevice, st);
      k_tree_copy<<<(int)pairs.size() / 2, 64, 0, st>>>(d_copy, (int)pairs.size() / 2, d_mix, d_fit);
    }
  }
  std::vector<float4> dn(std::max<size_t>(1, nodes.size()));
  auto bits = [](int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
  };
  for (size_t i = 0; i < nodes.size(); ++i)
    dn[i] = make_float4(nodes[i].split, bits(nodes[i].axis), bits(nodes[i].child[0]), bits(nodes[i].child[1]));
  if (!grow(&d_nodes, &node_cap, (int)dn.size(), st, false, err)) return false;
  cudaMemcpyAsync(d_nodes, dn.data(), dn.size() * sizeof(float4), cudaMemcpyHostToDevice, st);
  if (quad && !upload_quads(st, err)) return false;
  // The host vectors above are pageable: wait for the copies before they go out of scope.
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    *err = std::string("tree guider: ") + cudaGetErrorString(e);
    return false;
  }
  ++round;
  records_fitted += n;
  return true;
}

// The quadtree distributions of one round.  First round (AdaptInitial, path_guiding.cxx:
// 623-674): every cell's tree from its records (InitialFit + Bake) and the stochastic
// filter's frame from their positions.  Later rounds: FitTheSamples (:433-475) with the
// stochastic filter, whose copies of the records (jittered by the cells' current frames
// and trees, looked up again) are the ones the quadtrees fit (IncrementalFit skips the
// originals); then, as AdaptIncremental (:676-790) does per cell, IterationUpdateAndBake
// and a new frame from the round's positions when the cell received at least 10 records.
// Deviation: the reference adapts after each sweep of passes; here every round adapts.
// Runs f(begin, end) over [0, n) in contiguous chunks on the host's threads.
template <class F>
static void host_parallel(int n, F&& f) {
  const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), (n + 255) / 256));
  if (nt <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    const int b = (int)((long long)n * t / nt), e = (int)((long long)n * (t + 1) / nt);
    th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto& x : th) x.join();
}

void TreeGuide::fit_quads(const GuideRecord* recs, const std::vector<int>& cell_of, bool initial, uint64_t seed) {
  const int n = (int)cell_of.size();
  if (initial) {
    quads.assign(ncells, QuadDist{});
    frames.assign(ncells, std::array<double, 9>{1, 0, 0, 0, 1, 0, 0, 0, 1});
  }
  // The records the quadtrees fit: the originals in the first round, the stochastic
  // filter's copies (moved to the cell of their jittered position) later.  The filter's
  // uniforms are drawn in record order, so the result does not depend on the threading.
  std::vector<float> uv(2 * (size_t)n);
  std::vector<int> fit_cell(n);
  if (initial) {
    host_parallel(n, [&](int b, int e) {
      for (int i = b; i < e; ++i) {
        dir_to_square(recs[i].wi, &uv[2 * (size_t)i]);
        fit_cell[i] = cell_of[i];
      }
    });
  } else {
    std::mt19937_64 rng(seed * 0x9e3779b97f4a7c15ull + 0xd1b54a32d192ed03ull * (uint64_t)(round + 1));
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    std::vector<double> rr(5 * (size_t)n);
    for (double& x : rr) x = uni(rng);
    host_parallel(n, [&](int b, int e) {
      for (int i = b; i < e; ++i) {
        const int c = cell_of[i];
        float p2[3], d2[3];
        filter_record(quads[c], frames[c].data(), &rr[5 * (size_t)i], recs[i].pos, recs[i].wi, p2, d2);
        fit_cell[i] = lookup(p2[0], p2[1], p2[2]);
        dir_to_square(d2, &uv[2 * (size_t)i]);
      }
    });
  }
  // Records of every cell, in record order.
  std::vector<int> off(ncells + 1, 0);
  for (int c : fit_cell) off[c + 1]++;
  for (int c = 0; c < ncells; ++c) off[c + 1] += off[c];
  std::vector<int> fill(off.begin(), off.end() - 1), idx(n);
  for (int i = 0; i < n; ++i) idx[fill[fit_cell[i]]++] = i;
  std::vector<int> pos_off(ncells + 1, 0);
  for (int c : cell_of) pos_off[c + 1]++;
  for (int c = 0; c < ncells; ++c) pos_off[c + 1] += pos_off[c];
  std::vector<int> pfill(pos_off.begin(), pos_off.end() - 1), pidx(n);
  for (int i = 0; i < n; ++i) pidx[pfill[cell_of[i]]++] = i;
  host_parallel(ncells, [&](int c0, int c1) {
    std::vector<float> cu, cw;
    for (int c = c0; c < c1; ++c) {
      cu.clear();
      cw.clear();
      for (int k = off[c]; k < off[c + 1]; ++k) {
        const int i = idx[k];
        cu.push_back(uv[2 * (size_t)i]);
        cu.push_back(uv[2 * (size_t)i + 1]);
        cw.push_back(recs[i].f_over_q);
      }
      PointCov ps;
      for (int k = pos_off[c]; k < pos_off[c + 1]; ++k) ps.add(recs[pidx[k]].pos);
      const int m = (int)cw.size();
      if (initial) {
        quads[c].initial_fit(cu.data(), cw.data(), m);
        quads[c].bake();
        ps.frame(frames[c].data());
      } else {
        quads[c].incremental_fit(cu.data(), cw.data(), m, 1);
        quads[c].update_and_bake();
        if (ps.n >= 10.0) ps.frame(frames[c].data());
      }
    }
  });
}

bool TreeGuide::upload_quads(cudaStream_t st, std::string* err) {
  std::vector<int> roots(std::max(1, ncells));
  int total = 0;
  for (int c = 0; c < ncells; ++c) {
    roots[c] = total;
    total += quads[c].num_nodes();
  }
  std::vector<int4> ch(std::max(1, total));
  std::vector<float> pr(std::max(1, total));
  for (int c = 0; c < ncells; ++c) {
    const QuadDist& q = quads[c];
    for (int j = 0; j < q.num_nodes(); ++j) {
      const auto& k = q.child[j];
      ch[roots[c] + j] = k[0] < 0 ? make_int4(-1, -1, -1, -1)
                                  : make_int4(roots[c] + k[0], roots[c] + k[1], roots[c] + k[2], roots[c] + k[3]);
      pr[roots[c] + j] = q.probs[j];
    }
  }
  if (!grow(&d_qchild, &qchild_cap, (int)ch.size(), st, false, err) ||
      !grow(&d_qprob, &qprob_cap, (int)pr.size(), st, false, err) ||
      !grow(&d_qroot, &qroot_cap, (int)roots.size(), st, false, err))
    return false;
  cudaMemcpyAsync(d_qchild, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_qprob, pr.data(), pr.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_qroot, roots.data(), roots.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  const cudaError_t e = cudaStreamSynchronize(st);  // the host vectors are local
  if (e != cudaSuccess) {
    *err = std::string("tree guider: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool vmf_fit_one(const float* recs4, int n, const float* mix_in, const float* fit_in, int batch_iters, float* mix_out,
                 float* fit_out, std::string* err) {
  if (upload_prior() != cudaSuccess) {
    *err = "constant upload failed";
    return false;
  }
  float4* d_recs = nullptr;
  int* d_off = nullptr;
  float *d_mix = nullptr, *d_fit = nullptr;
  bool ok = cudaMalloc(&d_recs, std::max(1, n) * sizeof(float4)) == cudaSuccess &&
            cudaMalloc(&d_off, 2 * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&d_mix, kTreeMixFloats * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&d_fit, kTreeFitFloats * sizeof(float)) == cudaSuccess;
  if (ok) {
    std::vector<float> mix(kTreeMixFloats), fit(kTreeFitFloats, 0.f);
    if (mix_in) std::memcpy(mix.data(), mix_in, sizeof(float) * kTreeMixFloats);
    else tree_prior_mixture(mix.data());
    if (fit_in) std::memcpy(fit.data(), fit_in, sizeof(float) * kTreeFitFloats);
    const int off[2] = {0, n};
    cudaMemcpy(d_recs, recs4, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice);
    cudaMemcpy(d_off, off, sizeof(off), cudaMemcpyHostToDevice);
    cudaMemcpy(d_mix, mix.data(), sizeof(float) * kTreeMixFloats, cudaMemcpyHostToDevice);
    cudaMemcpy(d_fit, fit.data(), sizeof(float) * kTreeFitFloats, cudaMemcpyHostToDevice);
    launch_tree_fit(d_recs, d_off, d_mix, d_fit, 1, batch_iters, 0);
    ok = cudaMemcpy(mix_out, d_mix, sizeof(float) * kTreeMixFloats, cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(fit_out, d_fit, sizeof(float) * kTreeFitFloats, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (!ok) *err = std::string("vmf fit: ") + cudaGetErrorString(cudaGetLastError());
  } else {
    *err = "vmf fit: device allocation failed";
  }
  for (void* p : {(void*)d_recs, (void*)d_off, (void*)d_mix, (void*)d_fit})
    if (p) cudaFree(p);
  return ok;
}

}  // namespace tt
