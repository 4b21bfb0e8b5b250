// Shared host/device declarations of the CUDA path tracer: the device scene record, the
// wavefront path-state layout and the kernel entry points.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/toytrace_gpu.h"

namespace tt {

constexpr int NBINS = TT_NBINS;
constexpr int MAX_ENV_LIGHTS = 4;
constexpr int BVH_STACK = 64;        // per-thread traversal stack (entries), binary BVH
constexpr int BVH8_STACK = 32;       // per-thread stack of node groups, 8-wide BVH
constexpr uint32_t ERR_STACK = 1u;   // error-word bits written by kernels
constexpr uint32_t ERR_QUEUE = 2u;
constexpr uint32_t ERR_CROSSINGS = 4u;  // a ray crossed more medium boundaries than the cap
constexpr uint32_t ERR_TENSOR = 8u;     // a wait on the tcgen05 tensor cores gave up
constexpr int kMaxCrossings = 256;      // boundary crossings followed along one ray
constexpr int kMaxMedia = 254;          // medium indices are stored in bytes (0xff = empty)
// Shading keys of the material-sorted hit queue: escaped, volume vertex, then one per shader kind.
constexpr int kShadeKeys = 8;
// Per bounce: ext, shadow, done, guided queue lengths, then the shading-key counts and cursors.
constexpr int kCountersPerBounce = 4 + 2 * kShadeKeys;
constexpr int kSobolDims = 4096;       // quasi-random dimensions: subsequence ids < 64, 64 each
constexpr int kRotationBlock = 128;    // per-pixel rotations repeat every 128 pixels in x and y

// One training record of the learned guide: a guided surface vertex (position normalised to
// the scene box, shading normal, outgoing direction), the sampled incident direction, the
// BSDF density of that direction, and F / q = (path contribution after the vertex) /
// (throughput before it) averaged over the path's wavelengths.
struct GuideRecord {
  float pos[3];
  float n[3];
  float wo[3];
  float wi[3];
  float p_bsdf;
  float f_over_q;
};

// Surface material as stored on the device.
struct DevMaterial {
  int shader;
  int emissive;
  float alpha;
  float ior_ratio;
  int med_in;        // medium entered through the front side (winding normal), -1 none
  int med_out;       // medium on the front side, -1 none
  int tex_w, tex_h;  // diffuse texture size
  const float* tex;  // diffuse texture (linear RGB, row 0 at the top), or nullptr
  float spec;        // dense dielectric: coating reflectivity at normal incidence
  int pad;
  float reflectance[NBINS];
  float emission[NBINS];
};

// A participating medium: homogeneous (HomogeneousMedium, shader.cxx:1234-1316) with its
// phase function, or a tabulated planetary atmosphere (Atmosphere::Tabulated,
// atmosphere.cxx:18-126, 234-348; lengths in km).
struct DevMedium {
  int kind;          // TT_MEDIUM_*
  int priority;
  int phase;         // TT_PHASE_* (homogeneous)
  float g;           // Henyey-Greenstein asymmetry (homogeneous HG; atmosphere aerosols)
  int scattering;    // any sigma_s > 0
  // Atmosphere.
  int rows;          // altitude rows
  float h0, inv_dh;  // altitude of row 0, 1 / row spacing
  float center[3];
  float radius;
  const float4* table;  // rows x NBINS: (sigma_t, sigma_s molecules, sigma_s aerosols, 0)
  const float* maj;     // rows: majorant, non-increasing with altitude
  // Homogeneous.
  float sigma_s[NBINS];
  float sigma_ext[NBINS];
};

struct DevEnvLight {
  int kind;
  int w, h;
  float pdf_val, cos_opening;            // sun
  float X[3], Y[3], Z[3];                // frame columns (sun, dome, env map)
  float dir[3];                          // directional light
  float spectrum[NBINS];                 // dome / directional / sun emission (pre-scaled)
  const float* tex;                      // env map RGB, row 0 = top
  const float* cmf_rows;                 // h
  const float* cmf_cols;                 // w * h
  const int* guide_rows;                 // kEnvGuide + 1: search range of cmf_rows per 1/kEnvGuide of [0, 1]
  const int* guide_cols;                 // h * (kEnvGuide + 1): the same per row of cmf_cols
};
// Entries of the env map's CMF guide tables: guide[g] = the index that inverting the CMF
// gives for r = g / kEnvGuide (the first entry above r), so that a sample r needs only a
// bisection between guide[g] and guide[g + 1], g = floor(r kEnvGuide).  A power of two, so
// that g / kEnvGuide and r kEnvGuide are exact in float.
constexpr int kEnvGuide = 256;

struct DevCamera {
  int kind;
  int xres, yres;
  float pos[3], up[3], dir[3], right[3];
  float xmin, ymin, xperpixel, yperpixel, per_pixel_delta;
};

// Everything a kernel needs to know about the scene; passed by value (constant bank).
struct DevScene {
  const float4* nodes4;       // the surface BVH with four children per node (tt_build.h), when
                              // built: the binary layout's traversal then uses it
  int wide;                   // 1: the 8-wide BVH (nodes8 / vnodes8) is the active layout
  const uint4* nodes8;        // 8-wide BVH, 5 uint4 per node (tt_bvh.h)
  const uint4* vnodes8;
  const float4* nodes;        // BVH2, 4 float4 per node (when wide == 0)
  const float4* tris;         // 3 float4 per primitive slot of the active layout: v0 (w=prim), v1 (w=material), v2
  const uint4* tri_idx;       // per prim: vertex indices a, b, c and material
  const float* normals;       // per vertex xyz, or nullptr
  const float2* uvs;          // per vertex texture coordinates, or nullptr
  const DevMaterial* materials;
  const int* area_lights;     // prim of each area light
  const float4* area_verts;   // 3 float4 (v0, v1, v2) per area light
  const float* point_lights;  // per light: spectrum[36], pos[3]
  int num_area_lights;
  int num_point_lights;
  int num_env;
  int num_tris;
  DevEnvLight env[MAX_ENV_LIGHTS];
  DevCamera cam;
  float type_probs[4];        // ENV, AREA, POINT, VOLUME
  float in_class_area;
  float long_distance;        // 10 x bounding-box diagonal
  int max_path_nodes;         // max_ray_depth + 1
  int sample_lights;
  int sample_bsdf;
  // Participating media: medium boundaries live in their own BVH (same layout as the
  // surface BVH), as in Scene::BuildAccelStructure (scene.cxx:116-141).
  const float4* vnodes;
  const float4* vtris;
  int num_vol_tris;
  int num_spheres;            // spheres share the BVH slot arrays (tt_bvh.h)
  int num_media;
  const DevMedium* media;
  uint2 cam_track;            // medium tracker at the camera position
  // Learned guiding (tt_guide.cuh): sample diffuse and microfacet surfaces by one-sample
  // MIS of the BSDF and the network's vMF mixture.
  int guide;                  // 1: guided scattering
  int guide_record;           // 1: collect training records
  int guide_depth;            // guided vertices only at bounces < guide_depth
  int guide_cold;             // 1: the network still has its random initial weights: guided
                              // vertices sample the BSDF only (records are still collected)
  float guide_keep;           // probability that a finished path keeps its record (a uniform
                              // subsample when a pass would yield more than the pool holds)
  const __nv_bfloat16* guide_w16;  // network weights (BF16, flat layout of tt_guide.cuh)
  const float* guide_w32;          // FP32 master copy (the biases are read from it)
  float box_lo[3];            // scene box, for the position encoding
  float box_inv[3];           // 1 / extent per axis
  int algo;                   // TT_ALGO_PT or TT_ALGO_PT2 (tt_pt2.cuh)
  int sort_shading;           // 1: shade the bounce's hits in material-sorted order (algo pt)
  int block;                  // threads per block of the wavefront launches (0: 256), host side only
  // Tree guider (tt_tree.cu), when guide_method == TT_GUIDE_TREE: kd-tree nodes (split,
  // axis, child0, child1 as int bits; a child < 0 is ~cell), the root reference and the
  // cells' mixtures (40 floats each: weights[8], means[8][3], concentrations[8]).
  int guide_method;
  int guide_net;  // TT_GUIDE_NET_TCGEN05 or TT_GUIDE_NET_MMA: the kernel that runs the network
  const float4* tree_nodes;
  int tree_root;
  const float* tree_mix;
  int tree_quad;             // the cells' directional distributions are quadtrees
  const int4* tree_qchild;   // their nodes (absolute child indices, -1: leaf)
  const float* tree_qprob;   // sampling weights per node
  const int* tree_qroot;     // root node per cell
  // Quasi-random sampling (pt2 with qmc): Sobol generator matrices, 32 words per dimension
  // (TT_SOBOL_DIMS dimensions), and the per-pixel rotations [128 * 128][2]; null otherwise.
  const uint32_t* sobol;
  const float* rotations;
};

// Wavefront path state, structure of arrays, capacity `cap` paths.
struct PathState {
  int cap;
  float4* ray_o;       // origin
  float4* ray_d;       // direction, w = tfar
  float4* hit;         // t, u, v, triangle slot (int bits, -1 = miss)
  float4* beta;        // path throughput (3), w = pdf of the last scatter (negative: delta)
  float4* accum;       // spectral path sum (3)
  unsigned long long* rng_state;
  unsigned long long* rng_inc;
  uint4* meta;         // x pixel, y lambda idx (3 x 8 bits), z node count, w unused
  float4* sh_o;        // shadow ray origin, w = tfar
  float4* sh_d;        // direction, w = splat target pixel (int bits) or -1
  float4* sh_c;        // spectral contribution
  int* ext_q[2];
  int* sh_q;
  int* done_q;
  int* counters;       // kCountersPerBounce ints per bounce, (max bounces + 3) bounces
  int* sort_q;         // material-sorted hit queue (sort_shading only, else null)
  unsigned char* sort_key;  // shading key per entry of the bounce's hit queue
  unsigned int* err;
  // Media scenes only (null otherwise).
  uint2* track;        // medium tracker: x = 4 slot bytes (0xff empty), y = current medium (-1 vacuum)
  float4* vol;         // sigma_s at a volume interaction (xyz); w = transmittance pdf factor of the step
  uint2* sh_track;     // medium tracker of the shadow ray at its origin
  float4* sh_med;      // x = light pdf (< 0: MIS weight 1), y = scatter pdf before the transmittance
                       // factor, z/w = the path's random state at the connection (low/high words)
  // Guided scenes only (null otherwise).
  float4* ginp;        // network inputs per guided-queue entry: 3 float4 holding p01 xyz,
                       // shading normal xyz, outgoing direction xyz
  int* guide_q;        // guided-vertex queue (slots)
  float4* grec;        // pending training record per path: 6 float4 (tt_kernels.cu)
  float4* gnee;        // NEE at a guided vertex: light pdf (-1: no MIS), pdf conversion,
                       // BSDF pdf of the shadow direction, emitted flag
  float* rr;           // Russian-roulette throughput factor: (throughput with BSDF densities at
                       // the guided vertices) / beta
  GuideRecord* records;  // training-record pool, a ring of rec_cap records
  int* rec_count;        // records committed since the pool was emptied (index = count % rec_cap)
  int rec_cap;
  // Null-path tracer (TT_ALGO_PT2) only.
  float* rough;        // path roughness: largest microfacet alpha met so far
  float* wt2;          // media scenes: weights_track, 9 floats per path (row-major 3 x 3)
  float* sh_wt;        // media scenes: the path's weights_track at the shadow ray's vertex
  uint4* qmc;          // quasi-random state: point index, rotations (32-bit fixed point),
                       // subsequence (dimension offset | draw counter << 16)
  uint4* sh_qmc;       // media scenes: the same at the shadow ray's connection
};

struct Framebuffer {
  float* accum;        // npix * 3, this pass
  float* light;        // npix * 3, this pass
};

// One camera view of a multi-view batch (tt_render_views).
struct DevView {
  DevCamera cam;
  long long path_begin;        // first path of the view in the batch's path numbering
  int pix_begin;               // first pixel of the view in the concatenated framebuffer
  int npix;
  int spp;
  uint2 cam_track;             // medium tracker at the camera
  unsigned long long seed;
};

struct ViewWave {
  long long wave_start;
  int wave_paths;
};

struct WaveArgs {
  long long wave_start;      // first path of this wave within the pass
  int wave_paths;
  int pixel_begin;
  int npix_range;
  int npix_total;
  unsigned long long sample_offset;
  unsigned long long seed;
};

// Kernel launchers (tt_kernels.cu).  `stats` (device, 4 x u64) receives node visits and
// triangle tests of extension and shadow rays when counting is on.
void upload_constant_tables();
void launch_generate(const DevScene& s, const PathState& p, const Framebuffer& fb, const WaveArgs& w, int grid,
                     cudaStream_t st);
// Multi-view batch: generate from waves[*wave_idx]; advance *wave_idx; per-view resolve.
void launch_generate_views(const DevScene& s, const PathState& p, const ViewWave* waves, const int* wave_idx,
                           const DevView* views, int nviews, int grid, cudaStream_t st);
void launch_wave_advance(int* wave_idx, cudaStream_t st);
void launch_resolve_views(const float* accum, const float* light, const DevView* views, int nviews, int npix,
                          float* rgb, cudaStream_t st);
// One-time launch set-up of the guided scatter (attributes, grid) outside stream capture.
void prepare_guide_launch();
void launch_extend(const DevScene& s, const PathState& p, int bounce, bool count, unsigned long long* stats,
                   int grid, cudaStream_t st);
// Launches the shading stage (with the material sort when it is on); how many kernels that is.
int shade_launches(const DevScene& s, const PathState& p, int bounce);
void launch_shade(const DevScene& s, const PathState& p, int bounce, int grid, cudaStream_t st);
void launch_shadow(const DevScene& s, const PathState& p, const Framebuffer& fb, int bounce, bool count,
                   unsigned long long* stats, int grid, cudaStream_t st);
void launch_flush(const DevScene& s, const PathState& p, const Framebuffer& fb, int bounce, int grid,
                  cudaStream_t st);
// End of a wave without guiding records: every path's accumulator is final, so each pixel
// of the pass range sums the RGB of its paths in the wave (its slots npix_range apart, in
// sample order) into the pass framebuffer; this replaces the wave's k_flush launches.
void launch_gather(const DevScene& s, const PathState& p, const Framebuffer& fb, const WaveArgs& w, int grid,
                   cudaStream_t st);
// Guided scenes: network evaluation and one-sample MIS scattering of the queued guided
// vertices (persistent kernel, as many CTAs as fit on the SMs).
void launch_guide(const DevScene& s, const PathState& p, int bounce, cudaStream_t st);
// Media scenes: spectral tracking from each extension ray's origin to its surface hit.
void launch_track(const DevScene& s, const PathState& p, int bounce, int grid, cudaStream_t st);
// Medium tracker at `pos` (MediumTracker::initializePosition); writes one uint2 to `out`.
void launch_init_tracker(const DevScene& s, float3 pos, float3 bb_lo, float3 bb_hi, uint2* out, unsigned int* err,
                         cudaStream_t st);
void launch_accumulate(const Framebuffer& fb, double* acc, double* light, int n3, cudaStream_t st);
void launch_intersect_rays(const DevScene& s, const float* rays, int n, int* prim, float* t, float* u, float* v,
                           unsigned int* err, cudaStream_t st);
void launch_occluded_rays(const DevScene& s, const float* rays, int n, unsigned char* occ, unsigned int* err,
                          cudaStream_t st);
void launch_count_rays(const DevScene& s, const float* rays, int n, unsigned long long* counters,
                       unsigned int* err, cudaStream_t st);
void launch_sample_bsdf(const DevScene& s, int material, float3 wi, int3 lambda, int n, unsigned long long seed,
                        float* dir, float* val, float* pdf, cudaStream_t st);
void launch_eval_bsdf(const DevScene& s, int material, float3 wi, int3 lambda, const float* dirs, int n, float* val,
                      float* pdf, cudaStream_t st);
void launch_quadtree_sample(const int4* child, const float* prob, const float* u, int n, float* dir, float* pdf,
                            float* pdf_eval, cudaStream_t st);
void launch_sample_phase(const DevScene& s, int medium, float3 pos, float3 wi, int3 lambda, int n,
                         unsigned long long seed, float* dir, float* val, float* pdf, cudaStream_t st);
void launch_eval_phase(const DevScene& s, int medium, float3 pos, float3 wi, int3 lambda, const float* dirs, int n,
                       float* val, float* pdf, cudaStream_t st);
// Blocks per SM that the shading kernel sustains (for grid sizing).
int kernel_blocks_per_sm();
// Framebuffer resolve: rgb = accum * inv_spp + splat_weight * light, per pixel.  inv_spp
// is per pixel when `inv_spp_px` is not null, else the scalar applies to all pixels.
void launch_resolve(const double* accum, const double* light, const double* inv_spp_px, double inv_spp,
                    double splat_weight, int npix, float* rgb, cudaStream_t st);

// Device memory from a per-device stream-ordered pool that keeps freed memory for reuse
// (unlimited release threshold): contexts created and destroyed in a loop do not pay for
// cudaMalloc / cudaFree of their path state each time.
cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t st);
void pool_free(void* p, cudaStream_t st);

}  // namespace tt
