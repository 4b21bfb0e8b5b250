// C ABI of the CUDA forward path tracer (include/toytrace_gpu.h): context lifetime, scene
// upload, the pass loop over wavefront waves, framebuffer readback and the batch queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/toytrace_gpu.h"
#include "tt_build.h"
#include "tt_bvh.h"
#include "tt_guide.cuh"
#include "tt_guide.h"
#include "tt_internal.h"
#include "tt_sobol_data.h"
#include "tt_tables.h"
#include "tt_quadtree.h"
#include "tt_tree.h"

using namespace tt;

namespace {

// Paths resident per wave: 2^27 paths hold about 30 GB of path state (more with media or
// guiding), a sixth of the B200's HBM; a large wave keeps every launch of the bounce loop
// full, so the latency-bound tail launches of the last bounces are paid once per 2^27 paths
// (the 1920x1080x64 frame: one wave, against 2 at 2^26 (2.6 % slower) and 32 at 2^22
// (1.6x slower)).  Path-slot indices stay below 2^31 in every array for waves up to 2^27.
// When the device cannot hold a wave, the wave is halved until it fits (down to 2^20).
constexpr int kDefaultWave = 1 << 27;

std::mutex g_err_mutex;
std::string g_create_error;

// Page-locked host memory for the contexts' scene copies, kept for reuse by later
// contexts (as the device memory pool keeps device buffers): the copies of tt_create then
// write into memory that is already mapped, and tt_upload_scene's host-to-device copies run
// as DMA from it instead of through pageable staging.  Blocks of 1 MiB and more are pinned
// (cudaHostAlloc, portable to every device), in multiples of 1 MiB; a freed block is kept
// while the pool holds at most kHostPoolKeep bytes, else released.  Smaller blocks, and all
// blocks once a pinned allocation has failed (no GPU, no driver), come from malloc.  The pool
// is never destroyed: blocks still cached at exit go with the process.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool* pool = new HostPool;
    return *pool;
  }
  void* alloc(size_t bytes) {
    constexpr size_t kMiB = 1 << 20;
    if (bytes >= kMiB) {
      const size_t rounded = (bytes + kMiB - 1) / kMiB * kMiB;
      std::lock_guard<std::mutex> g(mu_);
      auto it = free_.lower_bound(rounded);
      if (it != free_.end() && it->first <= 2 * rounded) {
        void* p = it->second;
        kept_ -= it->first;
        live_[p] = Block{it->first, true};
        free_.erase(it);
        return p;
      }
      if (pinned_ok_) {
        void* p = nullptr;
        if (cudaHostAlloc(&p, rounded, cudaHostAllocPortable) == cudaSuccess && p) {
          live_[p] = Block{rounded, true};
          return p;
        }
        cudaGetLastError();  // clear the failed call's error
        pinned_ok_ = false;
      }
    }
    void* p = std::malloc(bytes > 0 ? bytes : 1);
    if (!p) throw std::bad_alloc();
    std::lock_guard<std::mutex> g(mu_);
    live_[p] = Block{bytes, false};
    return p;
  }
  void release(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> g(mu_);
    auto it = live_.find(p);
    if (it == live_.end()) return;
    const Block b = it->second;
    live_.erase(it);
    if (!b.pinned) {
      std::free(p);
    } else if (kept_ + b.bytes <= kHostPoolKeep) {
      free_.emplace(b.bytes, p);
      kept_ += b.bytes;
    } else {
      cudaFreeHost(p);
    }
  }

 private:
  static constexpr size_t kHostPoolKeep = size_t(4) << 30;
  struct Block {
    size_t bytes;
    bool pinned;
  };
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  std::unordered_map<void*, Block> live_;
  size_t kept_ = 0;
  bool pinned_ok_ = true;
};

// Allocator of the scene copies: memory from the host pool, new elements left
// uninitialised, so that the copies of tt_create touch their pages once, from the threads
// that fill them.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  T* allocate(size_t n) { return static_cast<T*>(HostPool::get().alloc(n * sizeof(T))); }
  void deallocate(T* p, size_t) noexcept { HostPool::get().release(p); }
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T, class U>
bool operator==(const NoInitAlloc<T>&, const NoInitAlloc<U>&) noexcept {
  return true;
}
template <class T, class U>
bool operator!=(const NoInitAlloc<T>&, const NoInitAlloc<U>&) noexcept {
  return false;
}
template <class T>
using HostArray = std::vector<T, NoInitAlloc<T>>;

struct HostEnv {
  tt_env_light desc;
  HostArray<float> tex;
  HostArray<float> cmf_rows, cmf_cols;  // made at upload; kept until tt_destroy (DMA sources)
  HostArray<int> guide_rows, guide_cols;
};

// Guide table of a CMF (see kEnvGuide): guide[g] = the first index i with cmf[i] > g / kEnvGuide
// (n when there is none), for g = 0 .. kEnvGuide, by one merged sweep.
static void cmf_guide(const float* cmf, int n, int* guide) {
  int i = 0;
  for (int g = 0; g <= kEnvGuide; ++g) {
    const float u = (float)g / (float)kEnvGuide;
    while (i < n && !(cmf[i] > u)) ++i;
    guide[g] = i;
  }
}

// Device buffers owned by a context, from the library's memory pool, ordered on `stream`.
struct DeviceBuffers {
  std::vector<void*> allocs;
  cudaStream_t stream = nullptr;
  void* alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (pool_malloc(&p, bytes, stream) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return p;
  }
  void free_all() {
    for (void* p : allocs) pool_free(p, stream);
    allocs.clear();
  }
};

std::mutex g_pool_mutex;
cudaMemPool_t g_pools[64] = {nullptr};

// Primitive ids 0 .. n - 1 (the surface set of a mesh without medium boundaries).
__global__ void k_iota(uint32_t* out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

// Per global primitive: vertex indices and material (spheres after the triangles: material
// only), from the mesh as uploaded for the device BVH build.
__global__ void k_prim_table(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ mats, uint32_t ntri,
                             const uint32_t* __restrict__ sphere_mats, uint32_t nsph, uint4* __restrict__ out) {
  const uint32_t n = ntri + nsph;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = i < ntri ? make_uint4(idx[3 * (size_t)i], idx[3 * (size_t)i + 1], idx[3 * (size_t)i + 2], mats[i])
                      : make_uint4(0u, 0u, 0u, sphere_mats[i - ntri]);
}

__global__ void k_tally(const int* counters, int rounds, unsigned long long* stats) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long e = 0, s = 0;
    for (int b = 0; b <= rounds; ++b) {
      e += (unsigned long long)counters[kCountersPerBounce * b];
      s += (unsigned long long)counters[kCountersPerBounce * b + 1];
    }
    stats[4] += e;
    stats[5] += s;
  }
}

}  // namespace

namespace tt {
cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&g_pools[dev], &props);
      if (e != cudaSuccess) {
        g_pools[dev] = nullptr;
        return e;
      }
      uint64_t threshold = UINT64_MAX;
      cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &threshold);
    }
  }
  return cudaMallocFromPoolAsync(p, bytes, g_pools[dev], st);
}
void pool_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}
}  // namespace tt

struct tt_ctx {
  // Host copy of the scene.
  HostArray<float> verts, normals;
  HostArray<uint32_t> idx, mats;
  std::vector<tt_material> materials;
  std::vector<tt_medium> media;
  std::vector<std::vector<float>> media_tables;  // per medium: sigma_t, molecules, aerosols (rows x 36 each)
  std::vector<float> spheres;                    // 4 per sphere
  std::vector<uint32_t> sphere_mats;
  std::vector<HostEnv> envs;
  std::vector<tt_point_light> points;
  HostArray<float> uvs;                          // 2 per vertex, when given
  std::vector<float> views_done_ms;              // per view of the last multi-view batch: completion time
  std::vector<std::vector<float>> textures;      // linear RGB per texture
  std::vector<int2> texture_sizes;               // width, height
  tt_camera camera{};
  tt_params params{};
  int npix = 0;
  bool uploaded = false;
  // Device state.
  int device = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffers scene_mem, path_mem;
  DevScene dev{};
  PathState ps{};
  Framebuffer fb{};
  double* d_acc = nullptr;
  double* d_light = nullptr;
  unsigned long long* d_stats = nullptr;  // 0..3 traversal counts, 4 ext rays, 5 shadow rays
  unsigned int* d_err = nullptr;
  int grid = 0;
  int wave_cap = 0;
  int rounds = 0;
  // Accumulation bookkeeping.
  std::vector<uint64_t> spp_count;
  uint64_t splat_count = 0;
  uint64_t next_sample = 0;
  // Control.
  std::atomic<int> stop{0};
  std::atomic<int> interrupt{0};
  int profiling = 0;
  tt_stats stats{};
  std::string err;
  uint32_t bvh_nodes = 0, bvh_depth = 0, bvh_node_bytes = 64;
  // The two BVH layouts the autotuner can choose between: [0] the device-built tree (binary,
  // with its 4-wide collapse when built), [1] 8-wide compressed (built on the host on the
  // autotuner's first request).  Slot arrays belong to a layout.
  struct Layout {
    bool ready = false;
    const float4* nodes = nullptr;
    const float4* nodes4 = nullptr;
    const uint4* nodes8 = nullptr;
    const float4* tris = nullptr;
    const float4* vnodes = nullptr;
    const uint4* vnodes8 = nullptr;
    const float4* vtris = nullptr;
    uint32_t num_nodes = 0, depth = 0, node_bytes = 0;
  } layouts[2];
  // Learned guiding.
  std::unique_ptr<GuideNet> gnet;
  std::unique_ptr<TreeGuide> tree;   // tree guider (method TT_GUIDE_TREE)
  tt_guiding_params gparams{};
  GuideRecord* d_records = nullptr;   // record pool (ring)
  int* d_rec_count = nullptr;
  int rec_cap = 0;
  long long rec_seen = 0;             // pool counter at the end of the last pass
  double rec_rate = 0.0;              // records committed per path in the last training pass
  uint64_t draw_seed = 0;
  bool ps_guided = false;      // the path state carries the guiding arrays
  float bb_lo[3] = {0, 0, 0}, bb_hi[3] = {0, 0, 0};  // scene bounds (medium trackers of views)
};

// Runs f(lo, hi) over [0, n) split among up to 16 host threads (serially below 4096).
template <class F>
static void parallel_ranges(long long n, F&& f, long long serial_below = 4096) {
  const long long nt = std::min<long long>(16, std::max(1u, std::thread::hardware_concurrency()));
  if (n < serial_below || nt <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  const long long chunk = (n + nt - 1) / nt;
  for (long long lo = 0; lo < n; lo += chunk) th.emplace_back([&f, lo, hi = std::min(n, lo + chunk)] { f(lo, hi); });
  for (auto& t : th) t.join();
}

// dst = src[0 .. n), copied by parallel_ranges' threads.
template <class T>
static void parallel_copy(HostArray<T>& dst, const T* src, size_t n) {
  dst.resize(n);
  parallel_ranges((long long)n, [&](long long lo, long long hi) {
    std::memcpy(dst.data() + lo, src + lo, (size_t)(hi - lo) * sizeof(T));
  });
}

static tt_status fail(tt_ctx* c, tt_status s, const std::string& msg) {
  if (c) c->err = msg;
  else {
    std::lock_guard<std::mutex> g(g_err_mutex);
    g_create_error = msg;
  }
  return s;
}

// Generator matrices of the quasi-random sampler, 32 columns per dimension, each column
// left-aligned to bit 31 (sampler.cxx:224-251).  Dimension 0 is the van der Corput
// sequence.  Dimension d >= 1 takes (s, a, m_1..m_s) from the Joe-Kuo table and extends
// the m's by the recurrence of the reference's generator (misc/
// SobolSequenceGeneratorMatrices.ipynb, MakeTheMatrix): m_k = m_{k-s} ^ (m_{k-s} << s)
// ^ the sum over i < s - 1 of bit (s - 2 - i) of a times m_{k-s+i+1} << (s - 1 - i).
// (Joe and Kuo pair a's most significant bit with m_{k-1}; the reference pairs it with
// m_{k-s+1}.  The two agree for s <= 2, and the matrices here follow the reference.)
static void build_sobol_matrices(std::vector<uint32_t>* out) {
  static_assert(TT_SOBOL_DIMS == kSobolDims && TT_ROTATION_BLOCK == kRotationBlock, "table sizes");
  out->assign((size_t)kSobolDims * 32, 0u);
  uint32_t* C = out->data();
  for (int k = 0; k < 32; ++k) C[k] = 1u << (31 - k);
  size_t pos = 0;
  for (int d = 1; d < kSobolDims; ++d) {
    const int s = tt_sobol_sam[pos], a = tt_sobol_sam[pos + 1];
    const uint16_t* m = tt_sobol_sam + pos + 2;
    pos += 2 + (size_t)s;
    uint64_t mk[32];
    for (int k = 0; k < 32; ++k) {
      if (k < s) {
        mk[k] = m[k];
        continue;
      }
      uint64_t v = mk[k - s] ^ (mk[k - s] << s);
      for (int i = 0; i < s - 1; ++i)
        if ((a >> (s - 2 - i)) & 1) v ^= mk[k - s + i + 1] << (s - 1 - i);
      mk[k] = v;
    }
    for (int k = 0; k < 32; ++k) C[32 * (size_t)d + k] = (uint32_t)(mk[k] << (31 - k));
  }
}

#define TT_CUDA(ctx, call)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(ctx, TT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// OrthogonalSystemZAligned in double (vec3f.hxx:240-258); writes columns X, Y, Z.
static void frame_z_d(const double z[3], float X[3], float Y[3], float Z[3]) {
  const double sign = std::copysign(1.0, z[2]);
  const double a = -1.0 / (sign + z[2]);
  const double b = z[0] * z[1] * a;
  const double x[3] = {1.0 + sign * z[0] * z[0] * a, sign * b, -sign * z[0]};
  const double y[3] = {b, sign + z[1] * z[1] * a, -z[1]};
  for (int k = 0; k < 3; ++k) { X[k] = (float)x[k]; Y[k] = (float)y[k]; Z[k] = (float)z[k]; }
}

static void normalize_d(double v[3]) {
  const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  for (int k = 0; k < 3; ++k) v[k] /= l;
}

// Camera frame and pixel geometry (camera.hxx:38-108, 159-175), computed in double.
static DevCamera make_dev_camera(const tt_camera& cm) {
  DevCamera cam{};
  cam.kind = cm.kind;
  cam.xres = cm.xres;
  cam.yres = cm.yres;
  double up[3] = {cm.up[0], cm.up[1], cm.up[2]}, dir[3] = {cm.dir[0], cm.dir[1], cm.dir[2]};
  normalize_d(up);
  normalize_d(dir);
  const double r = up[0] * dir[0] + up[1] * dir[1] + up[2] * dir[2];
  if (!(std::fabs(r) > 1.0 - 2.220446049250313e-16)) {
    for (int k = 0; k < 3; ++k) up[k] -= r * dir[k];
    normalize_d(up);
  }
  const double right[3] = {up[1] * dir[2] - up[2] * dir[1], up[2] * dir[0] - up[0] * dir[2],
                           up[0] * dir[1] - up[1] * dir[0]};
  for (int k = 0; k < 3; ++k) {
    cam.pos[k] = cm.pos[k];
    cam.up[k] = (float)up[k];
    cam.dir[k] = (float)dir[k];
    cam.right[k] = (float)right[k];
  }
  const double fov = cm.fov_deg * M_PI / 180.;
  const double aspect = (double)cm.yres / cm.xres;
  const double a = std::tan(fov * 0.5), b = a * aspect;
  cam.xmin = (float)-a;
  cam.ymin = (float)-b;
  cam.xperpixel = (float)(2. * a / cm.xres);
  cam.yperpixel = (float)(2. * b / cm.yres);
  cam.per_pixel_delta = (float)(2. / std::min(cm.xres, cm.yres));
  return cam;
}

extern "C" {

int32_t tt_abi_version(void) { return TT_ABI_VERSION; }

tt_status tt_create(const tt_scene_desc* d, const tt_params* p, tt_ctx** out) {
  if (!out) return fail(nullptr, TT_ERR_INVALID, "tt_create: out_ctx is NULL");
  *out = nullptr;
  if (!d || !p) return fail(nullptr, TT_ERR_INVALID, "tt_create: scene or params is NULL");
  if (d->num_triangles > (1u << 28)) return fail(nullptr, TT_ERR_CAPACITY, "more than 2^28 triangles");
  if (d->num_triangles > 0 && (!d->vertices || !d->indices || !d->material_ids))
    return fail(nullptr, TT_ERR_INVALID, "triangle arrays missing");
  if (d->num_materials > 0 && !d->materials) return fail(nullptr, TT_ERR_INVALID, "materials missing");
  if (d->camera.xres <= 0 || d->camera.yres <= 0) return fail(nullptr, TT_ERR_INVALID, "bad camera resolution");
  if ((int64_t)d->camera.xres * d->camera.yres > (1ll << 30)) return fail(nullptr, TT_ERR_CAPACITY, "too many pixels");
  if (d->num_env_lights > (uint32_t)MAX_ENV_LIGHTS) return fail(nullptr, TT_ERR_CAPACITY, "too many env lights");
  if (p->pt_sample_mode < 0 || p->pt_sample_mode > 2) return fail(nullptr, TT_ERR_INVALID, "bad pt_sample_mode");
  if (p->algo != TT_ALGO_PT && p->algo != TT_ALGO_PT2) return fail(nullptr, TT_ERR_INVALID, "unknown algo");
  if (p->algo == TT_ALGO_PT2 && p->qmc && (p->max_ray_depth <= 0 ? 25 : p->max_ray_depth) > 31)
    return fail(nullptr, TT_ERR_INVALID, "qmc needs max_ray_depth <= 31 (64 sampler subsequences)");
  if (p->max_ray_depth > 1000) return fail(nullptr, TT_ERR_INVALID, "max_ray_depth above 1000");
  {
    // The first triangle with an index out of range (threads keep the smallest they see).
    std::atomic<long long> bad{(long long)d->num_triangles};
    parallel_ranges(d->num_triangles, [&](long long lo, long long hi) {
      for (long long t = lo; t < hi && t < bad.load(std::memory_order_relaxed); ++t) {
        const uint32_t* v = d->indices + 3 * (size_t)t;
        if (v[0] >= d->num_vertices || v[1] >= d->num_vertices || v[2] >= d->num_vertices ||
            d->material_ids[t] >= d->num_materials) {
          long long cur = bad.load();
          while (t < cur && !bad.compare_exchange_weak(cur, t)) {
          }
          break;
        }
      }
    });
    const long long t = bad.load();
    if (t < (long long)d->num_triangles) {
      const uint32_t* v = d->indices + 3 * (size_t)t;
      if (v[0] >= d->num_vertices || v[1] >= d->num_vertices || v[2] >= d->num_vertices)
        return fail(nullptr, TT_ERR_INVALID, "vertex index out of range in triangle " + std::to_string(t));
      return fail(nullptr, TT_ERR_INVALID, "material index out of range in triangle " + std::to_string(t));
    }
  }
  for (uint32_t i = 0; i < d->num_materials; ++i) {
    const tt_material& m = d->materials[i];
    if (m.shader < TT_SHADER_DIFFUSE || m.shader > TT_SHADER_SPECULAR_DENSE_DIELECTRIC)
      return fail(nullptr, TT_ERR_INVALID, "unknown shader kind in material " + std::to_string(i));
    if ((m.shader == TT_SHADER_MICROFACET || m.shader == TT_SHADER_GLOSSY_DIELECTRIC) && !(m.alpha > 0.f))
      return fail(nullptr, TT_ERR_INVALID, "microfacet roughness must be positive");
    if ((m.shader == TT_SHADER_SPECULAR_DIELECTRIC || m.shader == TT_SHADER_GLOSSY_DIELECTRIC) && !(m.ior_ratio > 0.f))
      return fail(nullptr, TT_ERR_INVALID, "dielectric ior_ratio must be positive");
    if (m.medium_inside < 0 || m.medium_inside > (int)d->num_media || m.medium_outside < 0 ||
        m.medium_outside > (int)d->num_media)
      return fail(nullptr, TT_ERR_INVALID, "medium index out of range in material " + std::to_string(i));
    if (m.diffuse_texture < 0 || m.diffuse_texture > (int)d->num_textures)
      return fail(nullptr, TT_ERR_INVALID, "texture index out of range in material " + std::to_string(i));
    if (m.diffuse_texture > 0 && m.shader != TT_SHADER_DIFFUSE && m.shader != TT_SHADER_SPECULAR_DENSE_DIELECTRIC)
      return fail(nullptr, TT_ERR_INVALID, "a texture needs a diffuse base (material " + std::to_string(i) + ")");
    if (m.shader == TT_SHADER_SPECULAR_DENSE_DIELECTRIC &&
        !(m.specular_reflectivity >= 0.f && m.specular_reflectivity <= 1.f))
      return fail(nullptr, TT_ERR_INVALID, "dense dielectric reflectivity must lie in [0, 1]");
  }
  if (d->num_media > 0 && !d->media) return fail(nullptr, TT_ERR_INVALID, "media missing");
  if (d->num_spheres > (1u << 26)) return fail(nullptr, TT_ERR_CAPACITY, "more than 2^26 spheres");
  if (d->num_spheres > 0 && (!d->spheres || !d->sphere_material_ids))
    return fail(nullptr, TT_ERR_INVALID, "sphere arrays missing");
  for (uint32_t i = 0; i < d->num_spheres; ++i) {
    const float* q = d->spheres + 4 * (size_t)i;
    if (!std::isfinite(q[0]) || !std::isfinite(q[1]) || !std::isfinite(q[2]) || !(q[3] > 0.f) || !std::isfinite(q[3]))
      return fail(nullptr, TT_ERR_INVALID, "sphere " + std::to_string(i) + " needs a finite centre and positive radius");
    if (d->sphere_material_ids[i] >= d->num_materials)
      return fail(nullptr, TT_ERR_INVALID, "material index out of range in sphere " + std::to_string(i));
  }
  if (d->num_textures > 0 && !d->textures) return fail(nullptr, TT_ERR_INVALID, "textures missing");
  for (uint32_t i = 0; i < d->num_textures; ++i) {
    const tt_texture& t = d->textures[i];
    if (!t.rgb || t.width <= 0 || t.height <= 0 || (long long)t.width * t.height > (1ll << 28))
      return fail(nullptr, TT_ERR_INVALID, "texture " + std::to_string(i) + " needs pixels and a positive size");
  }
  if (d->uvs)
    for (size_t k = 0; k < 2 * (size_t)d->num_vertices; ++k)
      if (!std::isfinite(d->uvs[k])) return fail(nullptr, TT_ERR_INVALID, "texture coordinates must be finite");
  if (d->num_media > (uint32_t)kMaxMedia) return fail(nullptr, TT_ERR_CAPACITY, "more than 254 media");
  for (uint32_t i = 0; i < d->num_media; ++i) {
    const tt_medium& m = d->media[i];
    if (m.kind == TT_MEDIUM_ATMOSPHERE) {
      if (m.table_size < 2 || !m.sigma_t || !m.sigma_s_molecules || !m.sigma_s_aerosols)
        return fail(nullptr, TT_ERR_INVALID, "atmosphere " + std::to_string(i) + " needs tables of at least 2 rows");
      if (!(m.table_dh > 0.f) || !(m.planet_radius > 0.f) || !(std::fabs(m.phase_g) < 1.f))
        return fail(nullptr, TT_ERR_INVALID, "atmosphere needs positive row spacing and radius and |g| < 1");
      const float* tabs[3] = {m.sigma_t, m.sigma_s_molecules, m.sigma_s_aerosols};
      for (const float* t : tabs)
        for (size_t k = 0; k < (size_t)m.table_size * NBINS; ++k)
          if (!(t[k] >= 0.f) || !std::isfinite(t[k]))
            return fail(nullptr, TT_ERR_INVALID, "atmosphere tables must be finite and non-negative");
      continue;
    }
    if (m.kind != TT_MEDIUM_HOMOGENEOUS) return fail(nullptr, TT_ERR_INVALID, "unknown medium kind");
    if (m.phase < TT_PHASE_UNIFORM || m.phase > TT_PHASE_HENYEY_GREENSTEIN)
      return fail(nullptr, TT_ERR_INVALID, "unknown phase function in medium " + std::to_string(i));
    if (m.phase == TT_PHASE_HENYEY_GREENSTEIN && !(std::fabs(m.phase_g) < 1.f))
      return fail(nullptr, TT_ERR_INVALID, "Henyey-Greenstein g must lie in (-1, 1)");
    for (int b = 0; b < NBINS; ++b)
      if (!(m.sigma_s[b] >= 0.f) || !(m.sigma_a[b] >= 0.f) || !std::isfinite(m.sigma_s[b] + m.sigma_a[b]))
        return fail(nullptr, TT_ERR_INVALID, "medium coefficients must be finite and non-negative");
  }
  auto* c = new tt_ctx;
  parallel_copy(c->verts, d->vertices, 3 * (size_t)d->num_vertices);
  if (d->normals) parallel_copy(c->normals, d->normals, 3 * (size_t)d->num_vertices);
  parallel_copy(c->idx, d->indices, 3 * (size_t)d->num_triangles);
  parallel_copy(c->mats, d->material_ids, (size_t)d->num_triangles);
  c->materials.assign(d->materials, d->materials + d->num_materials);
  if (d->num_media > 0) c->media.assign(d->media, d->media + d->num_media);
  for (auto& m : c->media) {
    std::vector<float> tab;
    if (m.kind == TT_MEDIUM_ATMOSPHERE) {
      const size_t n = (size_t)m.table_size * NBINS;
      tab.insert(tab.end(), m.sigma_t, m.sigma_t + n);
      tab.insert(tab.end(), m.sigma_s_molecules, m.sigma_s_molecules + n);
      tab.insert(tab.end(), m.sigma_s_aerosols, m.sigma_s_aerosols + n);
    }
    m.sigma_t = m.sigma_s_molecules = m.sigma_s_aerosols = nullptr;
    c->media_tables.push_back(std::move(tab));
  }
  if (d->num_spheres > 0) {
    c->spheres.assign(d->spheres, d->spheres + 4 * (size_t)d->num_spheres);
    c->sphere_mats.assign(d->sphere_material_ids, d->sphere_material_ids + d->num_spheres);
  }
  for (uint32_t i = 0; i < d->num_env_lights; ++i) {
    HostEnv e;
    e.desc = d->env_lights[i];
    if (e.desc.kind < TT_ENV_DOME || e.desc.kind > TT_ENV_DIRECTIONAL) {
      delete c;
      return fail(nullptr, TT_ERR_INVALID, "unknown env light kind");
    }
    if (e.desc.kind == TT_ENV_MAP) {
      if (!e.desc.tex_rgb || e.desc.tex_width <= 0 || e.desc.tex_height <= 0) {
        delete c;
        return fail(nullptr, TT_ERR_INVALID, "env map without texture");
      }
      parallel_copy(e.tex, e.desc.tex_rgb, 3 * (size_t)e.desc.tex_width * e.desc.tex_height);
      e.desc.tex_rgb = nullptr;
    }
    c->envs.push_back(std::move(e));
  }
  if (d->num_point_lights > 0) c->points.assign(d->point_lights, d->point_lights + d->num_point_lights);
  if (d->uvs) parallel_copy(c->uvs, d->uvs, 2 * (size_t)d->num_vertices);
  for (uint32_t i = 0; i < d->num_textures; ++i) {
    const tt_texture& t = d->textures[i];
    c->textures.emplace_back(t.rgb, t.rgb + 3 * (size_t)t.width * t.height);
    c->texture_sizes.push_back(make_int2(t.width, t.height));
  }
  c->camera = d->camera;
  c->params = *p;
  if (c->params.max_ray_depth <= 0) c->params.max_ray_depth = 25;
  c->npix = d->camera.xres * d->camera.yres;
  c->device = p->device;
  c->spp_count.assign(c->npix, 0);
  *out = c;
  return TT_OK;
}

// The scene split into surface and medium-boundary inputs for the host BVH builders
// (Scene::BuildAccelStructure's two scenes, scene.cxx:116-141).
struct HostSplit {
  std::vector<uint32_t> sidx, smat, sid, vidx, vmat, vid, ssmat, ssid, vsmat, vsid;
  std::vector<float> ssph, vsph;
  void make(const tt_ctx* c) {
    const uint32_t ntri = (uint32_t)c->mats.size();
    for (uint32_t t = 0; t < ntri; ++t) {
      const bool vol = c->materials[c->mats[t]].volume_boundary != 0;
      (vol ? vid : sid).push_back(t);
      (vol ? vidx : sidx).insert((vol ? vidx : sidx).end(), &c->idx[3 * (size_t)t], &c->idx[3 * (size_t)t] + 3);
      (vol ? vmat : smat).push_back(c->mats[t]);
    }
    for (uint32_t i = 0; i < (uint32_t)c->sphere_mats.size(); ++i) {
      const bool vol = c->materials[c->sphere_mats[i]].volume_boundary != 0;
      (vol ? vsph : ssph).insert((vol ? vsph : ssph).end(), &c->spheres[4 * (size_t)i], &c->spheres[4 * (size_t)i] + 4);
      (vol ? vsmat : ssmat).push_back(c->sphere_mats[i]);
      (vol ? vsid : ssid).push_back(ntri + i);
    }
  }
  BvhInput surface(const tt_ctx* c) const {
    BvhInput b{c->verts.data(), sidx.data(), smat.data(), (uint32_t)sid.size(), sid.data()};
    b.num_spheres = (uint32_t)ssid.size();
    b.spheres = ssph.data();
    b.sphere_material_ids = ssmat.data();
    b.sphere_prim_ids = ssid.data();
    return b;
  }
  BvhInput volume(const tt_ctx* c) const {
    BvhInput b{c->verts.data(), vidx.data(), vmat.data(), (uint32_t)vid.size(), vid.data()};
    b.num_spheres = (uint32_t)vsid.size();
    b.spheres = vsph.data();
    b.sphere_material_ids = vsmat.data();
    b.sphere_prim_ids = vsid.data();
    return b;
  }
};

static void save_layout(tt_ctx* c) {
  tt_ctx::Layout& L = c->layouts[c->dev.wide ? 1 : 0];
  L.ready = true;
  L.nodes = c->dev.nodes;
  L.nodes4 = c->dev.nodes4;
  L.nodes8 = c->dev.nodes8;
  L.tris = c->dev.tris;
  L.vnodes = c->dev.vnodes;
  L.vnodes8 = c->dev.vnodes8;
  L.vtris = c->dev.vtris;
  L.num_nodes = c->bvh_nodes;
  L.depth = c->bvh_depth;
  L.node_bytes = c->bvh_node_bytes;
}

// Makes `wide` the active BVH layout, building the 8-wide one on the host the first time.
static tt_status use_layout(tt_ctx* c, bool wide) {
  if ((c->dev.wide != 0) == wide) return TT_OK;
  save_layout(c);
  tt_ctx::Layout& L = c->layouts[wide ? 1 : 0];
  if (!L.ready) {
    if (!wide) return fail(c, TT_ERR_INVALID, "binary BVH layout missing");
    HostSplit hs;
    hs.make(c);
    Bvh8Output bo, vbo;
    if (!build_bvh8(hs.surface(c), &bo) || !build_bvh8(hs.volume(c), &vbo))
      return fail(c, TT_ERR_INVALID, "8-wide BVH build failed");
    if (bo.max_depth + 2 >= (uint32_t)BVH8_STACK || vbo.max_depth + 2 >= (uint32_t)BVH8_STACK)
      return fail(c, TT_ERR_CAPACITY, "BVH deeper than the traversal stack");
    auto up = [&](const void* src, size_t bytes) -> void* {
      void* p = c->scene_mem.alloc(bytes);
      if (p && bytes) cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, c->stream);
      return p;
    };
    L.nodes8 = (const uint4*)up(bo.nodes.data(), bo.nodes.size() * sizeof(uint32_t));
    L.tris = (const float4*)up(bo.tris.data(), bo.tris.size() * sizeof(float));
    L.vnodes8 = (const uint4*)up(vbo.nodes.data(), vbo.nodes.size() * sizeof(uint32_t));
    L.vtris = (const float4*)up(vbo.tris.data(), vbo.tris.size() * sizeof(float));
    L.num_nodes = bo.num_nodes;
    L.depth = bo.max_depth;
    L.node_bytes = 80;
    L.ready = true;
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
    TT_CUDA(c, cudaGetLastError());
  }
  c->dev.wide = wide ? 1 : 0;
  c->dev.nodes = L.nodes;
  c->dev.nodes4 = L.nodes4;
  c->dev.nodes8 = L.nodes8;
  c->dev.tris = L.tris;
  c->dev.vnodes = L.vnodes;
  c->dev.vnodes8 = L.vnodes8;
  c->dev.vtris = L.vtris;
  c->bvh_nodes = L.num_nodes;
  c->bvh_depth = L.depth;
  c->bvh_node_bytes = L.node_bytes;
  return TT_OK;
}

tt_status tt_upload_scene(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  TT_CUDA(c, cudaSetDevice(c->device));
  if (c->uploaded) return TT_OK;
  const auto t_enter = std::chrono::steady_clock::now();
  TT_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->scene_mem.stream = c->stream;
  c->path_mem.stream = c->stream;
  upload_constant_tables();
  TT_CUDA(c, cudaGetLastError());
  // TT_UPLOAD_TIMING=1 prints the time of the upload's phases to stderr, each phase ended
  // by a stream synchronisation; TT_UPLOAD_TIMING=2 prints the host time of each phase
  // without synchronising (queued device work then counts where the host waits for it).
  const char* tm_env = std::getenv("TT_UPLOAD_TIMING");
  const bool tm = tm_env != nullptr;
  const bool tm_sync = tm && std::atoi(tm_env) != 2;
  auto t_last = t_enter;
  auto mark = [&](const char* what) {
    if (!tm) return;
    if (tm_sync) cudaStreamSynchronize(c->stream);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "upload %-12s %8.2f ms\n", what, std::chrono::duration<double, std::milli>(now - t_last).count());
    t_last = now;
  };
  mark("stream+consts");
  const uint32_t ntri = (uint32_t)c->mats.size();
  // Surfaces and medium boundaries go into separate BVHs (Scene::BuildAccelStructure,
  // scene.cxx:116-141); both store global triangle ids in their slots.
  std::vector<uint32_t> sidx, smat, sid, vidx, vmat, vid;
  bool any_vol = false;
  for (const auto& m : c->materials) any_vol |= m.volume_boundary != 0;
  // Without medium boundaries every triangle is a surface and the surface ids are the
  // identity: the device build writes them itself, the host builders get them listed.
  if (any_vol)
    for (uint32_t t = 0; t < ntri; ++t) (c->materials[c->mats[t]].volume_boundary ? vid : sid).push_back(t);
  const size_t nsurf = any_vol ? sid.size() : ntri;
  // Index and material lists per BVH for the host builders (the device builder reads the
  // mesh as uploaded, with the prim-id sets above).
  auto host_split = [&]() {
    if (!any_vol) {
      sid.resize(ntri);
      std::iota(sid.begin(), sid.end(), 0u);
    }
    for (uint32_t t : sid) {
      sidx.insert(sidx.end(), &c->idx[3 * (size_t)t], &c->idx[3 * (size_t)t] + 3);
      smat.push_back(c->mats[t]);
    }
    for (uint32_t t : vid) {
      vidx.insert(vidx.end(), &c->idx[3 * (size_t)t], &c->idx[3 * (size_t)t] + 3);
      vmat.push_back(c->mats[t]);
    }
  };
  std::vector<float> ssph, vsph;
  std::vector<uint32_t> ssmat, ssid, vsmat, vsid;
  const uint32_t nsph = (uint32_t)c->sphere_mats.size();
  for (uint32_t i = 0; i < nsph; ++i) {
    const bool vol = c->materials[c->sphere_mats[i]].volume_boundary != 0;
    (vol ? vsph : ssph).insert((vol ? vsph : ssph).end(), &c->spheres[4 * (size_t)i], &c->spheres[4 * (size_t)i] + 4);
    (vol ? vsmat : ssmat).push_back(c->sphere_mats[i]);
    (vol ? vsid : ssid).push_back(ntri + i);
  }
  mark("split");
  auto host_inputs = [&](BvhInput* bi, BvhInput* vbi) {
    host_split();
    *bi = BvhInput{c->verts.data(), sidx.data(), smat.data(), (uint32_t)sid.size(), sid.data()};
    bi->num_spheres = (uint32_t)ssid.size();
    bi->spheres = ssph.data();
    bi->sphere_material_ids = ssmat.data();
    bi->sphere_prim_ids = ssid.data();
    *vbi = BvhInput{c->verts.data(), vidx.data(), vmat.data(), (uint32_t)vid.size(), vid.data()};
    vbi->num_spheres = (uint32_t)vsid.size();
    vbi->spheres = vsph.data();
    vbi->sphere_material_ids = vsmat.data();
    vbi->sphere_prim_ids = vsid.data();
  };
  auto upload = [&](const void* src, size_t bytes) -> void* {
    void* p = c->scene_mem.alloc(bytes);
    if (p && bytes) cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, c->stream);
    return p;
  };
  DevScene& s = c->dev;
  s.tri_idx = nullptr;  // set below, by the device build or from the host table
  // The default layout is the device-built tree with four children per node (the binary
  // tree collapsed on the device; its traversal fetches half as many nodes per ray: 6 % less
  // closest-hit time than the binary tree on the terrain workload);
  // TT_BVH_WIDTH=2 keeps the binary layout, TT_BVH_WIDTH=8 selects the 8-wide compressed BVH
  // (80-byte nodes, about half the bytes per ray but more arithmetic per node, which
  // measured slower on the terrain workload).
  const char* width_env = std::getenv("TT_BVH_WIDTH");
  s.wide = width_env && std::atoi(width_env) == 8;
  const bool binary_only = width_env && std::atoi(width_env) == 2;
  s.nodes4 = nullptr;
  // The binary BVH is built on the device (PLOC) unless TT_BVH_BUILD=host asks for the
  // host binned-SAH builder.
  const char* build_env = std::getenv("TT_BVH_BUILD");
  if (s.wide) {
    BvhInput bi{}, vbi{};
    host_inputs(&bi, &vbi);
    Bvh8Output bo, vbo;
    if (!build_bvh8(bi, &bo)) return fail(c, TT_ERR_INVALID, "BVH build failed");
    if (!build_bvh8(vbi, &vbo)) return fail(c, TT_ERR_INVALID, "medium-boundary BVH build failed");
    c->bvh_nodes = bo.num_nodes;
    c->bvh_depth = bo.max_depth;
    c->bvh_node_bytes = 80;
    if (bo.max_depth + 2 >= (uint32_t)BVH8_STACK || vbo.max_depth + 2 >= (uint32_t)BVH8_STACK)
      return fail(c, TT_ERR_CAPACITY, "BVH deeper than the traversal stack");
    s.nodes8 = (const uint4*)upload(bo.nodes.data(), bo.nodes.size() * sizeof(uint32_t));
    s.tris = (const float4*)upload(bo.tris.data(), bo.tris.size() * sizeof(float));
    s.vnodes8 = (const uint4*)upload(vbo.nodes.data(), vbo.nodes.size() * sizeof(uint32_t));
    s.vtris = (const float4*)upload(vbo.tris.data(), vbo.tris.size() * sizeof(float));
  } else if (!(build_env && std::string(build_env) == "host")) {
    // Build on the device: the mesh goes up once, the tree is built next to it.
    DeviceBuffers tmp;
    tmp.stream = c->stream;
    auto up = [&](const void* src, size_t bytes) -> void* {
      void* p = tmp.alloc(bytes);
      if (p && bytes) cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, c->stream);
      return p;
    };
    // Prim-id sets: the triangle ids, then the sphere ids (generated on the device when the
    // surface set is every triangle).
    const size_t ns = nsurf + ssid.size(), nv = vid.size() + vsid.size();
    uint32_t* d_sset = (uint32_t*)tmp.alloc(ns * sizeof(uint32_t));
    uint32_t* d_vset = (uint32_t*)tmp.alloc(nv * sizeof(uint32_t));
    if (d_sset) {
      if (!any_vol) {
        if (ntri) k_iota<<<std::min<uint32_t>(4096, (ntri + 255) / 256), 256, 0, c->stream>>>(d_sset, ntri);
      } else if (!sid.empty()) {
        cudaMemcpyAsync(d_sset, sid.data(), sid.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
      }
      if (!ssid.empty())
        cudaMemcpyAsync(d_sset + nsurf, ssid.data(), ssid.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                        c->stream);
    }
    if (d_vset) {
      if (!vid.empty())
        cudaMemcpyAsync(d_vset, vid.data(), vid.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
      if (!vsid.empty())
        cudaMemcpyAsync(d_vset + vid.size(), vsid.data(), vsid.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                        c->stream);
    }
    BuildInput in{};
    in.vertices = (const float*)up(c->verts.data(), c->verts.size() * sizeof(float));
    in.indices = (const uint32_t*)up(c->idx.data(), c->idx.size() * sizeof(uint32_t));
    in.material_ids = (const uint32_t*)up(c->mats.data(), c->mats.size() * sizeof(uint32_t));
    in.num_triangles = ntri;
    in.spheres = (const float*)up(c->spheres.data(), c->spheres.size() * sizeof(float));
    in.sphere_material_ids = (const uint32_t*)up(c->sphere_mats.data(), c->sphere_mats.size() * sizeof(uint32_t));
    mark("mesh H2D");
    for (void* p : tmp.allocs)
      if (!p) {
        tmp.free_all();
        return fail(c, TT_ERR_CUDA, "device allocation failed");
      }
    DeviceBvh sb{}, vb{};
    std::string berr;
    mark("mesh check");
    in.prim_ids = d_sset;
    bool built = device_build_bvh2(in, d_sset, (uint32_t)ns, &sb, c->stream, &berr);
    if (sb.nodes) c->scene_mem.allocs.push_back(sb.nodes);
    if (sb.tris) c->scene_mem.allocs.push_back(sb.tris);
    if (built) {
      in.prim_ids = d_vset;
      built = device_build_bvh2(in, d_vset, (uint32_t)nv, &vb, c->stream, &berr);
      if (vb.nodes) c->scene_mem.allocs.push_back(vb.nodes);
      if (vb.tris) c->scene_mem.allocs.push_back(vb.tris);
    }
    mark("device build");
    // The primitive table from the uploaded mesh, before the mesh's buffers go.
    if (built) {
      uint4* table = (uint4*)c->scene_mem.alloc(((size_t)ntri + nsph) * sizeof(uint4));
      if (table && ntri + nsph > 0)
        k_prim_table<<<std::min<uint32_t>(4096, (ntri + nsph + 255) / 256), 256, 0, c->stream>>>(
            in.indices, in.material_ids, ntri, in.sphere_material_ids, nsph, table);
      s.tri_idx = table;
    }
    cudaStreamSynchronize(c->stream);
    tmp.free_all();
    if (!built) return fail(c, TT_ERR_CUDA, berr);
    if (sb.nodes4) c->scene_mem.allocs.push_back(sb.nodes4);
    if (vb.nodes4) c->scene_mem.allocs.push_back(vb.nodes4);
    c->bvh_nodes = sb.num_nodes;
    c->bvh_depth = sb.max_depth;
    c->bvh_node_bytes = 64;
    if (sb.max_depth + 2 >= (uint32_t)BVH_STACK || vb.max_depth + 2 >= (uint32_t)BVH_STACK)
      return fail(c, TT_ERR_CAPACITY, "BVH deeper than the traversal stack");
    s.nodes = sb.nodes;
    s.tris = sb.tris;
    s.vnodes = vb.nodes;
    s.vtris = vb.tris;
    if (sb.nodes4 && !binary_only) {
      // Closest hit runs on the 4-wide nodes; a counted node visit reads 112 bytes (the
      // eighth float4 of a node is padding).
      s.nodes4 = sb.nodes4;
      c->bvh_nodes = sb.num_nodes4;
      c->bvh_node_bytes = 112;
    }
  } else {
    BvhInput bi{}, vbi{};
    host_inputs(&bi, &vbi);
    BvhOutput bo, vbo;
    if (!build_bvh(bi, 4, &bo)) return fail(c, TT_ERR_INVALID, "BVH build failed");
    if (!build_bvh(vbi, 4, &vbo)) return fail(c, TT_ERR_INVALID, "medium-boundary BVH build failed");
    c->bvh_nodes = bo.num_nodes;
    c->bvh_depth = bo.max_depth;
    c->bvh_node_bytes = 64;
    if (bo.max_depth + 2 >= (uint32_t)BVH_STACK || vbo.max_depth + 2 >= (uint32_t)BVH_STACK)
      return fail(c, TT_ERR_CAPACITY, "BVH deeper than the traversal stack");
    s.nodes = (const float4*)upload(bo.nodes.data(), bo.nodes.size() * sizeof(float));
    s.tris = (const float4*)upload(bo.tris.data(), bo.tris.size() * sizeof(float));
    s.vnodes = (const float4*)upload(vbo.nodes.data(), vbo.nodes.size() * sizeof(float));
    s.vtris = (const float4*)upload(vbo.tris.data(), vbo.tris.size() * sizeof(float));
  }
  s.num_vol_tris = (int)(vid.size() + vsid.size());
  s.num_spheres = (int)nsph;
  // Per global primitive: vertex indices and material (spheres: material only); the device
  // build made it on the device already.
  if (!s.tri_idx) {
    std::vector<uint32_t> ti(4 * ((size_t)ntri + nsph), 0u);
    parallel_ranges(ntri, [&](long long lo, long long hi) {
      for (long long t = lo; t < hi; ++t) {
        ti[4 * t] = c->idx[3 * t];
        ti[4 * t + 1] = c->idx[3 * t + 1];
        ti[4 * t + 2] = c->idx[3 * t + 2];
        ti[4 * t + 3] = c->mats[t];
      }
    });
    for (uint32_t i = 0; i < nsph; ++i) ti[4 * ((size_t)ntri + i) + 3] = c->sphere_mats[i];
    s.tri_idx = (const uint4*)upload(ti.data(), ti.size() * sizeof(uint32_t));
  }
  mark("bvh");
  s.normals = c->normals.empty() ? nullptr : (const float*)upload(c->normals.data(), c->normals.size() * sizeof(float));
  s.num_tris = (int)(nsurf + ssid.size());
  // Materials.
  std::vector<DevMaterial> dm(c->materials.size());
  for (size_t i = 0; i < dm.size(); ++i) {
    const tt_material& m = c->materials[i];
    dm[i].shader = m.shader;
    dm[i].emissive = m.emissive ? 1 : 0;
    dm[i].alpha = m.alpha;
    dm[i].ior_ratio = m.ior_ratio;
    dm[i].med_in = m.medium_inside - 1;
    dm[i].med_out = m.medium_outside - 1;
    std::memcpy(dm[i].reflectance, m.reflectance, sizeof(m.reflectance));
    std::memcpy(dm[i].emission, m.emission, sizeof(m.emission));
    dm[i].tex = nullptr;
    dm[i].tex_w = dm[i].tex_h = 0;
    dm[i].spec = m.specular_reflectivity;
  }
  // Textures (one device array each) and the per-vertex texture coordinates.
  {
    std::vector<const float*> dtex(c->textures.size(), nullptr);
    for (size_t k = 0; k < c->textures.size(); ++k)
      dtex[k] = (const float*)upload(c->textures[k].data(), c->textures[k].size() * sizeof(float));
    for (size_t i = 0; i < dm.size(); ++i) {
      const int t = c->materials[i].diffuse_texture - 1;
      if (t < 0) continue;
      dm[i].tex = dtex[t];
      dm[i].tex_w = c->texture_sizes[t].x;
      dm[i].tex_h = c->texture_sizes[t].y;
    }
    s.uvs = c->uvs.empty() ? nullptr : (const float2*)upload(c->uvs.data(), c->uvs.size() * sizeof(float));
  }
  s.materials = (const DevMaterial*)upload(dm.data(), dm.size() * sizeof(DevMaterial));
  // Media.
  std::vector<DevMedium> dmed(c->media.size());
  for (size_t i = 0; i < dmed.size(); ++i) {
    const tt_medium& m = c->media[i];
    DevMedium& o = dmed[i];
    o.kind = m.kind;
    o.priority = m.priority;
    o.phase = m.phase;
    o.g = m.phase_g;
    o.scattering = 0;
    for (int b = 0; b < NBINS; ++b) {
      o.sigma_s[b] = m.sigma_s[b];
      o.sigma_ext[b] = m.sigma_s[b] + m.sigma_a[b];
      o.scattering |= m.sigma_s[b] > 0.f;
    }
    if (m.kind == TT_MEDIUM_ATMOSPHERE) {
      // Rows of (sigma_t, molecules, aerosols) per bin as float4, and the majorant per row
      // made non-increasing upwards (TabulatedConstituents, atmosphere.cxx:260-272).
      const int rows = m.table_size;
      const std::vector<float>& t = c->media_tables[i];
      const size_t n = (size_t)rows * NBINS;
      std::vector<float> inter(4 * n, 0.f), maj(rows, 0.f);
      for (size_t k = 0; k < n; ++k) {
        inter[4 * k] = t[k];
        inter[4 * k + 1] = t[n + k];
        inter[4 * k + 2] = t[2 * n + k];
      }
      for (int r = 0; r < rows; ++r)
        for (int b = 0; b < NBINS; ++b) maj[r] = std::max(maj[r], t[(size_t)r * NBINS + b]);
      for (int r = rows - 2; r >= 0; --r) maj[r] = std::max(maj[r], maj[r + 1]);
      o.scattering = 1;
      o.rows = rows;
      o.h0 = m.table_h0;
      o.inv_dh = 1.f / m.table_dh;
      for (int k = 0; k < 3; ++k) o.center[k] = m.planet_center[k];
      o.radius = m.planet_radius;
      o.table = (const float4*)upload(inter.data(), inter.size() * sizeof(float));
      o.maj = (const float*)upload(maj.data(), maj.size() * sizeof(float));
    }
  }
  s.media = (const DevMedium*)upload(dmed.data(), dmed.size() * sizeof(DevMedium));
  s.num_media = (int)dmed.size();
  s.cam_track = make_uint2(0xffffffffu, (unsigned)-1);
  // Area lights: every triangle of an emissive material, in triangle order
  // (Scene::UpdateEmissiveIndexOffset numbers emissive primitives consecutively).
  std::vector<int> al;
  std::vector<float> av;
  bool any_emitter = false;
  for (const auto& m : c->materials) any_emitter |= m.emissive && !m.volume_boundary;
  for (uint32_t t = 0; any_emitter && t < ntri; ++t) {
    const tt_material& mt = c->materials[c->mats[t]];
    if (!mt.emissive || mt.volume_boundary) continue;
    al.push_back((int)t);
    for (int j = 0; j < 3; ++j) {
      const float* v = &c->verts[3 * (size_t)c->idx[3 * t + j]];
      av.push_back(v[0]);
      av.push_back(v[1]);
      av.push_back(v[2]);
      av.push_back(0.f);
    }
  }
  for (uint32_t i = 0; i < nsph; ++i) {
    const tt_material& mt = c->materials[c->sphere_mats[i]];
    if (!mt.emissive || mt.volume_boundary) continue;
    const float* q = &c->spheres[4 * (size_t)i];
    al.push_back((int)(ntri + i));
    const float rec[12] = {q[0], q[1], q[2], 1.f, q[3], 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    av.insert(av.end(), rec, rec + 12);
  }
  mark("tables");
  s.area_lights = (const int*)upload(al.data(), al.size() * sizeof(int));
  s.area_verts = (const float4*)upload(av.data(), av.size() * sizeof(float));
  s.num_area_lights = (int)al.size();
  std::vector<float> pl;
  for (auto& p : c->points) {
    pl.insert(pl.end(), p.spectrum, p.spectrum + NBINS);
    pl.insert(pl.end(), p.pos, p.pos + 3);
  }
  s.point_lights = (const float*)upload(pl.data(), pl.size() * sizeof(float));
  s.num_point_lights = (int)c->points.size();
  // Environmental lights.
  s.num_env = (int)c->envs.size();
  for (size_t i = 0; i < c->envs.size(); ++i) {
    const tt_env_light& e = c->envs[i].desc;
    DevEnvLight& L = s.env[i];
    std::memset(&L, 0, sizeof(L));
    L.kind = e.kind;
    double dir[3] = {e.dir[0], e.dir[1], e.dir[2]};
    if (e.kind == TT_ENV_SUN) {
      // Sun::Sun (light.hxx:253-263).
      const double cos_open = std::cos(M_PI / 180. * e.scalar2);
      const double pdf_val = 1. / (2. * M_PI * (1. - cos_open));
      L.cos_opening = (float)cos_open;
      L.pdf_val = (float)pdf_val;
      normalize_d(dir);
      frame_z_d(dir, L.X, L.Y, L.Z);
      for (int b = 0; b < NBINS; ++b) L.spectrum[b] = (float)(kSunSpectrum[b] * e.scalar * pdf_val);
    } else if (e.kind == TT_ENV_DOME) {
      normalize_d(dir);
      double down[3] = {-dir[0], -dir[1], -dir[2]};
      frame_z_d(down, L.X, L.Y, L.Z);
      std::memcpy(L.spectrum, e.spectrum, sizeof(e.spectrum));
    } else if (e.kind == TT_ENV_DIRECTIONAL) {
      normalize_d(dir);
      for (int k = 0; k < 3; ++k) L.dir[k] = (float)dir[k];
      std::memcpy(L.spectrum, e.spectrum, sizeof(e.spectrum));
    } else {
      // EnvMapLight (light.cxx:88-115): float frame from the (unnormalized) up vector,
      // row CMFs weighted by sin(theta) * mean(rgb).
      const float up[3] = {e.dir[0], e.dir[1], e.dir[2]};
      const float sign = std::copysign(1.0f, up[2]);
      const float a = -1.0f / (sign + up[2]);
      const float b = up[0] * up[1] * a;
      const float X[3] = {1.0f + sign * up[0] * up[0] * a, sign * b, -sign * up[0]};
      const float Y[3] = {b, sign + up[1] * up[1] * a, -up[1]};
      for (int k = 0; k < 3; ++k) { L.X[k] = X[k]; L.Y[k] = Y[k]; L.Z[k] = up[k]; }
      const int w = e.tex_width, h = e.tex_height;
      const auto& tex = c->envs[i].tex;
      HostArray<float>& rows = c->envs[i].cmf_rows;
      HostArray<float>& cols = c->envs[i].cmf_cols;
      HostArray<int>& grows = c->envs[i].guide_rows;
      HostArray<int>& gcols = c->envs[i].guide_cols;
      rows.resize(h);
      cols.resize((size_t)w * h);
      grows.resize(kEnvGuide + 1);
      gcols.resize((size_t)h * (kEnvGuide + 1));
      std::atomic<bool> zero_row{false};
      parallel_ranges(h, [&](long long y0, long long y1) {
        for (long long y = y0; y < y1; ++y) {
          const float v = ((float)(h - 1 - y) + 0.5f) / h;
          const double sin_theta = std::sin(v * (float)M_PI);
          double row_weight = 0.;
          for (int x = 0; x < w; ++x) {
            const float* px = &tex[3 * ((size_t)y * w + x)];
            const double mean = ((double)px[0] + px[1] + px[2]) / 3.;
            row_weight += sin_theta * mean;
            cols[(size_t)y * w + x] = (float)row_weight;
          }
          if (!(row_weight > 0.)) zero_row = true;
          for (int x = 0; x < w; ++x) cols[(size_t)y * w + x] /= (float)row_weight;
          cmf_guide(&cols[(size_t)y * w], w, &gcols[(size_t)y * (kEnvGuide + 1)]);
          rows[y] = (float)row_weight;
        }
      }, /*serial_below=*/64);  // rows of a few thousand texels each
      if (zero_row) return fail(c, TT_ERR_INVALID, "env map row with zero weight");
      for (int y = 1; y < h; ++y) rows[y] += rows[y - 1];
      const float inv = 1.f / rows[h - 1];
      for (int y = 0; y < h; ++y) rows[y] *= inv;
      cmf_guide(rows.data(), h, grows.data());
      L.w = w;
      L.h = h;
      L.tex = (const float*)upload(tex.data(), tex.size() * sizeof(float));
      L.cmf_rows = (const float*)upload(rows.data(), rows.size() * sizeof(float));
      L.cmf_cols = (const float*)upload(cols.data(), cols.size() * sizeof(float));
      L.guide_rows = (const int*)upload(grows.data(), grows.size() * sizeof(int));
      L.guide_cols = (const int*)upload(gcols.data(), gcols.size() * sizeof(int));
    }
  }
  mark("env maps");
  // Camera (camera.hxx:38-108, 159-175), computed in double.
  s.cam = make_dev_camera(c->camera);
  // Light picker (TrivialLightPicker, lightpicker_trivial.cxx:11-31) and scene bounds.
  const double nl = (double)c->points.size(), ne = c->envs.empty() ? 0. : 1., na = (double)al.size();
  const double tot = nl + ne + na;
  const double norm = tot > 0 ? 1. / tot : 0.;
  s.type_probs[0] = (float)(ne * norm);
  s.type_probs[1] = (float)(na * norm);
  s.type_probs[2] = (float)(nl * norm);
  s.type_probs[3] = 0.f;
  s.in_class_area = na > 0 ? (float)(1. / na) : 0.f;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  std::mutex box_mutex;
  parallel_ranges((long long)(c->verts.size() / 3), [&](long long v0, long long v1) {
    float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (long long v = v0; v < v1; ++v)
      for (int k = 0; k < 3; ++k) {
        l[k] = std::min(l[k], c->verts[3 * v + k]);
        h[k] = std::max(h[k], c->verts[3 * v + k]);
      }
    std::lock_guard<std::mutex> g(box_mutex);
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], (double)l[k]);
      hi[k] = std::max(hi[k], (double)h[k]);
    }
  });
  for (uint32_t i = 0; i < nsph; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], (double)c->spheres[4 * (size_t)i + k] - c->spheres[4 * (size_t)i + 3]);
      hi[k] = std::max(hi[k], (double)c->spheres[4 * (size_t)i + k] + c->spheres[4 * (size_t)i + 3]);
    }
  if (c->verts.empty() && nsph == 0) for (int k = 0; k < 3; ++k) { lo[k] = hi[k] = 0; }
  const double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                (hi[2] - lo[2]) * (hi[2] - lo[2]));
  for (int k = 0; k < 3; ++k) {
    c->bb_lo[k] = (float)lo[k];
    c->bb_hi[k] = (float)hi[k];
    s.box_lo[k] = (float)lo[k];
    s.box_inv[k] = hi[k] > lo[k] ? (float)(1.0 / (hi[k] - lo[k])) : 1.f;
  }
  mark("bounds");
  s.long_distance = (float)(10. * diag);
  s.max_path_nodes = c->params.max_ray_depth + 1;
  s.algo = c->params.algo;
  // Material-sorted shading pays where the hits of a bounce mix many shader kinds: by
  // default (sort_shading = 0) it is on in scenes without media whose surfaces use three or
  // more shader kinds.  (Measured per sample: 7 % faster on the terrain with Lambert, metal
  // and glass; 5 % slower on a Lambert-only box, 1.5x slower on the gap-lit room with
  // Lambert walls and a glossy floor and 1.27x slower in the medium-filled box, where the
  // sorted order's scattered path-state reads outweigh the divergence it removes.)
  bool sort = c->params.sort_shading > 0;
  if (c->params.sort_shading == 0 && c->media.empty()) {
    unsigned kinds = 0u;
    std::mutex kinds_mutex;
    parallel_ranges((long long)c->mats.size(), [&](long long t0, long long t1) {
      unsigned k = 0u;
      for (long long t = t0; t < t1; ++t) k |= 1u << (c->materials[c->mats[t]].shader & 31);
      std::lock_guard<std::mutex> g(kinds_mutex);
      kinds |= k;
    });
    for (uint32_t m : c->sphere_mats) kinds |= 1u << (c->materials[m].shader & 31);
    sort = __builtin_popcount(kinds) >= 3;
  }
  s.sort_shading = (sort && c->params.algo == TT_ALGO_PT) ? 1 : 0;
  mark("sort keys");
  // Quasi-random sampling: pt2 only, as in the reference (CameraRenderWorker's sampler).
  s.sobol = nullptr;
  s.rotations = nullptr;
  std::vector<uint32_t> sobol;
  if (c->params.qmc && c->params.algo == TT_ALGO_PT2) {
    build_sobol_matrices(&sobol);
    s.sobol = (const uint32_t*)upload(sobol.data(), sobol.size() * sizeof(uint32_t));
    s.rotations = (const float*)upload(tt_rotation_offsets, sizeof(tt_rotation_offsets));
  }
  s.sample_lights = c->params.pt_sample_mode != TT_SAMPLE_BSDF;
  s.sample_bsdf = c->params.pt_sample_mode != TT_SAMPLE_LIGHTS;
  if (tot == 0. && s.sample_lights) s.sample_lights = 0;  // no light to sample
  for (void* p : c->scene_mem.allocs)
    if (!p) return fail(c, TT_ERR_CUDA, "device allocation failed");
  c->d_err = (unsigned int*)c->scene_mem.alloc(sizeof(unsigned int));
  if (!c->d_err) return fail(c, TT_ERR_CUDA, "device allocation failed");
  TT_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(unsigned int), c->stream));
  if (s.num_media > 0) {
    // Medium tracker at the camera (every camera path starts there).
    uint2* d_track = (uint2*)c->scene_mem.alloc(sizeof(uint2));
    if (!d_track) return fail(c, TT_ERR_CUDA, "device allocation failed");
    launch_init_tracker(s, make_float3(c->camera.pos[0], c->camera.pos[1], c->camera.pos[2]),
                        make_float3((float)lo[0], (float)lo[1], (float)lo[2]),
                        make_float3((float)hi[0], (float)hi[1], (float)hi[2]), d_track, c->d_err, c->stream);
    TT_CUDA(c, cudaGetLastError());
    uint2 h_track;
    TT_CUDA(c, cudaMemcpyAsync(&h_track, d_track, sizeof(uint2), cudaMemcpyDeviceToHost, c->stream));
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
    s.cam_track = h_track;
  }
  mark("lights+env");
  // Framebuffers and counters.
  const size_t n3 = 3 * (size_t)c->npix;
  c->fb.accum = (float*)c->scene_mem.alloc(n3 * sizeof(float));
  c->fb.light = (float*)c->scene_mem.alloc(n3 * sizeof(float));
  c->d_acc = (double*)c->scene_mem.alloc(n3 * sizeof(double));
  c->d_light = (double*)c->scene_mem.alloc(n3 * sizeof(double));
  c->d_stats = (unsigned long long*)c->scene_mem.alloc(8 * sizeof(unsigned long long));
  if (!c->fb.accum || !c->fb.light || !c->d_acc || !c->d_light || !c->d_stats)
    return fail(c, TT_ERR_CUDA, "device allocation failed");
  TT_CUDA(c, cudaMemsetAsync(c->fb.accum, 0, n3 * sizeof(float), c->stream));
  TT_CUDA(c, cudaMemsetAsync(c->fb.light, 0, n3 * sizeof(float), c->stream));
  TT_CUDA(c, cudaMemsetAsync(c->d_acc, 0, n3 * sizeof(double), c->stream));
  TT_CUDA(c, cudaMemsetAsync(c->d_light, 0, n3 * sizeof(double), c->stream));
  TT_CUDA(c, cudaMemsetAsync(c->d_stats, 0, 8 * sizeof(unsigned long long), c->stream));
  int sms = 0;
  TT_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  c->grid = sms * kernel_blocks_per_sm();
  c->rounds = c->params.max_ray_depth;
  TT_CUDA(c, cudaDeviceSynchronize());
  mark("framebuffer");
  c->uploaded = true;
  return TT_OK;
}

}  // extern "C"

static tt_status ensure_path_state(tt_ctx* c, int cap) {
  const bool guided = c->dev.guide != 0;
  if (c->ps.cap >= cap && c->ps_guided == guided) return TT_OK;
  cudaStreamSynchronize(c->stream);
  c->path_mem.free_all();
  PathState& p = c->ps;
  p = PathState{};
  DeviceBuffers& m = c->path_mem;
  const size_t n = (size_t)cap;
  p.ray_o = (float4*)m.alloc(n * sizeof(float4));
  p.ray_d = (float4*)m.alloc(n * sizeof(float4));
  p.hit = (float4*)m.alloc(n * sizeof(float4));
  p.beta = (float4*)m.alloc(n * sizeof(float4));
  p.accum = (float4*)m.alloc(n * sizeof(float4));
  p.rng_state = (unsigned long long*)m.alloc(n * 8);
  p.rng_inc = (unsigned long long*)m.alloc(n * 8);
  p.meta = (uint4*)m.alloc(n * sizeof(uint4));
  p.sh_o = (float4*)m.alloc(n * sizeof(float4));
  p.sh_d = (float4*)m.alloc(n * sizeof(float4));
  p.sh_c = (float4*)m.alloc(n * sizeof(float4));
  p.ext_q[0] = (int*)m.alloc(n * sizeof(int));
  p.ext_q[1] = (int*)m.alloc(n * sizeof(int));
  p.sh_q = (int*)m.alloc(n * sizeof(int));
  p.done_q = (int*)m.alloc(n * sizeof(int));
  p.counters = (int*)m.alloc(kCountersPerBounce * (size_t)(c->rounds + 3) * sizeof(int));
  if (c->dev.sort_shading && c->dev.algo == TT_ALGO_PT) {
    p.sort_q = (int*)m.alloc(n * sizeof(int));
    p.sort_key = (unsigned char*)m.alloc(n);
  }
  if (c->dev.num_media > 0) {
    p.track = (uint2*)m.alloc(n * sizeof(uint2));
    p.vol = (float4*)m.alloc(n * sizeof(float4));
    p.sh_track = (uint2*)m.alloc(n * sizeof(uint2));
    p.sh_med = (float4*)m.alloc(n * sizeof(float4));
  }
  if (c->dev.algo == TT_ALGO_PT2) {
    p.rough = (float*)m.alloc(n * sizeof(float));
    if (c->dev.num_media > 0) {
      p.wt2 = (float*)m.alloc(n * 9 * sizeof(float));
      p.sh_wt = (float*)m.alloc(n * 9 * sizeof(float));
    }
    if (c->dev.sobol) {
      p.qmc = (uint4*)m.alloc(n * sizeof(uint4));
      if (c->dev.num_media > 0) p.sh_qmc = (uint4*)m.alloc(n * sizeof(uint4));
    }
  }
  if (guided) {
    p.ginp = (float4*)m.alloc(n * 3 * sizeof(float4));
    p.guide_q = (int*)m.alloc(n * sizeof(int));
    p.grec = (float4*)m.alloc(n * 6 * sizeof(float4));
    p.gnee = (float4*)m.alloc(n * sizeof(float4));
    p.rr = (float*)m.alloc(n * sizeof(float));
    p.records = c->d_records;
    p.rec_count = c->d_rec_count;
    p.rec_cap = c->rec_cap;
  }
  p.err = c->d_err;
  for (void* a : m.allocs)
    if (!a) {
      m.free_all();
      p = PathState{};
      return fail(c, TT_ERR_CUDA, "path state allocation failed (capacity " + std::to_string(cap) + ")");
    }
  p.cap = cap;
  c->ps_guided = guided;
  return TT_OK;
}

// ensure_path_state for a wave of *cap paths, halving the wave while the allocation fails
// (down to 2^20 paths); *cap is the capacity obtained.
static tt_status ensure_path_state_fit(tt_ctx* c, int* cap) {
  for (;;) {
    const tt_status st = ensure_path_state(c, *cap);
    if (st == TT_OK || *cap <= (1 << 20)) return st;
    cudaGetLastError();
    *cap = std::max(1 << 20, *cap / 2);
  }
}

// The tree guider's device arrays into the scene the kernels see.
static void tree_to_dev(tt_ctx* c) {
  c->dev.tree_nodes = c->tree->d_nodes;
  c->dev.tree_root = c->tree->root_ref();
  c->dev.tree_mix = c->tree->d_mix;
  c->dev.tree_quad = c->tree->distribution == TT_TREE_QUADTREE ? 1 : 0;
  c->dev.tree_qchild = c->tree->d_qchild;
  c->dev.tree_qprob = c->tree->d_qprob;
  c->dev.tree_qroot = c->tree->d_qroot;
}

// After a pass: `steps_per_pass` Adam steps, each on a mini-batch drawn from the record
// pool; also updates the pool's yield per path, from which the next pass's keep
// probability follows.
static tt_status guide_train(tt_ctx* c, long long paths) {
  int cnt = 0;
  TT_CUDA(c, cudaMemcpyAsync(&cnt, c->d_rec_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  const long long count = (long long)(unsigned)cnt;
  const long long fresh = count - c->rec_seen;
  if (paths > 0 && fresh >= 0) c->rec_rate = (double)fresh / ((double)paths * std::max(1e-6, (double)c->dev.guide_keep));
  if (count > (1ll << 30)) {
    // Keep the ring position and a full pool while the counter stays far from overflow.
    const int wrapped = (int)(c->rec_cap + count % c->rec_cap);
    TT_CUDA(c, cudaMemcpyAsync(c->d_rec_count, &wrapped, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
    c->rec_seen = wrapped;
  } else {
    c->rec_seen = count;
  }
  const int pool = (int)std::min<long long>(count, c->rec_cap);
  if (c->dev.guide_method == TT_GUIDE_TREE) {
    // One round of the tree guider on this pass's records: the newest min(fresh, pool) of
    // the ring, ending at index count % rec_cap.
    const int n = (int)std::min<long long>(std::max(0ll, fresh), pool);
    if (n <= 0) return TT_OK;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<GuideRecord> recs(n);
    const long long end = count % c->rec_cap;
    const long long start = ((end - n) % c->rec_cap + c->rec_cap) % c->rec_cap;
    const long long first = std::min<long long>(n, c->rec_cap - start);
    TT_CUDA(c, cudaMemcpy(recs.data(), c->d_records + start, (size_t)first * sizeof(GuideRecord),
                          cudaMemcpyDeviceToHost));
    if (first < n)
      TT_CUDA(c, cudaMemcpy(recs.data() + first, c->d_records, (size_t)(n - first) * sizeof(GuideRecord),
                            cudaMemcpyDeviceToHost));
    std::string gerr;
    if (!c->tree->fit_round(recs.data(), n, c->gparams.seed, c->stream, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
    tree_to_dev(c);
    c->stats.guide_records += (uint64_t)n;
    c->stats.guide_steps += 1;
    c->stats.guide_train_ms +=
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return TT_OK;
  }
  if (pool >= 256) {
    const int n = std::min(pool, c->gparams.batch > 0 ? c->gparams.batch : 8192);
    std::string gerr;
    if (!c->gnet->ensure_capacity(n, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, c->stream);
    const int steps = c->gparams.steps_per_pass > 0 ? c->gparams.steps_per_pass : 16;
    const float lr = c->gparams.learning_rate > 0.f ? c->gparams.learning_rate : 1e-3f;
    for (int k = 0; k < steps; ++k) {
      c->gnet->gradient(c->d_records, n, c->stream, true, lr, pool,
                        c->gparams.seed * 0x9e3779b97f4a7c15ull + (++c->draw_seed));
    }
    cudaEventRecord(b, c->stream);
    float loss = 0.f, ms = 0.f;
    cudaMemcpyAsync(&loss, c->gnet->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
    TT_CUDA(c, cudaGetLastError());
    if (c->gnet->tensor_error(c->stream)) {
      c->stats.error_flags |= ERR_TENSOR;
      return fail(c, TT_ERR_LOOP_CAP, "a tensor-core wait of the training step timed out");
    }
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    c->stats.guide_records += (uint64_t)std::max(0ll, fresh);
    c->stats.guide_steps += (uint64_t)steps;
    c->stats.guide_loss = loss;
    c->stats.guide_train_ms += ms;
  }
  return TT_OK;
}

static tt_status render_range(tt_ctx* c, int32_t spp, uint64_t seed, int32_t pb, int32_t pe) {
  if (!c) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  if (spp <= 0) return fail(c, TT_ERR_INVALID, "spp must be positive");
  if (pb < 0 || pe > c->npix || pb >= pe) return fail(c, TT_ERR_INVALID, "bad pixel range");
  TT_CUDA(c, cudaSetDevice(c->device));
  const int npix_range = pe - pb;
  const long long total = (long long)spp * npix_range;
  const int wave_limit = c->params.wave_paths > 0 ? c->params.wave_paths : kDefaultWave;
  int cap = (int)std::min<long long>(total, wave_limit);
  if (c->dev.guide_record) {
    // Keep about 80 % of a pool's worth of this pass's records at most.
    const double expected = c->rec_rate * (double)total;
    c->dev.guide_keep = expected > 0.0 ? (float)std::min(1.0, 0.8 * c->rec_cap / expected) : 1.f;
  }
  c->dev.guide_cold = (c->dev.guide && c->dev.guide_method == TT_GUIDE_LEARNED && c->gnet && c->gnet->fresh) ? 1 : 0;
  tt_status st = ensure_path_state_fit(c, &cap);
  if (st != TT_OK) return st;
  const bool counting = c->profiling >= 2;
  const bool timing = c->profiling >= 1;
  std::vector<cudaEvent_t> ev;   // begin/end pairs of timed launches
  std::vector<int> ev_kind;      // 0 closest hit, 1 shadow
  auto timed = [&](int kind, auto&& launch) {
    if (!timing) { launch(); return; }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, c->stream);
    launch();
    cudaEventRecord(b, c->stream);
    ev.push_back(a);
    ev.push_back(b);
    ev_kind.push_back(kind);
  };
  cudaEvent_t pass_begin, pass_end, wave_ev[2];
  TT_CUDA(c, cudaEventCreate(&pass_begin));
  TT_CUDA(c, cudaEventCreate(&pass_end));
  TT_CUDA(c, cudaEventCreateWithFlags(&wave_ev[0], cudaEventDisableTiming));
  TT_CUDA(c, cudaEventCreateWithFlags(&wave_ev[1], cudaEventDisableTiming));
  TT_CUDA(c, cudaEventRecord(pass_begin, c->stream));
  const int grid = c->grid;
  const int rounds = c->rounds;
  uint64_t launches = 0;
  bool stopped = false;
  int wave_index = 0;
  for (long long ws = 0; ws < total; ws += cap, ++wave_index) {
    if (c->stop.load()) { stopped = true; break; }
    if (wave_index >= 2) cudaEventSynchronize(wave_ev[wave_index & 1]);
    WaveArgs w;
    w.wave_start = ws;
    w.wave_paths = (int)std::min<long long>(cap, total - ws);
    w.pixel_begin = pb;
    w.npix_range = npix_range;
    w.npix_total = c->npix;
    w.sample_offset = c->next_sample;
    w.seed = seed;
    cudaMemsetAsync(c->ps.counters, 0, kCountersPerBounce * (size_t)(rounds + 3) * sizeof(int), c->stream);
    launch_generate(c->dev, c->ps, c->fb, w, grid, c->stream);
    launches++;
    for (int b = 0; b < rounds; ++b) {
      timed(1, [&] { launch_shadow(c->dev, c->ps, c->fb, b, counting, c->d_stats + 2, grid, c->stream); });
      if (c->dev.guide_record) launch_flush(c->dev, c->ps, c->fb, b, grid, c->stream);
      timed(0, [&] { launch_extend(c->dev, c->ps, b, counting, c->d_stats, grid, c->stream); });
      if (c->dev.num_media > 0) {
        launch_track(c->dev, c->ps, b, grid, c->stream);
        launches++;
      }
      launch_shade(c->dev, c->ps, b, grid, c->stream);
      if (c->dev.guide && b < c->dev.guide_depth) {
        launch_guide(c->dev, c->ps, b, c->stream);
        launches++;
      }
      launches += (c->dev.guide_record ? 3 : 2) + shade_launches(c->dev, c->ps, b);
    }
    timed(1, [&] { launch_shadow(c->dev, c->ps, c->fb, rounds, counting, c->d_stats + 2, grid, c->stream); });
    // Finished paths into the pass framebuffer: with guiding records, k_flush after every
    // bounce (it also commits the records); without, one gather at the end of the wave.
    if (c->dev.guide_record) launch_flush(c->dev, c->ps, c->fb, rounds, grid, c->stream);
    else launch_gather(c->dev, c->ps, c->fb, w, grid, c->stream);
    k_tally<<<1, 32, 0, c->stream>>>(c->ps.counters, rounds, c->d_stats);
    launches += 3;
    cudaEventRecord(wave_ev[wave_index & 1], c->stream);
  }
  launch_accumulate(c->fb, c->d_acc, c->d_light, 3 * c->npix, c->stream);
  launches++;
  TT_CUDA(c, cudaEventRecord(pass_end, c->stream));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  TT_CUDA(c, cudaGetLastError());
  float pass_ms = 0.f;
  cudaEventElapsedTime(&pass_ms, pass_begin, pass_end);
  c->stats.pass_ms += pass_ms;
  for (size_t k = 0; k < ev_kind.size(); ++k) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
    if (ev_kind[k] == 0) { c->stats.extend_ms += ms; c->stats.extend_launches++; }
    else { c->stats.shadow_ms += ms; c->stats.shadow_launches++; }
    cudaEventDestroy(ev[2 * k]);
    cudaEventDestroy(ev[2 * k + 1]);
  }
  if (!timing) {
    c->stats.extend_launches += (uint64_t)rounds * wave_index;
    c->stats.shadow_launches += (uint64_t)(rounds + 1) * wave_index;
  }
  cudaEventDestroy(pass_begin);
  cudaEventDestroy(pass_end);
  cudaEventDestroy(wave_ev[0]);
  cudaEventDestroy(wave_ev[1]);
  c->stats.kernel_launches += launches;
  c->stats.paths += (uint64_t)std::min<long long>(total, (long long)wave_index * cap);
  // Bookkeeping as in SimplePixelByPixelRenderingAlgo: the sample count of the pass is
  // added whether or not the pass completed.
  for (int px = pb; px < pe; ++px) c->spp_count[px] += (uint64_t)spp;
  c->splat_count += (uint64_t)spp * (uint64_t)npix_range;
  c->next_sample += (uint64_t)spp;
  if (c->dev.guide_record && !stopped && c->gparams.train == 1) {
    const tt_status gs = guide_train(c, total);
    if (gs != TT_OK) return gs;
  }
  unsigned int errw = 0;
  TT_CUDA(c, cudaMemcpy(&errw, c->d_err, sizeof(errw), cudaMemcpyDeviceToHost));
  if (errw) {
    c->stats.error_flags |= errw;
    return fail(c, TT_ERR_LOOP_CAP, "a device loop hit its cap (error word " + std::to_string(errw) + ")");
  }
  if (stopped) return fail(c, TT_ERR_INTERRUPTED, "stopped by tt_request_stop");
  return TT_OK;
}

namespace tt {
// Read access to an uploaded context's scene record for tt_render_pass_noalloc.
bool context_scene(tt_ctx* c, DevScene* scene, int* device, int* npix, int* max_depth, std::string** err) {
  if (!c->uploaded) {
    c->err = "tt_upload_scene has not run";
    return false;
  }
  *scene = c->dev;
  *device = c->device;
  *npix = c->npix;
  *max_depth = c->rounds;
  *err = &c->err;
  return true;
}
}  // namespace tt

extern "C" {

tt_status tt_render_pass(tt_ctx* c, int32_t spp, uint64_t seed) {
  if (!c) return TT_ERR_INVALID;
  return render_range(c, spp, seed, 0, c->npix);
}

tt_status tt_render_pass_range(tt_ctx* c, int32_t spp, uint64_t seed, int32_t pb, int32_t pe) {
  return render_range(c, spp, seed, pb, pe);
}

tt_status tt_request_interrupt(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  c->interrupt.store(1);
  return TT_OK;
}

tt_status tt_request_stop(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  c->stop.store(1);
  return TT_OK;
}

int32_t tt_poll_interrupt(tt_ctx* c) { return c ? c->interrupt.exchange(0) : 0; }
int32_t tt_stop_requested(tt_ctx* c) { return c ? c->stop.load() : 0; }

tt_status tt_read_accumulators(tt_ctx* c, double* accum, double* light, uint64_t* spp, uint64_t* splat) {
  if (!c) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  const size_t n3 = 3 * (size_t)c->npix;
  if (accum) TT_CUDA(c, cudaMemcpy(accum, c->d_acc, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (light) TT_CUDA(c, cudaMemcpy(light, c->d_light, n3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (spp) std::memcpy(spp, c->spp_count.data(), c->npix * sizeof(uint64_t));
  if (splat) *splat = c->splat_count;
  return TT_OK;
}

// Spectral3ImageBuffer::ToImage before the clamp (renderbuffer.hxx:172-200), resolved on
// the device: average the pixel samples, add the camera splats weighted by
// npix / splat_count, and copy back npix x 3 floats.
tt_status tt_read_framebuffer(tt_ctx* c, float* rgb, uint64_t* counts) {
  if (!c || !rgb) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  const double sw = c->splat_count > 0 ? (double)c->npix / (double)c->splat_count : 0.;
  bool uniform = true;
  for (int p = 1; p < c->npix && uniform; ++p) uniform = c->spp_count[p] == c->spp_count[0];
  DeviceBuffers tmp;
  tmp.stream = c->stream;
  double* inv_px = nullptr;
  double inv_all = 0.;
  if (uniform) {
    inv_all = c->npix > 0 && c->spp_count[0] > 0 ? 1.0 / (double)c->spp_count[0] : 0.;
  } else {
    std::vector<double> inv(c->npix);
    for (int p = 0; p < c->npix; ++p) inv[p] = c->spp_count[p] > 0 ? 1.0 / (double)c->spp_count[p] : 0.;
    inv_px = (double*)tmp.alloc(inv.size() * sizeof(double));
    if (!inv_px) return fail(c, TT_ERR_CUDA, "device allocation failed");
    TT_CUDA(c, cudaMemcpyAsync(inv_px, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  float* d_rgb = (float*)tmp.alloc(3 * (size_t)c->npix * sizeof(float));
  if (!d_rgb) return fail(c, TT_ERR_CUDA, "device allocation failed");
  launch_resolve(c->d_acc, c->d_light, inv_px, inv_all, sw, c->npix, d_rgb, c->stream);
  TT_CUDA(c, cudaGetLastError());
  TT_CUDA(c, cudaMemcpyAsync(rgb, d_rgb, 3 * (size_t)c->npix * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  tmp.free_all();
  if (counts) std::memcpy(counts, c->spp_count.data(), c->npix * sizeof(uint64_t));
  return TT_OK;
}

tt_status tt_generate_image(tt_ctx* c, int32_t linear_output, uint8_t* out) {
  if (!c || !out) return TT_ERR_INVALID;
  std::vector<float> rgb(3 * (size_t)c->npix);
  tt_status st = tt_read_framebuffer(c, rgb.data(), nullptr);
  if (st != TT_OK) return st;
  const int xres = c->camera.xres, yres = c->camera.yres;
  for (int y = 0; y < yres; ++y)
    for (int x = 0; x < xres; ++x) {
      const size_t src = 3 * ((size_t)y * xres + x);
      const size_t dst = 3 * ((size_t)(yres - 1 - y) * xres + x);
      for (int k = 0; k < 3; ++k) {
        double v = std::min(1.0, std::max(0.0, (double)rgb[src + k]));
        if (!linear_output) v = v <= 0.0031308 ? 12.92 * v : 1.055 * std::pow(v, 1.0 / 2.4) - 0.055;
        out[dst + k] = (uint8_t)(v * 255.999);
      }
    }
  return TT_OK;
}

tt_status tt_clear_framebuffer(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  const size_t n3 = 3 * (size_t)c->npix;
  TT_CUDA(c, cudaMemsetAsync(c->d_acc, 0, n3 * sizeof(double), c->stream));
  TT_CUDA(c, cudaMemsetAsync(c->d_light, 0, n3 * sizeof(double), c->stream));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  std::fill(c->spp_count.begin(), c->spp_count.end(), 0);
  c->splat_count = 0;
  c->next_sample = 0;
  return TT_OK;
}

static tt_status batch_prep(tt_ctx* c, const void* rays, int32_t n) {
  if (!c || n < 0 || (n > 0 && !rays)) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  return TT_OK;
}

tt_status tt_intersect_batch(tt_ctx* c, const float* rays, int32_t n, int32_t* prim, float* t, float* u, float* v) {
  tt_status st = batch_prep(c, rays, n);
  if (st != TT_OK || n == 0) return st;
  float *dr = nullptr, *dt = nullptr, *du = nullptr, *dv = nullptr;
  int* dp = nullptr;
  TT_CUDA(c, cudaMalloc(&dr, 8 * (size_t)n * sizeof(float)));
  cudaMalloc(&dt, n * sizeof(float));
  cudaMalloc(&du, n * sizeof(float));
  cudaMalloc(&dv, n * sizeof(float));
  cudaMalloc(&dp, n * sizeof(int));
  cudaMemcpy(dr, rays, 8 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  launch_intersect_rays(c->dev, dr, n, dp, dt, du, dv, c->d_err, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(prim, dp, n * sizeof(int), cudaMemcpyDeviceToHost);
  cudaMemcpy(t, dt, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (u) cudaMemcpy(u, du, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (v) cudaMemcpy(v, dv, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dr); cudaFree(dt); cudaFree(du); cudaFree(dv); cudaFree(dp);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_occluded_batch(tt_ctx* c, const float* rays, int32_t n, uint8_t* occ) {
  tt_status st = batch_prep(c, rays, n);
  if (st != TT_OK || n == 0) return st;
  float* dr = nullptr;
  unsigned char* docc = nullptr;
  TT_CUDA(c, cudaMalloc(&dr, 8 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&docc, n));
  cudaMemcpy(dr, rays, 8 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  launch_occluded_rays(c->dev, dr, n, docc, c->d_err, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(occ, docc, n, cudaMemcpyDeviceToHost);
  cudaFree(dr);
  cudaFree(docc);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_intersect_batch_device(tt_ctx* c, const float* d_rays, int32_t n, int32_t* d_prim, float* d_t,
                                    float* d_u, float* d_v, void* stream) {
  tt_status st = batch_prep(c, d_rays, n);
  if (st != TT_OK || n == 0) return st;
  if (!d_prim || !d_t || !d_u || !d_v) return fail(c, TT_ERR_INVALID, "output pointer is NULL");
  launch_intersect_rays(c->dev, d_rays, n, d_prim, d_t, d_u, d_v, c->d_err, (cudaStream_t)stream);
  TT_CUDA(c, cudaGetLastError());
  return TT_OK;
}

tt_status tt_count_traversal(tt_ctx* c, const float* rays, int32_t n) {
  tt_status st = batch_prep(c, rays, n);
  if (st != TT_OK || n == 0) return st;
  float* dr = nullptr;
  TT_CUDA(c, cudaMalloc(&dr, 8 * (size_t)n * sizeof(float)));
  cudaMemcpy(dr, rays, 8 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  launch_count_rays(c->dev, dr, n, c->d_stats, c->d_err, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaFree(dr);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  c->stats.counted_rays += (uint64_t)n;
  return TT_OK;
}

static tt_status bsdf_prep(tt_ctx* c, int32_t material, const float* wi, const int32_t* li, int32_t n) {
  if (!c || !wi || !li || n < 0) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  if (material < 0 || material >= (int)c->materials.size()) return fail(c, TT_ERR_INVALID, "bad material index");
  for (int k = 0; k < 3; ++k)
    if (li[k] < 0 || li[k] >= NBINS) return fail(c, TT_ERR_INVALID, "bad wavelength bin");
  TT_CUDA(c, cudaSetDevice(c->device));
  return TT_OK;
}

tt_status tt_sample_bsdf_batch(tt_ctx* c, int32_t material, const float* wi, const int32_t* li, int32_t n,
                               uint64_t seed, float* out_dir, float* out_val, float* out_pdf) {
  tt_status st = bsdf_prep(c, material, wi, li, n);
  if (st != TT_OK || n == 0) return st;
  float *dd = nullptr, *dv = nullptr, *dp = nullptr;
  TT_CUDA(c, cudaMalloc(&dd, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dv, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dp, (size_t)n * sizeof(float)));
  launch_sample_bsdf(c->dev, material, make_float3(wi[0], wi[1], wi[2]), make_int3(li[0], li[1], li[2]), n, seed, dd,
                     dv, dp, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(out_dir, dd, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_val, dv, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_pdf, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dd); cudaFree(dv); cudaFree(dp);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_eval_bsdf_batch(tt_ctx* c, int32_t material, const float* wi, const int32_t* li, const float* dirs,
                             int32_t n, float* out_val, float* out_pdf) {
  tt_status st = bsdf_prep(c, material, wi, li, n);
  if (st != TT_OK || n == 0) return st;
  if (!dirs) return TT_ERR_INVALID;
  float *di = nullptr, *dv = nullptr, *dp = nullptr;
  TT_CUDA(c, cudaMalloc(&di, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dv, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dp, (size_t)n * sizeof(float)));
  cudaMemcpy(di, dirs, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  launch_eval_bsdf(c->dev, material, make_float3(wi[0], wi[1], wi[2]), make_int3(li[0], li[1], li[2]), di, n, dv, dp,
                   c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(out_val, dv, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_pdf, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(di); cudaFree(dv); cudaFree(dp);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

static tt_status phase_prep(tt_ctx* c, int32_t medium, const float* pos, const float* wi, const int32_t* li, int32_t n) {
  if (!c || !pos || !wi || !li || n < 0) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  if (medium < 0 || medium >= (int)c->media.size()) return fail(c, TT_ERR_INVALID, "bad medium index");
  for (int k = 0; k < 3; ++k)
    if (li[k] < 0 || li[k] >= NBINS) return fail(c, TT_ERR_INVALID, "bad wavelength bin");
  TT_CUDA(c, cudaSetDevice(c->device));
  return TT_OK;
}

tt_status tt_sample_phase_batch(tt_ctx* c, int32_t medium, const float* pos, const float* wi, const int32_t* li,
                                int32_t n, uint64_t seed, float* out_dir, float* out_val, float* out_pdf) {
  tt_status st = phase_prep(c, medium, pos, wi, li, n);
  if (st != TT_OK || n == 0) return st;
  if (!out_dir || !out_val || !out_pdf) return fail(c, TT_ERR_INVALID, "output buffer is NULL");
  float *dd = nullptr, *dv = nullptr, *dp = nullptr;
  TT_CUDA(c, cudaMalloc(&dd, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dv, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dp, (size_t)n * sizeof(float)));
  launch_sample_phase(c->dev, medium, make_float3(pos[0], pos[1], pos[2]), make_float3(wi[0], wi[1], wi[2]),
                      make_int3(li[0], li[1], li[2]), n, seed, dd, dv, dp, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(out_dir, dd, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_val, dv, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_pdf, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dd); cudaFree(dv); cudaFree(dp);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_eval_phase_batch(tt_ctx* c, int32_t medium, const float* pos, const float* wi, const int32_t* li,
                              const float* dirs, int32_t n, float* out_val, float* out_pdf) {
  tt_status st = phase_prep(c, medium, pos, wi, li, n);
  if (st != TT_OK || n == 0) return st;
  if (!dirs || !out_val || !out_pdf) return fail(c, TT_ERR_INVALID, "buffer is NULL");
  float *di = nullptr, *dv = nullptr, *dp = nullptr;
  TT_CUDA(c, cudaMalloc(&di, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dv, 3 * (size_t)n * sizeof(float)));
  TT_CUDA(c, cudaMalloc(&dp, (size_t)n * sizeof(float)));
  cudaMemcpy(di, dirs, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  launch_eval_phase(c->dev, medium, make_float3(pos[0], pos[1], pos[2]), make_float3(wi[0], wi[1], wi[2]),
                    make_int3(li[0], li[1], li[2]), di, n, dv, dp, c->stream);
  cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaGetLastError();
  cudaMemcpy(out_val, dv, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(out_pdf, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(di); cudaFree(dv); cudaFree(dp);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_read_accumulators_device(tt_ctx* c, double* d_accum, double* d_light, void* stream) {
  if (!c || !d_accum || !d_light) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  const size_t bytes = 3 * (size_t)c->npix * sizeof(double);
  // Order after the last pass on the context's stream, then copy on the caller's stream.
  cudaEvent_t ev;
  TT_CUDA(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaEventRecord(ev, c->stream);
  cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
  cudaEventDestroy(ev);
  TT_CUDA(c, cudaMemcpyAsync(d_accum, c->d_acc, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  TT_CUDA(c, cudaMemcpyAsync(d_light, c->d_light, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return TT_OK;
}

tt_status tt_last_wave_queue_lengths(tt_ctx* c, int32_t* out, int32_t n) {
  if (!c || !out || n < 0) return TT_ERR_INVALID;
  if (!c->uploaded || c->ps.cap == 0) return fail(c, TT_ERR_NOT_READY, "no pass has run");
  if (n > c->rounds + 1) return fail(c, TT_ERR_INVALID, "more bounces requested than a pass has");
  TT_CUDA(c, cudaSetDevice(c->device));
  std::vector<int> buf(kCountersPerBounce * (size_t)(c->rounds + 3));
  TT_CUDA(c, cudaMemcpy(buf.data(), c->ps.counters, buf.size() * sizeof(int), cudaMemcpyDeviceToHost));
  for (int b = 0; b < n; ++b)
    for (int k = 0; k < 3; ++k) out[3 * b + k] = buf[kCountersPerBounce * b + k];
  return TT_OK;
}

tt_status tt_set_profiling(tt_ctx* c, int32_t on) {
  if (!c) return TT_ERR_INVALID;
  c->profiling = on;
  return TT_OK;
}

tt_status tt_get_stats(tt_ctx* c, tt_stats* out) {
  if (!c || !out) return TT_ERR_INVALID;
  *out = c->stats;
  if (c->uploaded) {
    TT_CUDA(c, cudaSetDevice(c->device));
    unsigned long long s[8];
    TT_CUDA(c, cudaMemcpy(s, c->d_stats, sizeof(s), cudaMemcpyDeviceToHost));
    out->node_visits = s[0];
    out->tri_tests = s[1];
    out->shadow_node_visits = s[2];
    out->shadow_tri_tests = s[3];
    out->extension_rays = s[4];
    out->shadow_rays = s[5];
    unsigned int errw = 0;
    TT_CUDA(c, cudaMemcpy(&errw, c->d_err, sizeof(errw), cudaMemcpyDeviceToHost));
    out->error_flags |= errw;
  }
  out->bvh_nodes = c->bvh_nodes;
  out->bvh_node_bytes = c->bvh_node_bytes;
  out->tri_bytes = 48;
  out->bvh_depth = c->bvh_depth;
  return TT_OK;
}

tt_status tt_reset_stats(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  c->stats = tt_stats{};
  if (c->uploaded) {
    TT_CUDA(c, cudaSetDevice(c->device));
    TT_CUDA(c, cudaMemsetAsync(c->d_stats, 0, 8 * sizeof(unsigned long long), c->stream));
    TT_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return TT_OK;
}

tt_status tt_last_error(tt_ctx* c, char* buf, int32_t n) {
  if (!buf || n <= 0) return TT_ERR_INVALID;
  std::string msg;
  if (c) msg = c->err;
  else {
    std::lock_guard<std::mutex> g(g_err_mutex);
    msg = g_create_error;
  }
  std::snprintf(buf, (size_t)n, "%s", msg.c_str());
  return TT_OK;
}

void tt_destroy(tt_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->d_records) cudaFree(c->d_records);
  if (c->d_rec_count) cudaFree(c->d_rec_count);
  c->gnet.reset();
  c->tree.reset();
  c->path_mem.free_all();
  c->scene_mem.free_all();
  if (c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  delete c;
}

// ---- Learned guiding ----------------------------------------------------------------
tt_status tt_set_guiding(tt_ctx* c, const tt_guiding_params* gp) {
  if (!c || !gp) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  if (!gp->enabled) {
    c->dev.guide = 0;
    c->dev.guide_record = 0;
    c->gparams = *gp;
    return TT_OK;
  }
  if (c->dev.algo != TT_ALGO_PT) return fail(c, TT_ERR_INVALID, "guiding needs algo pt");
  if (gp->record_pool < 0 || gp->batch < 0 || gp->steps_per_pass < 0 || gp->max_depth < 0 ||
      !(gp->learning_rate >= 0.f) || gp->train < 0 || gp->train > 2 ||
      (gp->method != TT_GUIDE_LEARNED && gp->method != TT_GUIDE_TREE) || gp->tree_subdivision < 0 ||
      gp->tree_em_iters < 0 || (gp->network != TT_GUIDE_NET_TCGEN05 && gp->network != TT_GUIDE_NET_MMA) ||
      (gp->tree_distribution != TT_TREE_VMF && gp->tree_distribution != TT_TREE_QUADTREE))
    return fail(c, TT_ERR_INVALID, "bad guiding parameters");
  const int cap = gp->record_pool > 0 ? gp->record_pool : (1 << 16);
  // A tree fitted with the other directional distribution starts over.
  if (c->tree && c->tree->distribution != gp->tree_distribution) c->tree.reset();
  if (gp->method == TT_GUIDE_TREE && !c->tree) {
    c->tree = std::make_unique<TreeGuide>();
    std::string gerr;
    c->tree->distribution = gp->tree_distribution;
    if (!c->tree->init(gp->tree_subdivision, c->stream, &gerr)) {
      c->tree.reset();
      return fail(c, TT_ERR_CUDA, gerr);
    }
  }
  if (c->tree) c->tree->em_iters = gp->tree_em_iters;
  if (!c->gnet) {
    c->gnet = std::make_unique<GuideNet>();
    std::string gerr;
    if (!c->gnet->init(gp->seed, &gerr)) {
      c->gnet.reset();
      return fail(c, TT_ERR_CUDA, gerr);
    }
  }
  if (cap != c->rec_cap) {
    if (c->d_records) cudaFree(c->d_records);
    c->d_records = nullptr;
    c->rec_cap = 0;
    TT_CUDA(c, cudaMalloc(&c->d_records, (size_t)cap * sizeof(GuideRecord)));
    if (!c->d_rec_count) TT_CUDA(c, cudaMalloc(&c->d_rec_count, sizeof(int)));
    c->rec_cap = cap;
    c->ps_guided = false;  // the path state picks up the new record buffer
    TT_CUDA(c, cudaMemset(c->d_rec_count, 0, sizeof(int)));
    c->rec_seen = 0;
    c->rec_rate = 0.0;
  }
  if (gp->train == 1) {
    // Training scratch for one mini-batch now, not inside the first pass.
    std::string gerr;
    if (!c->gnet->ensure_capacity(std::min(cap, gp->batch > 0 ? gp->batch : 8192), &gerr))
      return fail(c, TT_ERR_CUDA, gerr);
  }
  c->gparams = *gp;
  c->gnet->wgrad_tc = gp->network == TT_GUIDE_NET_TCGEN05;
  c->dev.guide_w16 = c->gnet->params16;
  c->dev.guide_w32 = c->gnet->params;
  c->dev.guide = 1;
  c->dev.guide_method = gp->method;
  c->dev.guide_net = gp->network;
  if (gp->method == TT_GUIDE_TREE) tree_to_dev(c);
  c->dev.guide_record = gp->train ? 1 : 0;
  c->dev.guide_depth = gp->max_depth > 0 ? gp->max_depth : (1 << 30);
  return TT_OK;
}

int32_t tt_guide_num_params(void) { return kGParams; }

static tt_status guide_prep(tt_ctx* c) {
  if (!c) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  if (!c->gnet) {
    c->gnet = std::make_unique<GuideNet>();
    std::string gerr;
    if (!c->gnet->init(1, &gerr)) {
      c->gnet.reset();
      return fail(c, TT_ERR_CUDA, gerr);
    }
  }
  return TT_OK;
}

tt_status tt_guide_get_params(tt_ctx* c, float* out, int32_t n) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!out || n != kGParams) return fail(c, TT_ERR_INVALID, "parameter count mismatch");
  TT_CUDA(c, cudaMemcpy(out, c->gnet->params, kGParams * sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_set_params(tt_ctx* c, const float* in, int32_t n) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!in || n != kGParams) return fail(c, TT_ERR_INVALID, "parameter count mismatch");
  std::string gerr;
  if (!c->gnet->set_params(in, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
  return TT_OK;
}

static tt_status guide_forward(tt_ctx* c, const float* features, int32_t n, float* out, bool tcgen05) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!features || !out || n <= 0) return fail(c, TT_ERR_INVALID, "bad batch");
  std::string gerr;
  if (!c->gnet->ensure_capacity(n, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
  std::vector<__nv_bfloat16> x((size_t)n * kGIn);
  for (size_t i = 0; i < x.size(); ++i) x[i] = __float2bfloat16(features[i]);
  TT_CUDA(c, cudaMemcpy(c->gnet->x0, x.data(), x.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
  if (tcgen05) {
    if (!c->gnet->forward_tc(c->gnet->x0, n, c->gnet->out, c->stream))
      return fail(c, TT_ERR_LOOP_CAP, "tensor-core forward: a wait timed out");
  } else {
    c->gnet->forward(c->gnet->x0, n, c->gnet->out, c->stream);
  }
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  TT_CUDA(c, cudaGetLastError());
  TT_CUDA(c, cudaMemcpy(out, c->gnet->out, (size_t)n * kGOut * sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_forward_batch(tt_ctx* c, const float* features, int32_t n, float* out) {
  return guide_forward(c, features, n, out, false);
}

tt_status tt_guide_forward_batch_tc(tt_ctx* c, const float* features, int32_t n, float* out) {
  return guide_forward(c, features, n, out, true);
}

// Copies n host records to a temporary device buffer, runs `steps` gradients (and Adam
// steps when train is set) and releases the buffer.
static tt_status guide_batch(tt_ctx* c, const float* records, int32_t n, int32_t steps, bool train, float lr) {
  static_assert(sizeof(GuideRecord) == 14 * sizeof(float), "record layout");
  std::string gerr;
  if (!c->gnet->ensure_capacity(n, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
  GuideRecord* d = nullptr;
  TT_CUDA(c, cudaMalloc(&d, (size_t)n * sizeof(GuideRecord)));
  cudaError_t e = cudaMemcpy(d, records, (size_t)n * sizeof(GuideRecord), cudaMemcpyHostToDevice);
  for (int k = 0; k < steps && e == cudaSuccess; ++k) {
    c->gnet->gradient(d, n, c->stream, train, lr);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(d);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_guide_gradient_batch(tt_ctx* c, const float* records, int32_t n, float* grad, float* loss) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!records || !grad || n <= 0) return fail(c, TT_ERR_INVALID, "bad batch");
  st = guide_batch(c, records, n, 1, false, 0.f);
  if (st != TT_OK) return st;
  TT_CUDA(c, cudaMemcpy(grad, c->gnet->grad, kGParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) TT_CUDA(c, cudaMemcpy(loss, c->gnet->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_gradient_pool_batch(tt_ctx* c, const float* pool, int32_t pool_n, int32_t n, uint64_t seed,
                                       float* grad, float* loss) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!pool || !grad || n <= 0 || pool_n <= 0) return fail(c, TT_ERR_INVALID, "bad batch");
  std::string gerr;
  if (!c->gnet->ensure_capacity(n, &gerr)) return fail(c, TT_ERR_CUDA, gerr);
  GuideRecord* d = nullptr;
  TT_CUDA(c, cudaMalloc(&d, (size_t)pool_n * sizeof(GuideRecord)));
  cudaError_t e = cudaMemcpy(d, pool, (size_t)pool_n * sizeof(GuideRecord), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    c->gnet->gradient(d, n, c->stream, false, 0.f, pool_n, seed);
    e = cudaStreamSynchronize(c->stream);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(d);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  TT_CUDA(c, cudaMemcpy(grad, c->gnet->grad, kGParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) TT_CUDA(c, cudaMemcpy(loss, c->gnet->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_train_batch(tt_ctx* c, const float* records, int32_t n, int32_t steps, float lr, float* loss) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!records || n <= 0 || steps < 0 || !(lr >= 0.f)) return fail(c, TT_ERR_INVALID, "bad batch");
  st = guide_batch(c, records, n, steps, true, lr);
  if (st != TT_OK) return st;
  if (loss) TT_CUDA(c, cudaMemcpy(loss, c->gnet->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_read_records(tt_ctx* c, float* out, int32_t max_records, int32_t* n) {
  if (!c || !out || !n || max_records < 0) return TT_ERR_INVALID;
  *n = 0;
  if (!c->d_rec_count) return TT_OK;
  TT_CUDA(c, cudaSetDevice(c->device));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  int cnt = 0;
  TT_CUDA(c, cudaMemcpy(&cnt, c->d_rec_count, sizeof(int), cudaMemcpyDeviceToHost));
  cnt = (int)std::min<long long>(std::min<long long>((long long)(unsigned)cnt, c->rec_cap), max_records);
  if (cnt > 0) TT_CUDA(c, cudaMemcpy(out, c->d_records, (size_t)cnt * sizeof(GuideRecord), cudaMemcpyDeviceToHost));
  TT_CUDA(c, cudaMemset(c->d_rec_count, 0, sizeof(int)));
  c->rec_seen = 0;
  *n = cnt;
  return TT_OK;
}

tt_status tt_guide_tree_info(tt_ctx* c, int32_t* cells, int32_t* nodes, int32_t* rounds, int64_t* records) {
  if (!c) return TT_ERR_INVALID;
  if (!c->tree) return fail(c, TT_ERR_NOT_READY, "the tree guider is not enabled");
  if (cells) *cells = c->tree->ncells;
  if (nodes) *nodes = (int32_t)c->tree->nodes.size();
  if (rounds) *rounds = c->tree->round;
  if (records) *records = c->tree->records_fitted;
  return TT_OK;
}

tt_status tt_guide_tree_mixtures(tt_ctx* c, float* out, int32_t max_cells) {
  if (!c || !out || max_cells < 0) return TT_ERR_INVALID;
  if (!c->tree) return fail(c, TT_ERR_NOT_READY, "the tree guider is not enabled");
  TT_CUDA(c, cudaSetDevice(c->device));
  TT_CUDA(c, cudaStreamSynchronize(c->stream));
  const int n = std::min(max_cells, c->tree->ncells);
  if (n > 0) TT_CUDA(c, cudaMemcpy(out, c->tree->d_mix, (size_t)n * kTreeMixFloats * sizeof(float), cudaMemcpyDeviceToHost));
  return TT_OK;
}

tt_status tt_guide_tree_lookup_batch(tt_ctx* c, const float* points, int32_t n, int32_t* cells) {
  if (!c || (n > 0 && (!points || !cells)) || n < 0) return TT_ERR_INVALID;
  if (!c->tree) return fail(c, TT_ERR_NOT_READY, "the tree guider is not enabled");
  for (int i = 0; i < n; ++i) cells[i] = c->tree->lookup(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
  return TT_OK;
}

tt_status tt_vmf_fit_batch(const float* records, int32_t n, const float* mixture_in, const float* fit_in,
                           int32_t batch_iters, float* mixture_out, float* fit_out) {
  if (!records || n <= 0 || !mixture_out || !fit_out || batch_iters < 0)
    return fail(nullptr, TT_ERR_INVALID, "tt_vmf_fit_batch: bad arguments");
  std::string err;
  if (!vmf_fit_one(records, n, mixture_in, fit_in, batch_iters, mixture_out, fit_out, &err))
    return fail(nullptr, TT_ERR_CUDA, err);
  return TT_OK;
}

tt_status tt_kdtree_build_batch(const float* points, int32_t n, int32_t min_points, int32_t* cell_of_point,
                                int32_t* cells) {
  if (!points || n <= 0 || !cell_of_point || !cells || min_points < 0)
    return fail(nullptr, TT_ERR_INVALID, "tt_kdtree_build_batch: bad arguments");
  std::vector<TreeNodeHost> nodes;
  *cells = kdtree_build(points, n, min_points > 0 ? min_points : 100, &nodes, cell_of_point);
  return TT_OK;
}

// Children (-1 for a leaf) and weights of a quadtree into caller buffers.
static tt_status write_quad(const QuadDist& q, int32_t cap, int32_t* children, float* weights, float* prior,
                            int32_t* num_nodes) {
  *num_nodes = q.num_nodes();
  if (q.num_nodes() > cap) return fail(nullptr, TT_ERR_CAPACITY, "quadtree larger than the buffers");
  for (int j = 0; j < q.num_nodes(); ++j) {
    for (int k = 0; k < 4; ++k) children[4 * j + k] = q.child[j][k];
    if (weights) weights[j] = q.probs[j];
    if (prior) prior[j] = q.prior[j];
  }
  return TT_OK;
}

tt_status tt_guide_tree_quadtree(tt_ctx* c, int32_t cell, int32_t cap, int32_t* children, float* weights,
                                 int32_t* num_nodes) {
  if (!c || !children || !weights || !num_nodes || cap < 0) return TT_ERR_INVALID;
  if (!c->tree || c->tree->distribution != TT_TREE_QUADTREE)
    return fail(c, TT_ERR_NOT_READY, "the tree guider with quadtrees is not enabled");
  if (cell < 0 || cell >= c->tree->ncells) return fail(c, TT_ERR_INVALID, "no such cell");
  return write_quad(c->tree->quads[cell], cap, children, weights, nullptr, num_nodes);
}

tt_status tt_quadtree_fit_batch(const float* dirs_a, const float* weights_a, int32_t na, const float* dirs_b,
                                const float* weights_b, int32_t nb, int32_t stage, int32_t cap, int32_t* children,
                                float* weights, float* prior, int32_t* num_nodes) {
  if (na < 0 || nb < 0 || (na > 0 && (!dirs_a || !weights_a)) || (nb > 0 && (!dirs_b || !weights_b)) || stage < 0 ||
      stage > 2 || cap < 0 || !children || !weights || !prior || !num_nodes)
    return fail(nullptr, TT_ERR_INVALID, "tt_quadtree_fit_batch: bad arguments");
  auto to_square = [](const float* d, int n) {
    std::vector<float> uv(2 * (size_t)n);
    for (int i = 0; i < n; ++i) dir_to_square(d + 3 * (size_t)i, &uv[2 * (size_t)i]);
    return uv;
  };
  QuadDist q;
  const std::vector<float> ua = to_square(dirs_a, na);
  q.initial_fit(ua.data(), weights_a, na);
  q.bake();
  if (stage >= 1) {
    const std::vector<float> ub = to_square(dirs_b, nb);
    q.incremental_fit(ub.data(), weights_b, nb, 1);
  }
  if (stage >= 2) q.update_and_bake();
  return write_quad(q, cap, children, weights, prior, num_nodes);
}

tt_status tt_quadtree_sample_batch(const int32_t* children, const float* weights, int32_t num_nodes, const float* u,
                                   int32_t n, float* out_dir, float* out_pdf, float* out_pdf_eval) {
  if (!children || !weights || num_nodes <= 0 || n < 0 || (n > 0 && (!u || !out_dir || !out_pdf || !out_pdf_eval)))
    return fail(nullptr, TT_ERR_INVALID, "tt_quadtree_sample_batch: bad arguments");
  // Every child index must name a node after its parent (no cycles, all in range), so that
  // the device walk ends at a leaf.
  for (int j = 0; j < num_nodes; ++j) {
    const int32_t* k = children + 4 * (size_t)j;
    const bool leaf = k[0] < 0;
    for (int q = 0; q < 4; ++q)
      if (leaf ? k[q] >= 0 : (k[q] <= j || k[q] >= num_nodes))
        return fail(nullptr, TT_ERR_INVALID, "tt_quadtree_sample_batch: bad tree");
  }
  if (n == 0) return TT_OK;
  int4* dc = nullptr;
  float *dw = nullptr, *du = nullptr, *dd = nullptr, *dp = nullptr, *de = nullptr;
  cudaError_t e = cudaMalloc(&dc, (size_t)num_nodes * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc(&dw, (size_t)num_nodes * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&du, 2 * (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dd, 3 * (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dp, (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&de, (size_t)n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(dc, children, (size_t)num_nodes * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dw, weights, (size_t)num_nodes * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(du, u, 2 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    launch_quadtree_sample(dc, dw, du, n, dd, dp, de, 0);
    e = cudaDeviceSynchronize();
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out_dir, dd, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(out_pdf, dp, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(out_pdf_eval, de, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  for (void* p : {(void*)dc, (void*)dw, (void*)du, (void*)dd, (void*)dp, (void*)de})
    if (p) cudaFree(p);
  if (e != cudaSuccess) return fail(nullptr, TT_ERR_CUDA, cudaGetErrorString(e));
  return TT_OK;
}

tt_status tt_guide_features_batch(tt_ctx* c, const float* points, int32_t n, float* features) {
  tt_status st = guide_prep(c);
  if (st != TT_OK) return st;
  if (!points || !features || n <= 0) return fail(c, TT_ERR_INVALID, "bad batch");
  float* dp = nullptr;
  __nv_bfloat16* dx = nullptr;
  TT_CUDA(c, cudaMalloc(&dp, (size_t)n * 9 * sizeof(float)));
  if (cudaMalloc(&dx, (size_t)n * kGIn * sizeof(__nv_bfloat16)) != cudaSuccess) {
    cudaFree(dp);
    return fail(c, TT_ERR_CUDA, "allocation failed");
  }
  cudaError_t e = cudaMemcpy(dp, points, (size_t)n * 9 * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    c->gnet->features(dp, n, dx, c->stream);
    e = cudaStreamSynchronize(c->stream);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  std::vector<__nv_bfloat16> hx((size_t)n * kGIn);
  if (e == cudaSuccess) e = cudaMemcpy(hx.data(), dx, hx.size() * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost);
  cudaFree(dp);
  cudaFree(dx);
  if (e != cudaSuccess) return fail(c, TT_ERR_CUDA, cudaGetErrorString(e));
  for (size_t i = 0; i < hx.size(); ++i) features[i] = __bfloat162float(hx[i]);
  return TT_OK;
}

// ---- Multi-view batches ---------------------------------------------------------------
// All views of a batch are rendered as one wavefront over the concatenation of their
// (pixel, sample) ranges.  The first wave runs eagerly (it loads the kernels and does the
// one-time launch set-up); the per-wave launch sequence is then captured once into a CUDA
// graph whose kernels read the wave's arguments from device memory and which advances the
// wave index itself, and the graph is replayed for every further wave.
static tt_status render_views(tt_ctx* c, const tt_view* views, int32_t n, uint64_t seed, float* rgb,
                              int wave_limit, int grid, float* ms_out) {
  if (!c || !views || n <= 0) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  TT_CUDA(c, cudaSetDevice(c->device));
  std::vector<DevView> hv((size_t)n);
  long long paths = 0, npix_total = 0;
  for (int v = 0; v < n; ++v) {
    const tt_camera& cm = views[v].camera;
    if (cm.xres <= 0 || cm.yres <= 0 || views[v].spp <= 0 ||
        (cm.kind != TT_CAMERA_PINHOLE && cm.kind != TT_CAMERA_FISHEYE))
      return fail(c, TT_ERR_INVALID, "view " + std::to_string(v) + ": bad camera or spp");
    hv[v].cam = make_dev_camera(cm);
    hv[v].npix = cm.xres * cm.yres;
    hv[v].spp = views[v].spp;
    hv[v].pix_begin = (int)npix_total;
    hv[v].path_begin = paths;
    hv[v].seed = seed + (uint64_t)v;
    hv[v].cam_track = c->dev.cam_track;
    npix_total += hv[v].npix;
    paths += (long long)hv[v].npix * hv[v].spp;
    if (npix_total > (1ll << 30)) return fail(c, TT_ERR_CAPACITY, "views hold more than 2^30 pixels");
  }
  int cap = (int)std::min<long long>(paths, wave_limit);
  if (c->dev.guide_record) {
    const double expected = c->rec_rate * (double)paths;
    c->dev.guide_keep = expected > 0.0 ? (float)std::min(1.0, 0.8 * c->rec_cap / expected) : 1.f;
  }
  c->dev.guide_cold = (c->dev.guide && c->dev.guide_method == TT_GUIDE_LEARNED && c->gnet && c->gnet->fresh) ? 1 : 0;
  tt_status st = ensure_path_state_fit(c, &cap);
  if (st != TT_OK) return st;
  const int nwaves = (int)((paths + cap - 1) / cap);
  std::vector<ViewWave> hw((size_t)nwaves);
  for (int k = 0; k < nwaves; ++k) {
    hw[k].wave_start = (long long)k * cap;
    hw[k].wave_paths = (int)std::min<long long>(cap, paths - hw[k].wave_start);
  }
  DeviceBuffers m;
  m.stream = c->stream;
  DevView* d_views = (DevView*)m.alloc(hv.size() * sizeof(DevView));
  ViewWave* d_waves = (ViewWave*)m.alloc(hw.size() * sizeof(ViewWave));
  int* d_idx = (int*)m.alloc(sizeof(int));
  float* d_acc = (float*)m.alloc(3 * (size_t)npix_total * sizeof(float));
  float* d_light = (float*)m.alloc(3 * (size_t)npix_total * sizeof(float));
  float* d_rgb = (float*)m.alloc(3 * (size_t)npix_total * sizeof(float));
  if (!d_views || !d_waves || !d_idx || !d_acc || !d_light || !d_rgb) {
    m.free_all();
    return fail(c, TT_ERR_CUDA, "device allocation failed");
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> wave_end((size_t)nwaves, nullptr);  // recorded after each wave
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t& e : wave_end)
      if (e) cudaEventDestroy(e);
    m.free_all();
  };
  auto check = [&](cudaError_t e) -> tt_status {
    if (e == cudaSuccess) return TT_OK;
    cleanup();
    return fail(c, TT_ERR_CUDA, std::string("multi-view pass: ") + cudaGetErrorString(e));
  };
  if ((st = check(cudaMemcpyAsync(d_views, hv.data(), hv.size() * sizeof(DevView), cudaMemcpyHostToDevice,
                                  c->stream))) != TT_OK)
    return st;
  if ((st = check(cudaMemcpyAsync(d_waves, hw.data(), hw.size() * sizeof(ViewWave), cudaMemcpyHostToDevice,
                                  c->stream))) != TT_OK)
    return st;
  cudaMemsetAsync(d_idx, 0, sizeof(int), c->stream);
  cudaMemsetAsync(d_acc, 0, 3 * (size_t)npix_total * sizeof(float), c->stream);
  cudaMemsetAsync(d_light, 0, 3 * (size_t)npix_total * sizeof(float), c->stream);
  if (c->dev.num_media > 0) {
    // Medium tracker at each view's camera, written into its DevView.
    for (int v = 0; v < n; ++v) {
      const tt_camera& cm = views[v].camera;
      uint2* dst = reinterpret_cast<uint2*>(reinterpret_cast<char*>(d_views + v) + offsetof(DevView, cam_track));
      launch_init_tracker(c->dev, make_float3(cm.pos[0], cm.pos[1], cm.pos[2]),
                          make_float3(c->bb_lo[0], c->bb_lo[1], c->bb_lo[2]),
                          make_float3(c->bb_hi[0], c->bb_hi[1], c->bb_hi[2]), dst, c->d_err, c->stream);
    }
  }
  Framebuffer fb{d_acc, d_light};
  const int rounds = c->rounds;
  const DevScene& sc = c->dev;
  PathState& ps = c->ps;
  auto wave = [&](cudaStream_t s) {
    cudaMemsetAsync(ps.counters, 0, kCountersPerBounce * (size_t)(rounds + 3) * sizeof(int), s);
    launch_generate_views(sc, ps, d_waves, d_idx, d_views, n, grid, s);
    for (int b = 0; b < rounds; ++b) {
      launch_shadow(sc, ps, fb, b, false, nullptr, grid, s);
      launch_flush(sc, ps, fb, b, grid, s);
      launch_extend(sc, ps, b, false, nullptr, grid, s);
      if (sc.num_media > 0) launch_track(sc, ps, b, grid, s);
      launch_shade(sc, ps, b, grid, s);
      if (sc.guide && b < sc.guide_depth) launch_guide(sc, ps, b, s);
    }
    launch_shadow(sc, ps, fb, rounds, false, nullptr, grid, s);
    launch_flush(sc, ps, fb, rounds, grid, s);
    k_tally<<<1, 32, 0, s>>>(ps.counters, rounds, c->d_stats);
    launch_wave_advance(d_idx, s);
  };
  int per_wave = 4 + rounds * (3 + (sc.num_media > 0)) + (sc.guide ? std::min(rounds, sc.guide_depth) : 0) + 2;
  for (int b = 0; b < rounds; ++b) per_wave += shade_launches(sc, ps, b);
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, c->stream);
  bool stopped = false;
  int done_waves = 0;
  for (cudaEvent_t& e : wave_end)
    if ((st = check(cudaEventCreate(&e))) != TT_OK) return st;
  wave(c->stream);  // eager first wave
  cudaEventRecord(wave_end[0], c->stream);
  ++done_waves;
  if ((st = check(cudaGetLastError())) != TT_OK) return st;
  if (nwaves > 1) {
    if ((st = check(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal))) != TT_OK) return st;
    wave(c->stream);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if ((st = check(ce)) != TT_OK) return st;
    for (; done_waves < nwaves; ++done_waves) {
      if (c->stop.load()) { stopped = true; break; }
      if ((st = check(cudaGraphLaunch(exec, c->stream))) != TT_OK) return st;
      cudaEventRecord(wave_end[done_waves], c->stream);
    }
  }
  launch_resolve_views(d_acc, d_light, d_views, n, (int)npix_total, d_rgb, c->stream);
  cudaEventRecord(ev1, c->stream);
  if ((st = check(cudaMemcpyAsync(rgb, d_rgb, 3 * (size_t)npix_total * sizeof(float), cudaMemcpyDeviceToHost,
                                  c->stream))) != TT_OK)
    return st;
  if ((st = check(cudaStreamSynchronize(c->stream))) != TT_OK) return st;
  if ((st = check(cudaGetLastError())) != TT_OK) return st;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0, ev1);
  if (ms_out) *ms_out = ms;
  // A view is complete when the wave holding its last path has finished.
  c->views_done_ms.assign((size_t)n, -1.f);
  for (int v = 0; v < n; ++v) {
    const long long last = hv[v].path_begin + (long long)hv[v].npix * hv[v].spp - 1;
    const int w = (int)(last / cap);
    if (w < done_waves) cudaEventElapsedTime(&c->views_done_ms[v], ev0, wave_end[w]);
  }
  c->stats.pass_ms += ms;
  c->stats.kernel_launches += (uint64_t)done_waves * per_wave + 1;
  c->stats.extend_launches += (uint64_t)done_waves * rounds;
  c->stats.shadow_launches += (uint64_t)done_waves * (rounds + 1);
  c->stats.paths += (uint64_t)std::min<long long>(paths, (long long)done_waves * cap);
  cleanup();
  if (c->dev.guide_record && !stopped && c->gparams.train == 1) {
    const tt_status gs = guide_train(c, paths);
    if (gs != TT_OK) return gs;
  }
  unsigned int errw = 0;
  TT_CUDA(c, cudaMemcpy(&errw, c->d_err, sizeof(errw), cudaMemcpyDeviceToHost));
  if (errw) {
    c->stats.error_flags |= errw;
    return fail(c, TT_ERR_LOOP_CAP, "a device loop hit its cap (error word " + std::to_string(errw) + ")");
  }
  if (stopped) return fail(c, TT_ERR_INTERRUPTED, "stopped by tt_request_stop");
  return TT_OK;
}

tt_status tt_render_views(tt_ctx* c, const tt_view* views, int32_t n, uint64_t seed, float* rgb) {
  if (!c || !rgb) return TT_ERR_INVALID;
  const int wave_limit = c->params.wave_paths > 0 ? c->params.wave_paths : kDefaultWave;
  return render_views(c, views, n, seed, rgb, wave_limit, c->grid, nullptr);
}

tt_status tt_views_completion_ms(tt_ctx* c, float* out, int32_t n) {
  if (!c || !out) return TT_ERR_INVALID;
  if ((size_t)n != c->views_done_ms.size()) return fail(c, TT_ERR_INVALID, "view count differs from the last batch");
  std::copy(c->views_done_ms.begin(), c->views_done_ms.end(), out);
  return TT_OK;
}

tt_status tt_autotune_views(tt_ctx* c, const tt_view* views, int32_t n, tt_tune_result* out) {
  if (!c || !views || n <= 0 || !out) return TT_ERR_INVALID;
  if (!c->uploaded) return fail(c, TT_ERR_NOT_READY, "tt_upload_scene has not run");
  // Probe batch: every view at one sample.
  std::vector<tt_view> probe(views, views + n);
  long long npix = 0;
  for (auto& v : probe) {
    v.spp = 1;
    npix += (long long)v.camera.xres * v.camera.yres;
  }
  if (npix <= 0 || npix > (1ll << 30)) return fail(c, TT_ERR_INVALID, "bad views");
  std::vector<float> rgb(3 * (size_t)npix);
  const int waves[] = {1 << 22, 1 << 24, 1 << 25, 1 << 26};
  const int base_grid = c->grid;
  const int grids[] = {base_grid / 2 > 0 ? base_grid / 2 : base_grid, base_grid, 2 * base_grid};
  *out = tt_tune_result{};
  double best = 1e300;
  int k = 0;
  int best_block = 256;
  bool best_wide = false;
  auto probe_one = [&](int w, int g, int block, bool wide) -> tt_status {
    float ms = 0.f;
    c->dev.block = block;
    tt_status st = render_views(c, probe.data(), n, 1, rgb.data(), w, g, &ms);
    if (st != TT_OK) return st;
    if (k < TT_TUNE_MAX) {
      out->candidate_wave[k] = w;
      out->candidate_grid[k] = g;
      out->candidate_ms[k] = ms;
      out->candidate_block[k] = block;
      out->candidate_width[k] = wide ? 8 : (c->dev.nodes4 ? 4 : 2);
    }
    ++k;
    if (ms < best) {
      best = ms;
      out->wave_paths = w;
      out->grid = g;
      out->ms = ms;
      best_block = block;
      best_wide = wide;
    }
    return TT_OK;
  };
  const bool start_wide = c->dev.wide != 0;
  tt_status st = use_layout(c, false);
  if (st != TT_OK) return st;
  // One untimed call first (path state at the largest size, kernels loaded).
  c->dev.block = 256;
  st = render_views(c, probe.data(), n, 1, rgb.data(), waves[3], base_grid, nullptr);
  if (st != TT_OK) return st;
  for (int w : waves)
    for (int g : grids)
      if ((st = probe_one(w, g, 256, false)) != TT_OK) return st;
  // At the best queue capacity and launch width: half-size blocks, then the 8-wide BVH.
  const int w0 = out->wave_paths, g0 = out->grid;
  if ((st = probe_one(w0, 2 * g0, 128, false)) != TT_OK) return st;
  const int g1 = best_block == 128 ? 2 * g0 : g0;
  if ((st = use_layout(c, true)) != TT_OK) return st;
  c->dev.block = best_block;
  if ((st = render_views(c, probe.data(), n, 1, rgb.data(), w0, g1, nullptr)) != TT_OK) return st;  // warm-up
  if ((st = probe_one(w0, g1, best_block, true)) != TT_OK) return st;
  (void)start_wide;
  out->candidates = k;
  out->block = best_block;
  out->bvh_width = best_wide ? 8 : (c->layouts[0].nodes4 || (!c->dev.wide && c->dev.nodes4) ? 4 : 2);
  if ((st = use_layout(c, best_wide)) != TT_OK) return st;
  c->dev.block = best_block;
  c->params.wave_paths = out->wave_paths;
  c->grid = out->grid;
  return TT_OK;
}

}  // extern "C"
