// tt_render_pass_noalloc: a render pass that allocates no memory.
//
// The regular pass (tt_render_pass) keeps its wavefront path state in device memory that
// the library cudaMallocs on first use and grows on demand.  Some callers cannot let a
// library allocate at render time: a renderer embedded in an application that owns all
// GPU memory through its own pool or a fixed budget, or code running where a cudaMalloc
// would synchronise the device and stall other work.  For them this entry point keeps
// the path state in one statically sized device array that lives in the library image,
// and writes into output buffers the caller provides.
//
// Limits and sharing:
//  - at most kNoAllocMaxPaths = 65,536 camera samples (spp x pixels) per call, and
//    max_ray_depth <= kNoAllocMaxDepth; larger requests return TT_ERR_CAPACITY;
//  - the scratch array (about 14.7 MB) is part of the library image, so every GPU that
//    loads the library holds it until the process exits;
//  - all calls on a device share the one array: calls that overlap on the GPU (different
//    streams or host threads without ordering) race and corrupt each other;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that first call
//    before any stream capture begins.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/toytrace_gpu.h"
#include "tt_internal.h"

using namespace tt;

namespace {

constexpr int kNoAllocMaxPaths = 1 << 16;
constexpr int kNoAllocMaxDepth = 1000;
constexpr int kNoAllocMaxDevices = 64;

// Per-path bytes: 10 float4 + 1 uint4 + 2 u64 + 2 uint2 + 4 int queues = 224 B (the
// medium-tracking arrays are carved for every scene); each of the 21 arrays is padded to a
// 256-byte boundary.
constexpr size_t kPathBytes = 10 * sizeof(float4) + sizeof(uint4) + 2 * sizeof(unsigned long long) +
                              2 * sizeof(uint2) + 4 * sizeof(int);
constexpr size_t kCounterBytes = (size_t)kCountersPerBounce * (kNoAllocMaxDepth + 3) * sizeof(int);
constexpr size_t kErrBytes = 256;
constexpr size_t kPadBytes = 21 * 256;
constexpr size_t kNoAllocScratchBytes = kNoAllocMaxPaths * kPathBytes + kCounterBytes + kErrBytes + kPadBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
cudaError_t scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

// Carves the path-state arrays out of the scratch array (every piece stays 16-byte aligned).
PathState carve(unsigned char* base, int cap) {
  PathState p{};
  unsigned char* q = base;
  auto take = [&q](size_t bytes) {
    unsigned char* r = q;
    q += (bytes + 255) & ~(size_t)255;
    return r;
  };
  const size_t n = (size_t)cap;
  p.cap = cap;
  p.ray_o = (float4*)take(n * sizeof(float4));
  p.ray_d = (float4*)take(n * sizeof(float4));
  p.hit = (float4*)take(n * sizeof(float4));
  p.beta = (float4*)take(n * sizeof(float4));
  p.accum = (float4*)take(n * sizeof(float4));
  p.sh_o = (float4*)take(n * sizeof(float4));
  p.sh_d = (float4*)take(n * sizeof(float4));
  p.sh_c = (float4*)take(n * sizeof(float4));
  p.meta = (uint4*)take(n * sizeof(uint4));
  p.rng_state = (unsigned long long*)take(n * 8);
  p.rng_inc = (unsigned long long*)take(n * 8);
  p.ext_q[0] = (int*)take(n * sizeof(int));
  p.ext_q[1] = (int*)take(n * sizeof(int));
  p.sh_q = (int*)take(n * sizeof(int));
  p.done_q = (int*)take(n * sizeof(int));
  p.track = (uint2*)take(n * sizeof(uint2));
  p.vol = (float4*)take(n * sizeof(float4));
  p.sh_track = (uint2*)take(n * sizeof(uint2));
  p.sh_med = (float4*)take(n * sizeof(float4));
  p.counters = (int*)take(kCounterBytes);
  p.err = (unsigned int*)take(kErrBytes);
  return p;
}
static_assert(kNoAllocScratchBytes >= kNoAllocMaxPaths * kPathBytes + kCounterBytes + kErrBytes + kPadBytes,
              "scratch layout");
inline bool carve_fits(const unsigned char* base, const PathState& p) {
  return (const unsigned char*)p.err + kErrBytes <= base + kNoAllocScratchBytes;
}

}  // namespace

namespace tt {
// Scene record of an uploaded context (defined in tt_capi.cu).
bool context_scene(tt_ctx* ctx, DevScene* scene, int* device, int* npix, int* max_depth, std::string** err);
}

extern "C" tt_status tt_render_pass_noalloc(tt_ctx* ctx, int32_t spp, uint64_t seed, int32_t pixel_begin,
                                            int32_t pixel_end, uint64_t sample_offset, float* d_accum,
                                            float* d_light_accum, void* stream) {
  DevScene scene{};
  int device = 0, npix = 0, depth = 0;
  std::string* err = nullptr;
  if (!ctx) return TT_ERR_INVALID;
  if (!context_scene(ctx, &scene, &device, &npix, &depth, &err)) return TT_ERR_NOT_READY;
  // The learned guide needs buffers of its own; this pass renders unguided.
  scene.guide = 0;
  scene.guide_record = 0;
  auto fail = [err](tt_status s, const std::string& msg) {
    *err = msg;
    return s;
  };
  if (!d_accum || !d_light_accum) return fail(TT_ERR_INVALID, "tt_render_pass_noalloc: output buffer is NULL");
  // The null-path tracer's per-path matrices have no room in the static array.
  if (scene.algo != TT_ALGO_PT) return fail(TT_ERR_INVALID, "tt_render_pass_noalloc: algo pt only");
  if (spp <= 0) return fail(TT_ERR_INVALID, "tt_render_pass_noalloc: spp must be positive");
  if (pixel_begin < 0 || pixel_end > npix || pixel_begin >= pixel_end)
    return fail(TT_ERR_INVALID, "tt_render_pass_noalloc: bad pixel range");
  const long long paths = (long long)spp * (pixel_end - pixel_begin);
  if (paths > kNoAllocMaxPaths)
    return fail(TT_ERR_CAPACITY, "tt_render_pass_noalloc: " + std::to_string(paths) +
                                     " camera samples requested; at most 65536 (spp x pixels) per call");
  if (depth > kNoAllocMaxDepth)
    return fail(TT_ERR_CAPACITY, "tt_render_pass_noalloc: max_ray_depth above 1000");
  // A pending stop request ends this pass before it starts, as it ends every later
  // tt_render_pass.  Once launched, the pass (at most 65,536 samples) runs to completion.
  if (tt_stop_requested(ctx)) return fail(TT_ERR_INTERRUPTED, "tt_render_pass_noalloc: stop requested");
  if (device < 0 || device >= kNoAllocMaxDevices) return fail(TT_ERR_INVALID, "device ordinal out of range");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(TT_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  unsigned char* base = nullptr;
  e = scratch_address(device, &base);
  if (e != cudaSuccess) return fail(TT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  PathState p = carve(base, kNoAllocMaxPaths);
  if (!carve_fits(base, p)) return fail(TT_ERR_CAPACITY, "tt_render_pass_noalloc: scratch layout overflow");
  // The counters and the error word must start at zero; the path arrays are written before
  // they are read by every stage.
  const size_t zero_bytes = (size_t)((unsigned char*)p.err + kErrBytes - (unsigned char*)p.counters);
  e = cudaMemsetAsync(p.counters, 0, zero_bytes, st);
  if (e != cudaSuccess) return fail(TT_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  Framebuffer fb{d_accum, d_light_accum};
  WaveArgs w;
  w.wave_start = 0;
  w.wave_paths = (int)paths;
  w.pixel_begin = pixel_begin;
  w.npix_range = pixel_end - pixel_begin;
  w.npix_total = npix;
  w.sample_offset = sample_offset;
  w.seed = seed;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int grid = sms * kernel_blocks_per_sm();
  launch_generate(scene, p, fb, w, grid, st);
  for (int b = 0; b < depth; ++b) {
    launch_shadow(scene, p, fb, b, false, nullptr, grid, st);
    launch_flush(scene, p, fb, b, grid, st);
    launch_extend(scene, p, b, false, nullptr, grid, st);
    if (scene.num_media > 0) launch_track(scene, p, b, grid, st);
    launch_shade(scene, p, b, grid, st);
  }
  launch_shadow(scene, p, fb, depth, false, nullptr, grid, st);
  launch_flush(scene, p, fb, depth, grid, st);
  unsigned int errw = 0;
  e = cudaMemcpyAsync(&errw, p.err, sizeof(errw), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TT_ERR_CUDA, std::string("tt_render_pass_noalloc: ") + cudaGetErrorString(e));
  if (errw) return fail(TT_ERR_LOOP_CAP, "a device loop hit its cap (error word " + std::to_string(errw) + ")");
  return TT_OK;
}
