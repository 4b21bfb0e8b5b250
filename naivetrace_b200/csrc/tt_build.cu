// Device BVH construction: PLOC (parallel locally-ordered clustering, Meister and Bittner
// 2018) over Morton-ordered primitives, a bottom-up SAH pass that collapses small subtrees
// into leaves of at most four primitives, and emission in the binary layout of tt_bvh.h.
// Replaces the Embree scene commit (Scene::BuildAccelStructure, scene.cxx:116-141) on the
// GPU: the host sends the mesh once and the tree is built next to it.
//
// Clustering: clusters sit in Morton order; each finds the neighbour within kRadius
// positions whose merged box has the least surface area (ties broken by the pair's
// positions, so the relation is a strict order and the globally best pair is always
// mutual); mutual nearest neighbours merge into a new node at the lower position, and the
// array is compacted.  Node ids grow with the iteration that created them, so children
// always precede parents, and one kernel per iteration range walks the tree bottom-up or
// top-down.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "tt_build.h"
#include "tt_internal.h"

namespace tt {
namespace {

// PLOC neighbourhood (positions on either side); TT_PLOC_RADIUS overrides.  On the terrain
// workload a small radius gave the lowest SAH cost (radius 2: 35.4, 8: 37.2, 16: 38.1,
// 64: 40.1; the host binned-SAH builder: 33.4).
constexpr int kDefaultRadius = 2;
constexpr int kMaxLeaf = 4;
constexpr int kMaxIterations = 4096;
constexpr int kThreads = 256;

struct Aabb {
  float3 lo, hi;
};

__device__ __forceinline__ float half_area(const Aabb& b) {
  const float dx = b.hi.x - b.lo.x, dy = b.hi.y - b.lo.y, dz = b.hi.z - b.lo.z;
  return dx * dy + dy * dz + dz * dx;
}
__device__ __forceinline__ Aabb merge(const Aabb& a, const Aabb& b) {
  return Aabb{make_float3(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z)),
              make_float3(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z))};
}

// Order-preserving map of floats to unsigned ints (for atomic min / max of floats).
__device__ __forceinline__ unsigned ordered(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ Aabb prim_box(const BuildInput& in, uint32_t global) {
  Aabb b;
  if (global < in.num_triangles) {
    const uint32_t* t = in.indices + 3 * (size_t)global;
    const float* v0 = in.vertices + 3 * (size_t)t[0];
    const float* v1 = in.vertices + 3 * (size_t)t[1];
    const float* v2 = in.vertices + 3 * (size_t)t[2];
    b.lo = make_float3(fminf(v0[0], fminf(v1[0], v2[0])), fminf(v0[1], fminf(v1[1], v2[1])),
                       fminf(v0[2], fminf(v1[2], v2[2])));
    b.hi = make_float3(fmaxf(v0[0], fmaxf(v1[0], v2[0])), fmaxf(v0[1], fmaxf(v1[1], v2[1])),
                       fmaxf(v0[2], fmaxf(v1[2], v2[2])));
  } else {
    // One ulp outside centre -/+ radius (SphereBoundsFunc, embreeaccelerator.cxx:263-281).
    const float* q = in.spheres + 4 * (size_t)(global - in.num_triangles);
    b.lo = make_float3(nextafterf(q[0] - q[3], -INFINITY), nextafterf(q[1] - q[3], -INFINITY),
                       nextafterf(q[2] - q[3], -INFINITY));
    b.hi = make_float3(nextafterf(q[0] + q[3], INFINITY), nextafterf(q[1] + q[3], INFINITY),
                       nextafterf(q[2] + q[3], INFINITY));
  }
  return b;
}

__global__ void k_prim_boxes(BuildInput in, const uint32_t* set, uint32_t n, Aabb* boxes, unsigned* cbounds) {
  unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Aabb b = prim_box(in, set[i]);
    boxes[i] = b;
    const float c[3] = {0.5f * (b.lo.x + b.hi.x), 0.5f * (b.lo.y + b.hi.y), 0.5f * (b.lo.z + b.hi.z)};
    for (int k = 0; k < 3; ++k) {
      lo[k] = min(lo[k], ordered(c[k]));
      hi[k] = max(hi[k], ordered(c[k]));
    }
  }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&cbounds[k], lo[k]);
      atomicMax(&cbounds[3 + k], hi[k]);
    }
  }
}

__device__ __forceinline__ uint64_t spread21(uint64_t x) {
  x &= 0x1fffffull;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

// 63-bit Morton code of the box centre in the centroid bounds, with one scale for all three
// axes: cubic cells keep the curve's neighbours spatial neighbours in flat scenes.
__global__ void k_morton(const Aabb* boxes, uint32_t n, const unsigned* cbounds, uint64_t* keys, uint32_t* vals) {
  float lo[3], ext[3];
  float e = 0.f;
  for (int k = 0; k < 3; ++k) {
    lo[k] = unordered(cbounds[k]);
    e = fmaxf(e, unordered(cbounds[3 + k]) - lo[k]);
  }
  for (int k = 0; k < 3; ++k) ext[k] = e;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Aabb b = boxes[i];
    const float c[3] = {0.5f * (b.lo.x + b.hi.x), 0.5f * (b.lo.y + b.hi.y), 0.5f * (b.lo.z + b.hi.z)};
    uint64_t code = 0;
    for (int k = 0; k < 3; ++k) {
      const float f = ext[k] > 0.f ? (c[k] - lo[k]) / ext[k] : 0.f;
      const uint64_t q = (uint64_t)fminf(fmaxf(f * 2097152.f, 0.f), 2097151.f);
      code |= spread21(q) << (2 - k);
    }
    keys[i] = code;
    vals[i] = i;
  }
}

// Leaves 0..n-1 in Morton order: node box = primitive box, left = -1 - (set position).
__global__ void k_init_leaves(const Aabb* prim_boxes, const uint32_t* perm, uint32_t n, Aabb* node_box,
                              int* left, int* right, int* clusters) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    node_box[i] = prim_boxes[perm[i]];
    left[i] = -1 - (int)perm[i];
    right[i] = -1;
    clusters[i] = (int)i;
  }
}

// Pair order: merged area, then the pair's lower and higher positions.
__device__ __forceinline__ bool pair_less(float a, int lo, int hi, float b, int blo, int bhi) {
  return a < b || (a == b && (lo < blo || (lo == blo && hi < bhi)));
}

__global__ void k_nearest(const int* clusters, int c, const Aabb* node_box, int radius, int* nn) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const Aabb bi = node_box[clusters[i]];
    float best = INFINITY;
    int bj = -1;
    const int j0 = max(0, i - radius), j1 = min(c - 1, i + radius);
    for (int j = j0; j <= j1; ++j) {
      if (j == i) continue;
      const float a = half_area(merge(bi, node_box[clusters[j]]));
      if (bj < 0 || pair_less(a, min(i, j), max(i, j), best, min(i, bj), max(i, bj))) {
        best = a;
        bj = j;
      }
    }
    nn[i] = bj;
  }
}

// create[i]: i is the lower end of a mutual pair (it makes the new node); keep[i]: i stays
// a cluster after the merge (everything except the higher end of a mutual pair).
__global__ void k_merge_flags(const int* nn, int c, int* create, int* keep) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    create[i] = (mutual && i < j) ? 1 : 0;
    keep[i] = (mutual && i > j) ? 0 : 1;
  }
}

__global__ void k_merge(const int* clusters, int c, const int* nn, const int* create, const int* create_off,
                        const int* keep, const int* keep_off, int next_node, Aabb* node_box, int* left, int* right,
                        int* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    int id = clusters[i];
    if (create[i]) {
      const int j = nn[i];
      const int k = next_node + create_off[i];
      const int a = clusters[i], b = clusters[j];
      node_box[k] = merge(node_box[a], node_box[b]);
      left[k] = a;
      right[k] = b;
      id = k;
    }
    out[keep_off[i]] = id;
  }
}

// Bottom-up over one creation range: subtree sizes and SAH costs (traversal step 1,
// primitive test 1 per primitive), whether a subtree of at most kMaxLeaf primitives is
// cheaper as one leaf, and the number of inner nodes the subtree emits.
__global__ void k_costs(int first, int count, uint32_t n, const Aabb* node_box, const int* left, const int* right,
                        int* size, float* cost, unsigned char* collapse, int* inner) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    const int k = first + t;
    const int l = left[k], r = right[k];
    const int sl = l < (int)n ? 1 : size[l], sr = r < (int)n ? 1 : size[r];
    const float cl = l < (int)n ? 1.f : cost[l], cr = r < (int)n ? 1.f : cost[r];
    const float a = half_area(node_box[k]);
    const float split = a > 0.f ? 1.f + (half_area(node_box[l]) * cl + half_area(node_box[r]) * cr) / a
                                : 1.f + cl + cr;
    const int s = sl + sr;
    const float leaf = (float)s;
    const bool as_leaf = s <= kMaxLeaf && leaf <= split;
    size[k] = s;
    cost[k] = as_leaf ? leaf : split;
    collapse[k] = as_leaf ? 1 : 0;
    inner[k] = as_leaf ? 0 : 1 + (l < (int)n ? 0 : inner[l]) + (r < (int)n ? 0 : inner[r]);
  }
}

// Top-down over one creation range: primitive offsets and node indices (both in depth-first
// order: an inner node's first child follows it in memory, its second child follows the
// first child's subtree) and whether the node is emitted as an inner node, lies inside a
// leaf, or is a leaf itself.  state: bit 0 = inside a leaf (set by an ancestor that
// became a leaf).
__global__ void k_topdown(int first, int count, uint32_t n, const int* left, const int* right, const int* size,
                          const unsigned char* collapse, const int* inner, int* offset, int* index,
                          unsigned char* state, int* depth, unsigned char* emit, unsigned* max_depth) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    const int k = first + t;
    const bool inside = state[k] & 1u;
    const bool leafnode = inside || collapse[k];
    emit[k] = leafnode ? 0 : 1;
    const int l = left[k], r = right[k];
    const int sl = l < (int)n ? 1 : size[l];
    offset[l] = offset[k];
    offset[r] = offset[k] + sl;
    state[l] = leafnode ? 1 : 0;
    state[r] = leafnode ? 1 : 0;
    if (!leafnode) {
      depth[l] = depth[k] + 1;
      depth[r] = depth[k] + 1;
      index[l] = index[k] + 1;
      index[r] = index[k] + 1 + (l < (int)n ? 0 : inner[l]);
      atomicMax(max_depth, (unsigned)(depth[k] + 1));
    }
  }
}

// Primitive slots in depth-first order (layout in tt_bvh.h).
__global__ void k_write_slots(BuildInput in, const uint32_t* set, const int* left, const int* offset, uint32_t n,
                              float4* tris) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t pos = (uint32_t)(-1 - left[i]);
    const uint32_t g = set[pos];
    float4* dst = tris + 3 * (size_t)offset[i];
    if (g < in.num_triangles) {
      const uint32_t* t = in.indices + 3 * (size_t)g;
      const float* v0 = in.vertices + 3 * (size_t)t[0];
      const float* v1 = in.vertices + 3 * (size_t)t[1];
      const float* v2 = in.vertices + 3 * (size_t)t[2];
      dst[0] = make_float4(v0[0], v0[1], v0[2], __int_as_float((int)in.prim_ids[pos]));
      dst[1] = make_float4(v1[0], v1[1], v1[2], __int_as_float((int)in.material_ids[g]));
      dst[2] = make_float4(v2[0], v2[1], v2[2], 0.f);
    } else {
      const uint32_t k = g - in.num_triangles;
      const float* q = in.spheres + 4 * (size_t)k;
      dst[0] = make_float4(q[0], q[1], q[2], __int_as_float((int)in.prim_ids[pos]));
      dst[1] = make_float4(q[3], 0.f, 0.f, __int_as_float((int)in.sphere_material_ids[k]));
      dst[2] = make_float4(0.f, 0.f, 0.f, __int_as_float(1));
    }
  }
}

__device__ __forceinline__ int child_ref(int c, uint32_t n, const int* size, const int* offset,
                                         const unsigned char* emit, const int* index) {
  if (c >= (int)n && emit[c]) return index[c];
  const int cnt = c < (int)n ? 1 : size[c];
  return ~(int)(((unsigned)offset[c] << 3) | (unsigned)(cnt - 1));
}

// Emitted inner node k -> device node index[k] (the root is node 0).
__global__ void k_write_nodes(int first, int count, uint32_t n, const Aabb* node_box, const int* left,
                              const int* right, const int* size, const int* offset, const unsigned char* emit,
                              const int* index, float4* nodes) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    const int k = first + t;
    if (!emit[k]) continue;
    const int l = left[k], r = right[k];
    const Aabb a = node_box[l], b = node_box[r];
    float4* d = nodes + 4 * (size_t)index[k];
    d[0] = make_float4(a.lo.x, a.hi.x, a.lo.y, a.hi.y);
    d[1] = make_float4(b.lo.x, b.hi.x, b.lo.y, b.hi.y);
    d[2] = make_float4(a.lo.z, a.hi.z, b.lo.z, b.hi.z);
    d[3] = make_float4(__int_as_float(child_ref(l, n, size, offset, emit, index)),
                       __int_as_float(child_ref(r, n, size, offset, emit, index)), 0.f, 0.f);
  }
}

// 4-wide layout, built top down one level at a time: a 4-wide node starts from a binary
// inner node's two children and, while it has fewer than four, replaces the inner child of
// the largest surface area by that child's two children (the usual collapse of a binary
// tree into a wide one); its remaining inner children become the next level's 4-wide
// nodes, numbered by an atomic counter.  frontier: (binary node, 4-wide index) pairs.
__global__ void k_collapse4(const int2* frontier, int nfront, uint32_t n, const Aabb* node_box, const int* left,
                            const int* right, const int* size, const int* offset, const unsigned char* emit,
                            const int* index, int* counter, int2* next, int* nnext, float4* nodes4) {
  constexpr int kEmpty = 0x7fffffff;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nfront; t += gridDim.x * blockDim.x) {
    const int k = frontier[t].x, i4 = frontier[t].y;
    int slot[4] = {left[k], right[k], -1, -1};
    int m = 2;
    while (m < 4) {
      int best = -1;
      float best_area = -1.f;
      for (int j = 0; j < m; ++j) {
        const int c = slot[j];
        if (c >= (int)n && emit[c]) {
          const float a = half_area(node_box[c]);
          if (a > best_area) {
            best_area = a;
            best = j;
          }
        }
      }
      if (best < 0) break;
      const int c = slot[best];
      slot[best] = left[c];
      slot[m++] = right[c];
    }
    Aabb box[4];
    int ref[4];
    for (int j = 0; j < 4; ++j) {
      if (j >= m) {
        box[j] = Aabb{make_float3(INFINITY, INFINITY, INFINITY), make_float3(-INFINITY, -INFINITY, -INFINITY)};
        ref[j] = kEmpty;
        continue;
      }
      const int c = slot[j];
      box[j] = node_box[c];
      if (c >= (int)n && emit[c]) {
        const int j4 = atomicAdd(counter, 1);
        next[atomicAdd(nnext, 1)] = make_int2(c, j4);
        ref[j] = j4;
      } else {
        ref[j] = child_ref(c, n, size, offset, emit, index);
      }
    }
    float4* d = nodes4 + 8 * (size_t)i4;
    d[0] = make_float4(box[0].lo.x, box[1].lo.x, box[2].lo.x, box[3].lo.x);
    d[1] = make_float4(box[0].hi.x, box[1].hi.x, box[2].hi.x, box[3].hi.x);
    d[2] = make_float4(box[0].lo.y, box[1].lo.y, box[2].lo.y, box[3].lo.y);
    d[3] = make_float4(box[0].hi.y, box[1].hi.y, box[2].hi.y, box[3].hi.y);
    d[4] = make_float4(box[0].lo.z, box[1].lo.z, box[2].lo.z, box[3].lo.z);
    d[5] = make_float4(box[0].hi.z, box[1].hi.z, box[2].hi.z, box[3].hi.z);
    d[6] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
    d[7] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}
// 4-wide root of a tree whose root is a leaf: one slot with the leaf.
__global__ void k_leaf_root4(const Aabb* node_box, int root, int count, float4* nodes4) {
  const Aabb a = node_box[root];
  const float inf = INFINITY;
  nodes4[0] = make_float4(a.lo.x, inf, inf, inf);
  nodes4[1] = make_float4(a.hi.x, -inf, -inf, -inf);
  nodes4[2] = make_float4(a.lo.y, inf, inf, inf);
  nodes4[3] = make_float4(a.hi.y, -inf, -inf, -inf);
  nodes4[4] = make_float4(a.lo.z, inf, inf, inf);
  nodes4[5] = make_float4(a.hi.z, -inf, -inf, -inf);
  const int e = 0x7fffffff;
  nodes4[6] = make_float4(__int_as_float(~(int)(unsigned)(count - 1)), __int_as_float(e), __int_as_float(e),
                          __int_as_float(e));
  nodes4[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Root handling for trees whose root is a leaf: one node with the leaf as child 0 and an
// empty child 1 (inverted box, reference to slot 0 with count 1).
__global__ void k_leaf_root(const Aabb* node_box, int root, int count, float4* nodes) {
  const Aabb a = node_box[root];
  const float inf = INFINITY;
  nodes[0] = make_float4(a.lo.x, a.hi.x, a.lo.y, a.hi.y);
  nodes[1] = make_float4(inf, -inf, inf, -inf);
  nodes[2] = make_float4(a.lo.z, a.hi.z, inf, -inf);
  nodes[3] = make_float4(__int_as_float(~(int)(unsigned)(count - 1)), __int_as_float(~0), 0.f, 0.f);
}

int grid_for(long long n) {
  long long g = (n + kThreads - 1) / kThreads;
  return (int)(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

// Scratch allocations from the library's memory pool, released on scope exit.
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    if (pool_malloc(&p, (count ? count : 1) * sizeof(T), st) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~Scratch() {
    for (void* p : ptrs) pool_free(p, st);
  }
};

}  // namespace

bool device_build_bvh2(const BuildInput& in, const uint32_t* set, uint32_t n, DeviceBvh* out, cudaStream_t st,
                       std::string* err) {
  auto fail = [&](const std::string& m) {
    *err = "device BVH build: " + m;
    return false;
  };
  auto ok = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    *err = std::string("device BVH build: ") + what + ": " + cudaGetErrorString(e);
    return false;
  };
  out->num_nodes = 0;
  out->max_depth = 0;
  out->nodes = nullptr;
  out->tris = nullptr;
  out->nodes4 = nullptr;  // none for an empty tree: traversal uses the binary layout
  out->num_nodes4 = 0;
  if (n == 0) {
    // No primitives: a root with two empty children and one degenerate slot (prim -1).
    float host_node[16];
    const float inf = INFINITY;
    const float h[12] = {inf, -inf, inf, -inf, inf, -inf, inf, -inf, inf, -inf, inf, -inf};
    for (int k = 0; k < 12; ++k) host_node[k] = h[k];
    const int32_t r0 = ~0, zero = 0;
    std::memcpy(&host_node[12], &r0, 4);
    std::memcpy(&host_node[13], &r0, 4);
    std::memcpy(&host_node[14], &zero, 4);
    std::memcpy(&host_node[15], &zero, 4);
    float host_tri[12] = {0.f};
    const int32_t none = -1;
    std::memcpy(&host_tri[3], &none, 4);
    if (!ok(pool_malloc((void**)&out->nodes, sizeof(host_node), st), "allocation") ||
        !ok(pool_malloc((void**)&out->tris, sizeof(host_tri), st), "allocation"))
      return false;
    if (!ok(cudaMemcpyAsync(out->nodes, host_node, sizeof(host_node), cudaMemcpyHostToDevice, st), "copy") ||
        !ok(cudaMemcpyAsync(out->tris, host_tri, sizeof(host_tri), cudaMemcpyHostToDevice, st), "copy") ||
        !ok(cudaStreamSynchronize(st), "sync"))
      return false;
    out->num_nodes = 1;
    return true;
  }
  Scratch sc(st);
  // Small values read back (or sent) during the build go through page-locked host memory:
  // a copy into a pageable stack variable would make every one of them a synchronous round
  // trip, four per clustering iteration.  One 256-byte area per host thread that builds,
  // kept for the thread's lifetime.
  thread_local int* hb = nullptr;
  if (!hb && !ok(cudaHostAlloc((void**)&hb, 256, cudaHostAllocPortable), "page-locked read-back area")) return false;
  const uint32_t total = 2 * n - 1;
  // TT_BUILD_VERBOSE=1 prints the phase times and the iteration count to stderr.
  const bool verbose = std::getenv("TT_BUILD_VERBOSE") != nullptr;
  const auto t_start = std::chrono::steady_clock::now();
  auto ms_since = [&](std::chrono::steady_clock::time_point t0) {
    cudaStreamSynchronize(st);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  Aabb* prim_boxes = sc.alloc<Aabb>(n);
  unsigned* cbounds = sc.alloc<unsigned>(6);
  uint64_t* keys = sc.alloc<uint64_t>(n);
  uint64_t* keys2 = sc.alloc<uint64_t>(n);
  uint32_t* vals = sc.alloc<uint32_t>(n);
  uint32_t* perm = sc.alloc<uint32_t>(n);
  Aabb* node_box = sc.alloc<Aabb>(total);
  int* left = sc.alloc<int>(total);
  int* right = sc.alloc<int>(total);
  int* clusters = sc.alloc<int>(n);
  int* clusters2 = sc.alloc<int>(n);
  int* nn = sc.alloc<int>(n);
  int* create = sc.alloc<int>(n);
  int* create_off = sc.alloc<int>(n);
  int* keep = sc.alloc<int>(n);
  int* keep_off = sc.alloc<int>(n);
  if (!prim_boxes || !cbounds || !keys || !keys2 || !vals || !perm || !node_box || !left || !right || !clusters ||
      !clusters2 || !nn || !create || !create_off || !keep || !keep_off)
    return fail("out of device memory");
  const unsigned init_bounds[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  if (!ok(cudaMemcpyAsync(cbounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, st), "copy")) return false;
  k_prim_boxes<<<grid_for(n), kThreads, 0, st>>>(in, set, n, prim_boxes, cbounds);
  k_morton<<<grid_for(n), kThreads, 0, st>>>(prim_boxes, n, cbounds, keys, vals);
  // Sort primitives by Morton code (CUB radix sort).
  size_t sort_bytes = 0, scan_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys2, vals, perm, (int)n, 0, 63, st);
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, create, create_off, (int)n, st);
  void* temp = sc.alloc<unsigned char>(std::max(sort_bytes, scan_bytes));
  if (!temp) return fail("out of device memory");
  if (!ok(cub::DeviceRadixSort::SortPairs(temp, sort_bytes, keys, keys2, vals, perm, (int)n, 0, 63, st), "sort"))
    return false;
  k_init_leaves<<<grid_for(n), kThreads, 0, st>>>(prim_boxes, perm, n, node_box, left, right, clusters);
  const double t_sorted = verbose ? ms_since(t_start) : 0.0;
  // Clustering iterations; ranges[] records the node ids each iteration created.
  std::vector<std::pair<int, int>> ranges;
  int c = (int)n, next_node = (int)n;
  int* cur = clusters;
  int* nxt = clusters2;
  int iterations = 0;
  const char* radius_env = std::getenv("TT_PLOC_RADIUS");
  const int radius = radius_env ? std::max(1, std::min(256, std::atoi(radius_env))) : kDefaultRadius;
  while (c > 1) {
    if (++iterations > kMaxIterations) return fail("clustering did not converge");
    k_nearest<<<grid_for(c), kThreads, 0, st>>>(cur, c, node_box, radius, nn);
    k_merge_flags<<<grid_for(c), kThreads, 0, st>>>(nn, c, create, keep);
    size_t tb = std::max(sort_bytes, scan_bytes);
    cub::DeviceScan::ExclusiveSum(temp, tb, create, create_off, c, st);
    tb = std::max(sort_bytes, scan_bytes);
    cub::DeviceScan::ExclusiveSum(temp, tb, keep, keep_off, c, st);
    int* tail = hb;
    cudaMemcpyAsync(&tail[0], create_off + c - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&tail[1], create + c - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&tail[2], keep_off + c - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&tail[3], keep + c - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    k_merge<<<grid_for(c), kThreads, 0, st>>>(cur, c, nn, create, create_off, keep, keep_off, next_node, node_box, left,
                                             right, nxt);
    if (!ok(cudaStreamSynchronize(st), "clustering")) return false;
    const int made = tail[0] + tail[1], kept = tail[2] + tail[3];
    if (made <= 0 || next_node + made > (int)total) return fail("clustering made no progress");
    ranges.push_back({next_node, made});
    next_node += made;
    c = kept;
    std::swap(cur, nxt);
  }
  const double t_clustered = verbose ? ms_since(t_start) : 0.0;
  if (!ok(cudaMemcpyAsync(&hb[4], cur, sizeof(int), cudaMemcpyDeviceToHost, st), "copy") ||
      !ok(cudaStreamSynchronize(st), "sync"))
    return false;
  const int root = hb[4];
  // Bottom-up costs, top-down offsets and emission.
  int* size = sc.alloc<int>(total);
  float* cost = sc.alloc<float>(total);
  unsigned char* collapse = sc.alloc<unsigned char>(total);
  int* offset = sc.alloc<int>(total);
  unsigned char* state = sc.alloc<unsigned char>(total);
  int* depth = sc.alloc<int>(total);
  unsigned char* emit = sc.alloc<unsigned char>(total);
  int* inner = sc.alloc<int>(total);
  int* index = sc.alloc<int>(total);
  unsigned* max_depth = sc.alloc<unsigned>(1);
  if (!size || !cost || !collapse || !offset || !state || !depth || !emit || !inner || !index || !max_depth)
    return fail("out of device memory");
  cudaMemsetAsync(collapse, 1, n, st);  // primitive leaves
  cudaMemsetAsync(emit, 0, total, st);
  cudaMemsetAsync(max_depth, 0, sizeof(unsigned), st);
  for (const auto& r : ranges)
    k_costs<<<grid_for(r.second), kThreads, 0, st>>>(r.first, r.second, n, node_box, left, right, size, cost, collapse,
                                                      inner);
  cudaMemsetAsync(offset + root, 0, sizeof(int), st);
  cudaMemsetAsync(index + root, 0, sizeof(int), st);
  cudaMemsetAsync(state + root, 0, 1, st);  // no state
  cudaMemsetAsync(depth + root, 0, sizeof(int), st);
  for (auto it = ranges.rbegin(); it != ranges.rend(); ++it)
    k_topdown<<<grid_for(it->second), kThreads, 0, st>>>(it->first, it->second, n, left, right, size, collapse, inner,
                                                          offset, index, state, depth, emit, max_depth);
  hb[5] = 0;
  hb[6] = 0;
  hb[7] = 0;
  if (root >= (int)n) cudaMemcpyAsync(&hb[5], inner + root, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&hb[6], max_depth, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&hb[7], emit + root, 1, cudaMemcpyDeviceToHost, st);
  if (!ok(cudaStreamSynchronize(st), "emission")) return false;
  const int emitted = hb[5];
  const unsigned depth_host = (unsigned)hb[6];
  const unsigned char root_emit = (unsigned char)(hb[7] & 0xff);
  const int num_nodes = root_emit ? emitted : 1;
  // The 4-wide nodes are at most the emitted binary nodes (each 4-wide node replaces at
  // least one); the actual count comes from the collapse.
  const int cap4 = root_emit ? std::max(1, emitted) : 1;
  if (!ok(pool_malloc((void**)&out->nodes, 4 * sizeof(float4) * (size_t)num_nodes, st), "allocation") ||
      !ok(pool_malloc((void**)&out->tris, 3 * sizeof(float4) * (size_t)n, st), "allocation") ||
      !ok(pool_malloc((void**)&out->nodes4, 8 * sizeof(float4) * (size_t)cap4, st), "allocation"))
    return false;
  int num4 = 1;
  // The root is a leaf when the whole tree collapses (or n == 1): its subtree starts at 0.
  if (!root_emit) {
    cudaMemsetAsync(offset + root, 0, sizeof(int), st);
    k_leaf_root<<<1, 1, 0, st>>>(node_box, root, (int)n, out->nodes);
    k_leaf_root4<<<1, 1, 0, st>>>(node_box, root, (int)n, out->nodes4);
  } else {
    for (const auto& r : ranges)
      k_write_nodes<<<grid_for(r.second), kThreads, 0, st>>>(r.first, r.second, n, node_box, left, right, size, offset,
                                                              emit, index, out->nodes);
    int2* front[2] = {sc.alloc<int2>(cap4), sc.alloc<int2>(cap4)};
    int* counts = sc.alloc<int>(2);  // [0] 4-wide nodes numbered, [1] next level's size
    if (!front[0] || !front[1] || !counts) return fail("out of device memory");
    hb[8] = root;  // the first front: (root, 0); counts: {1, 0}
    hb[9] = 0;
    hb[10] = 1;
    hb[11] = 0;
    cudaMemcpyAsync(front[0], &hb[8], sizeof(int2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(counts, &hb[10], 2 * sizeof(int), cudaMemcpyHostToDevice, st);
    int nfront = 1;
    for (int level = 0; nfront > 0 && level < 64; ++level) {
      cudaMemsetAsync(counts + 1, 0, sizeof(int), st);
      k_collapse4<<<grid_for(nfront), kThreads, 0, st>>>(front[level & 1], nfront, n, node_box, left, right, size,
                                                          offset, emit, index, counts, front[(level + 1) & 1],
                                                          counts + 1, out->nodes4);
      int* c2 = &hb[12];
      cudaMemcpyAsync(c2, counts, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
      if (!ok(cudaStreamSynchronize(st), "4-wide collapse")) return false;
      nfront = c2[1];
      num4 = c2[0];
    }
    if (nfront > 0) return fail("4-wide collapse deeper than 64 levels");
    // Keep the nodes in a buffer of their exact size (the collapse wrote into an upper bound).
    float4* exact = nullptr;
    if (!ok(pool_malloc((void**)&exact, 8 * sizeof(float4) * (size_t)num4, st), "allocation")) return false;
    cudaMemcpyAsync(exact, out->nodes4, 8 * sizeof(float4) * (size_t)num4, cudaMemcpyDeviceToDevice, st);
    pool_free(out->nodes4, st);
    out->nodes4 = exact;
  }
  k_write_slots<<<grid_for(n), kThreads, 0, st>>>(in, set, left, offset, n, out->tris);
  if (!ok(cudaStreamSynchronize(st), "emission") || !ok(cudaGetLastError(), "kernels")) return false;
  out->num_nodes = (uint32_t)num_nodes;
  out->num_nodes4 = (uint32_t)num4;
  out->max_depth = root_emit ? depth_host : 0;
  if (verbose) {
    float root_cost = 0.f;
    if (root >= (int)n) cudaMemcpy(&root_cost, cost + root, sizeof(float), cudaMemcpyDeviceToHost);
    std::fprintf(stderr,
                 "device BVH build: %u prims, %d iterations, %d nodes, depth %u, SAH cost %.2f; sorted %.1f ms, "
                 "clustered %.1f ms, done %.1f ms\n",
                 n, iterations, num_nodes, out->max_depth, root_cost, t_sorted, t_clustered, ms_since(t_start));
  }
  return true;
}

}  // namespace tt
