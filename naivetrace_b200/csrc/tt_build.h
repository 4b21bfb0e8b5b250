// Device BVH construction (tt_build.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tt {

// Device pointers to the whole scene's primitives; a build covers the subset `set` of
// global primitive ids (triangles 0..T-1, spheres T..T+S-1) and stores prim_ids[i] as the
// id of set position i.
struct BuildInput {
  const float* vertices;              // V x 3
  const uint32_t* indices;            // T x 3
  const uint32_t* material_ids;       // T
  uint32_t num_triangles;
  const float* spheres;               // S x 4
  const uint32_t* sphere_material_ids;
  const uint32_t* prim_ids;           // per set position: the id written into the slot
};

struct DeviceBvh {
  float4* nodes;        // binary layout of tt_bvh.h, from the memory pool (caller frees)
  float4* tris;         // primitive slots, from the memory pool (caller frees)
  uint32_t num_nodes;
  uint32_t max_depth;
  // The same tree with up to four children per node (a binary node's children, the inner
  // child of the largest surface area replaced by its children until there are four; 8
  // float4: lo.x[4], hi.x[4], lo.y[4], hi.y[4], lo.z[4], hi.z[4], int4 references (inner
  // node, leaf reference as in the binary layout, or 0x7fffffff for an empty slot with an
  // empty box), padding; the root is node 0), from the memory pool.
  float4* nodes4;
  uint32_t num_nodes4;
};

// Builds the binary BVH of the `n` primitives whose global ids are in `set` (device array).
// Synchronises `st`.  Returns false with a message on failure.
bool device_build_bvh2(const BuildInput& in, const uint32_t* set, uint32_t n, DeviceBvh* out, cudaStream_t st,
                       std::string* err);

}  // namespace tt
