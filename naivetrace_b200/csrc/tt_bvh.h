// Host SAH BVH builder producing the device layout of the closest-hit / occlusion kernels.
//
// Replaces the Embree scene commit (EmbreeAccelerator::Build, embreeaccelerator.cxx:31-35;
// Scene::BuildAccelStructure, scene.cxx:116-141).
//
// Device layout, binary BVH with both child boxes stored in the parent (64 bytes/node):
//   float4 n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   float4 n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   float4 n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   int4   n3 = (c0 ref, c1 ref, 0, 0)
// A child ref >= 0 is an inner node index; a ref < 0 is a leaf: v = ~ref,
// first triangle slot = v >> 3, triangle count = (v & 7) + 1.  An empty child has an
// inverted box and refers to slot 0; an empty triangle set gets one degenerate slot.
// Spheres share the slot array: (centre.xyz | prim id, radius, 0, 0 | material id,
// 0, 0, 0 | 1); a triangle slot has 0 in the last word, a sphere slot the integer 1.  Triangles are stored per leaf slot as three float4
// (v0.xyz | prim id, v1.xyz | material id, v2.xyz | 0).
#pragma once

#include <cstdint>
#include <vector>

namespace tt {

struct BvhInput {
  const float* vertices;        // V x 3
  const uint32_t* indices;      // T x 3
  const uint32_t* material_ids; // T
  uint32_t num_triangles;
  const uint32_t* prim_ids = nullptr;  // T ids stored in the slots (nullptr: 0 .. T-1)
  uint32_t num_spheres = 0;
  const float* spheres = nullptr;              // S x 4: centre, radius
  const uint32_t* sphere_material_ids = nullptr;
  const uint32_t* sphere_prim_ids = nullptr;   // S ids stored in the slots
};

struct BvhOutput {
  std::vector<float> nodes;     // 16 floats per node
  std::vector<float> tris;      // 12 floats per triangle slot
  uint32_t num_nodes = 0;
  uint32_t max_depth = 0;
  double sah_cost = 0;
};

// max_leaf <= 8.  Returns false on invalid input.
bool build_bvh(const BvhInput& in, int max_leaf, BvhOutput* out);

}  // namespace tt
