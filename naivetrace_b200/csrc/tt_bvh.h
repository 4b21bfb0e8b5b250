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

// 8-wide BVH with quantised child boxes (80 bytes per node), collapsed from the binary SAH
// tree (leaves of at most 3 primitives).  Node words:
//   0-2  origin p (float x, y, z) = lower corner of the node box
//   3    exponents e_x, e_y, e_z (biased by 127) and the inner-child mask (bits 24-31)
//   4    index of the first inner child node (inner children are consecutive, slot order)
//   5    first primitive slot of the node's leaf children (consecutive, slot order)
//   6-7  meta byte per child slot: leaf = (slot offset from word 5) << 2 | count (1..3),
//        0 for inner and empty slots
//   8-13 quantised lower bounds per axis (x: 8-9, y: 10-11, z: 12-13), one byte per slot
//   14-19 quantised upper bounds (x: 14-15, y: 16-17, z: 18-19)
// Child box = p + q * 2^e per axis, containing the child's exact box.  Slot s holds the
// child nearest the box corner whose axes with bit set in s are on the + side, so that
// visiting slot ^ octant(ray) in increasing order approximates near-to-far.  Primitive
// slots as in the binary layout.
struct Bvh8Output {
  std::vector<uint32_t> nodes;  // 20 words per node
  std::vector<float> tris;      // 12 floats per primitive slot
  uint32_t num_nodes = 0;
  uint32_t max_depth = 0;
};
bool build_bvh8(const BvhInput& in, Bvh8Output* out);

}  // namespace tt
