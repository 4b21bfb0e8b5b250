// Binned-SAH BVH build on the host, emitted in the device layout described in tt_bvh.h.
#include "tt_bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>

namespace tt {
namespace {

struct Box {
  float lo[3], hi[3];
  void reset() {
    for (int k = 0; k < 3; ++k) { lo[k] = std::numeric_limits<float>::infinity(); hi[k] = -lo[k]; }
  }
  void grow(const Box& b) {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
  }
  void grow(const float* p) {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
  }
  float half_area() const {
    float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
    if (!(d0 >= 0.f) || !(d1 >= 0.f) || !(d2 >= 0.f)) return 0.f;
    return d0 * d1 + d1 * d2 + d2 * d0;
  }
};

struct BuildNode {
  Box box;
  int left = -1, right = -1;  // children (build-node indices), -1 for leaves
  int start = 0, count = 0;
};

constexpr int kBins = 32;
constexpr int kParallelThreshold = 1 << 17;

struct Builder {
  std::vector<Box> tri_box;
  std::vector<float> cen;     // 3 per triangle
  std::vector<int> order;
  int max_leaf;

  // Builds the subtree of order[start, start+count) into `nodes` (local pool), returns
  // the local index of its root.
  int build(std::vector<BuildNode>& nodes, int start, int count, int depth, uint32_t* max_depth) {
    const int me = (int)nodes.size();
    nodes.push_back(BuildNode{});
    Box bb, cb;
    bb.reset();
    cb.reset();
    for (int i = start; i < start + count; ++i) {
      const int t = order[i];
      bb.grow(tri_box[t]);
      cb.grow(&cen[3 * (size_t)t]);
    }
    nodes[me].box = bb;
    *max_depth = std::max(*max_depth, (uint32_t)depth);
    auto make_leaf = [&]() {
      nodes[me].start = start;
      nodes[me].count = count;
    };
    if (count <= 2) { make_leaf(); return me; }
    // Binned SAH over the three axes.
    int best_axis = -1, best_split = -1;
    float best_cost = std::numeric_limits<float>::infinity();
    for (int axis = 0; axis < 3; ++axis) {
      const float ext = cb.hi[axis] - cb.lo[axis];
      if (!(ext > 0.f)) continue;
      const float scale = kBins / ext;
      Box bins[kBins];
      int cnt[kBins] = {0};
      for (auto& b : bins) b.reset();
      for (int i = start; i < start + count; ++i) {
        const int t = order[i];
        int b = (int)((cen[3 * (size_t)t + axis] - cb.lo[axis]) * scale);
        b = std::min(std::max(b, 0), kBins - 1);
        cnt[b]++;
        bins[b].grow(tri_box[t]);
      }
      float right_area[kBins];
      int right_cnt[kBins];
      Box acc;
      acc.reset();
      int c = 0;
      for (int b = kBins - 1; b > 0; --b) {
        acc.grow(bins[b]);
        c += cnt[b];
        right_area[b] = acc.half_area();
        right_cnt[b] = c;
      }
      acc.reset();
      c = 0;
      for (int b = 0; b < kBins - 1; ++b) {
        acc.grow(bins[b]);
        c += cnt[b];
        if (c == 0 || right_cnt[b + 1] == 0) continue;
        const float cost = c * acc.half_area() + right_cnt[b + 1] * right_area[b + 1];
        if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = b; }
      }
    }
    const float parent_area = bb.half_area();
    const float leaf_cost = (float)count;
    const float split_cost = parent_area > 0.f ? 1.0f + best_cost / parent_area : std::numeric_limits<float>::infinity();
    if (count <= max_leaf && (best_axis < 0 || leaf_cost <= split_cost)) { make_leaf(); return me; }
    int mid;
    if (best_axis < 0) {
      mid = start + count / 2;  // coincident centroids: split by count
    } else {
      const float scale = kBins / (cb.hi[best_axis] - cb.lo[best_axis]);
      const float lo = cb.lo[best_axis];
      auto it = std::partition(order.begin() + start, order.begin() + start + count, [&](int t) {
        int b = (int)((cen[3 * (size_t)t + best_axis] - lo) * scale);
        b = std::min(std::max(b, 0), kBins - 1);
        return b <= best_split;
      });
      mid = (int)(it - order.begin());
      if (mid == start || mid == start + count) mid = start + count / 2;
    }
    const int lcount = mid - start, rcount = start + count - mid;
    if (count >= kParallelThreshold) {
      // Build the right subtree in a separate pool on another thread, then splice.
      std::vector<BuildNode> rpool;
      uint32_t rdepth = 0;
      auto fut = std::async(std::launch::async, [&]() { return build(rpool, mid, rcount, depth + 1, &rdepth); });
      const int l = build(nodes, start, lcount, depth + 1, max_depth);
      fut.get();
      const int offset = (int)nodes.size();
      for (auto n : rpool) {
        if (n.left >= 0) { n.left += offset; n.right += offset; }
        nodes.push_back(n);
      }
      *max_depth = std::max(*max_depth, rdepth);
      nodes[me].left = l;
      nodes[me].right = offset;  // the right root is the first node of its pool
    } else {
      const int l = build(nodes, start, lcount, depth + 1, max_depth);
      const int r = build(nodes, mid, rcount, depth + 1, max_depth);
      nodes[me].left = l;
      nodes[me].right = r;
    }
    return me;
  }
};

}  // namespace

bool build_bvh(const BvhInput& in, int max_leaf, BvhOutput* out) {
  if (max_leaf < 1 || max_leaf > 8 || !out) return false;
  if (in.num_spheres > 0 && (!in.spheres || !in.sphere_material_ids || !in.sphere_prim_ids)) return false;
  // Primitive p < T is triangle p, p >= T is sphere p - T.
  const uint32_t T = in.num_triangles;
  const uint32_t n = T + in.num_spheres;
  Builder b;
  b.max_leaf = max_leaf;
  b.tri_box.resize(n);
  b.cen.resize(3 * (size_t)n);
  b.order.resize(n);
  for (uint32_t t = 0; t < n; ++t) {
    Box bx;
    bx.reset();
    if (t < T) {
      for (int j = 0; j < 3; ++j) bx.grow(&in.vertices[3 * (size_t)in.indices[3 * (size_t)t + j]]);
    } else {
      // Bounds one ulp outside centre -/+ radius (SphereBoundsFunc, embreeaccelerator.cxx:263-281).
      const float* q = &in.spheres[4 * (size_t)(t - T)];
      for (int k = 0; k < 3; ++k) {
        bx.lo[k] = std::nextafter(q[k] - q[3], -std::numeric_limits<float>::infinity());
        bx.hi[k] = std::nextafter(q[k] + q[3], std::numeric_limits<float>::infinity());
      }
    }
    b.tri_box[t] = bx;
    for (int k = 0; k < 3; ++k) b.cen[3 * (size_t)t + k] = 0.5f * (bx.lo[k] + bx.hi[k]);
    b.order[t] = (int)t;
  }
  std::vector<BuildNode> nodes;
  nodes.reserve(2 * (size_t)std::max<uint32_t>(n, 1) / 2 + 16);
  uint32_t depth = 0;
  if (n > 0) b.build(nodes, 0, (int)n, 0, &depth);
  out->max_depth = depth;

  // Triangle slots in leaf order.  An empty set still gets one slot: a degenerate triangle
  // at the origin (prim id -1) that no ray can hit, so that the synthetic root's leaf
  // reference to slot 0 stays in bounds.  (An empty child box is stored inverted, which
  // the slab test does not reject, so traversal may visit slot 0 through it.)
  out->tris.assign(12 * (size_t)std::max<uint32_t>(n, 1), 0.f);
  if (n == 0) {
    const int32_t none = -1;
    std::memcpy(&out->tris[3], &none, 4);
  }
  for (uint32_t i = 0; i < n; ++i) {
    const int t = b.order[i];
    float* dst = &out->tris[12 * (size_t)i];
    if ((uint32_t)t >= T) {
      const uint32_t k = (uint32_t)t - T;
      const float* q = &in.spheres[4 * (size_t)k];
      dst[0] = q[0];
      dst[1] = q[1];
      dst[2] = q[2];
      dst[4] = q[3];
      const int32_t prim = (int32_t)in.sphere_prim_ids[k], mat = (int32_t)in.sphere_material_ids[k], tag = 1;
      std::memcpy(&dst[3], &prim, 4);
      std::memcpy(&dst[7], &mat, 4);
      std::memcpy(&dst[11], &tag, 4);
      continue;
    }
    for (int j = 0; j < 3; ++j) {
      const float* v = &in.vertices[3 * (size_t)in.indices[3 * (size_t)t + j]];
      dst[4 * j] = v[0];
      dst[4 * j + 1] = v[1];
      dst[4 * j + 2] = v[2];
    }
    int32_t prim = in.prim_ids ? (int32_t)in.prim_ids[t] : t, mat = (int32_t)in.material_ids[t];
    std::memcpy(&dst[3], &prim, 4);
    std::memcpy(&dst[7], &mat, 4);
  }

  // Device nodes: one per inner build node; a leaf-only tree gets a synthetic root.
  std::vector<int> dev_index(nodes.size(), -1);
  int num_inner = 0;
  for (size_t i = 0; i < nodes.size(); ++i)
    if (nodes[i].left >= 0) dev_index[i] = num_inner++;
  const bool synthetic_root = nodes.empty() || nodes[0].left < 0;
  const int total = synthetic_root ? 1 : num_inner;
  out->nodes.assign(16 * (size_t)total, 0.f);
  out->num_nodes = (uint32_t)total;
  auto child_ref = [&](int bi) -> int32_t {
    const BuildNode& c = nodes[bi];
    if (c.left >= 0) return dev_index[bi];
    const uint32_t v = ((uint32_t)c.start << 3) | (uint32_t)(c.count - 1);
    return ~(int32_t)v;
  };
  auto write = [&](int slot, const Box* b0, int32_t r0, const Box* b1, int32_t r1) {
    float* d = &out->nodes[16 * (size_t)slot];
    Box empty;
    empty.reset();
    const Box& a = b0 ? *b0 : empty;
    const Box& c = b1 ? *b1 : empty;
    d[0] = a.lo[0]; d[1] = a.hi[0]; d[2] = a.lo[1]; d[3] = a.hi[1];
    d[4] = c.lo[0]; d[5] = c.hi[0]; d[6] = c.lo[1]; d[7] = c.hi[1];
    d[8] = a.lo[2]; d[9] = a.hi[2]; d[10] = c.lo[2]; d[11] = c.hi[2];
    std::memcpy(&d[12], &r0, 4);
    std::memcpy(&d[13], &r1, 4);
    int32_t zero = 0;
    std::memcpy(&d[14], &zero, 4);
    std::memcpy(&d[15], &zero, 4);
  };
  if (synthetic_root) {
    if (nodes.empty()) {
      write(0, nullptr, ~(int32_t)0, nullptr, ~(int32_t)0);
    } else {
      write(0, &nodes[0].box, child_ref(0), nullptr, ~(int32_t)0);
    }
  } else {
    double sah = 0;
    const float root_area = std::max(nodes[0].box.half_area(), 1e-30f);
    for (size_t i = 0; i < nodes.size(); ++i) {
      const BuildNode& nd = nodes[i];
      if (nd.left >= 0) {
        write(dev_index[i], &nodes[nd.left].box, child_ref(nd.left), &nodes[nd.right].box, child_ref(nd.right));
        sah += 1.0 * nd.box.half_area() / root_area;
      } else {
        sah += (double)nd.count * nd.box.half_area() / root_area;
      }
    }
    out->sah_cost = sah;
  }
  return true;
}

}  // namespace tt
