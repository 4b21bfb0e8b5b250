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

// Primitive p < T is triangle p, p >= T is sphere p - T.  Builds the binary SAH tree.
static bool build_tree(const BvhInput& in, int max_leaf, Builder& b, std::vector<BuildNode>& nodes,
                       uint32_t* depth) {
  if (max_leaf < 1 || max_leaf > 8) return false;
  if (in.num_spheres > 0 && (!in.spheres || !in.sphere_material_ids || !in.sphere_prim_ids)) return false;
  const uint32_t T = in.num_triangles;
  const uint32_t n = T + in.num_spheres;
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
  nodes.reserve(2 * (size_t)std::max<uint32_t>(n, 1) / 2 + 16);
  *depth = 0;
  if (n > 0) b.build(nodes, 0, (int)n, 0, depth);
  return true;
}

// Writes primitive t's 48-byte slot (layout in tt_bvh.h).
static void write_slot(const BvhInput& in, int t, float* dst) {
  const uint32_t T = in.num_triangles;
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
    return;
  }
  for (int j = 0; j < 3; ++j) {
    const float* v = &in.vertices[3 * (size_t)in.indices[3 * (size_t)t + j]];
    dst[4 * j] = v[0];
    dst[4 * j + 1] = v[1];
    dst[4 * j + 2] = v[2];
  }
  const int32_t prim = in.prim_ids ? (int32_t)in.prim_ids[t] : t, mat = (int32_t)in.material_ids[t];
  std::memcpy(&dst[3], &prim, 4);
  std::memcpy(&dst[7], &mat, 4);
}

bool build_bvh(const BvhInput& in, int max_leaf, BvhOutput* out) {
  if (!out) return false;
  Builder b;
  std::vector<BuildNode> nodes;
  uint32_t depth = 0;
  if (!build_tree(in, max_leaf, b, nodes, &depth)) return false;
  const uint32_t n = in.num_triangles + in.num_spheres;
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
  for (uint32_t i = 0; i < n; ++i) write_slot(in, b.order[i], &out->tris[12 * (size_t)i]);

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

namespace {

// Octant-ordered slots: slot s holds the child nearest the corner with + sides on the axes
// whose bit is set in s, so that visiting permuted positions (slot ^ ray octant) in
// increasing order approximates near-to-far for the ray.  Greedy assignment by the
// largest projection of the child centroid offset onto the corner direction.
void assign_slots(const std::vector<Box>& boxes, const Box& parent, int slot_of[8]) {
  const int k = (int)boxes.size();
  float pc[3];
  for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (parent.lo[a] + parent.hi[a]);
  float score[8][8];
  for (int c = 0; c < k; ++c)
    for (int sl = 0; sl < 8; ++sl) {
      float v = 0.f;
      for (int a = 0; a < 3; ++a) {
        const float off = 0.5f * (boxes[c].lo[a] + boxes[c].hi[a]) - pc[a];
        v += ((sl >> a) & 1) ? off : -off;
      }
      score[c][sl] = v;
    }
  bool used_c[8] = {false}, used_s[8] = {false};
  for (int round = 0; round < k; ++round) {
    int bc = -1, bs = -1;
    float best = -std::numeric_limits<float>::infinity();
    for (int c = 0; c < k; ++c) {
      if (used_c[c]) continue;
      for (int sl = 0; sl < 8; ++sl)
        if (!used_s[sl] && score[c][sl] > best) { best = score[c][sl]; bc = c; bs = sl; }
    }
    if (bc < 0) {  // scores may be NaN for degenerate boxes: take the first free pair
      for (int c = 0; c < k && bc < 0; ++c)
        if (!used_c[c]) bc = c;
      for (int sl = 0; sl < 8 && bs < 0; ++sl)
        if (!used_s[sl]) bs = sl;
    }
    used_c[bc] = used_s[bs] = true;
    slot_of[bc] = bs;
  }
}

// Smallest e with 255 * 2^e >= extent, clamped so that 2^e is a normal float.
int quant_exponent(float extent) {
  if (!(extent > 0.f)) return -126;
  int e = (int)std::ceil(std::log2((double)extent / 255.0));
  while (std::ldexp(255.0, e) < (double)extent) ++e;
  while (e > -126 && std::ldexp(255.0, e - 1) >= (double)extent) --e;
  return std::min(std::max(e, -126), 127);
}

}  // namespace

bool build_bvh8(const BvhInput& in, Bvh8Output* out) {
  if (!out) return false;
  Builder b;
  std::vector<BuildNode> nodes;
  uint32_t depth2 = 0;
  if (!build_tree(in, 3, b, nodes, &depth2)) return false;
  const uint32_t n = in.num_triangles + in.num_spheres;
  out->nodes.clear();
  out->tris.clear();
  out->max_depth = 0;
  if (n == 0) {
    // Root without children; one degenerate triangle slot (prim id -1) keeps reads in bounds.
    out->nodes.assign(20, 0u);
    out->tris.assign(12, 0.f);
    const int32_t none = -1;
    std::memcpy(&out->tris[3], &none, 4);
    out->num_nodes = 1;
    return true;
  }
  struct Item {
    int bnode;  // binary build node whose subtree this wide node covers
    int depth;
  };
  std::vector<Item> queue;
  queue.push_back({0, 0});
  out->nodes.assign(20, 0u);  // node 0 reserved for the root
  for (size_t qi = 0; qi < queue.size(); ++qi) {
    const Item it = queue[qi];
    out->max_depth = std::max(out->max_depth, (uint32_t)it.depth);
    // Collapse: open the largest inner child until eight children or only leaves remain.
    std::vector<int> kids;
    if (nodes[it.bnode].left >= 0) kids = {nodes[it.bnode].left, nodes[it.bnode].right};
    else kids = {it.bnode};
    while (kids.size() < 8) {
      int pick = -1;
      float area = -1.f;
      for (size_t i = 0; i < kids.size(); ++i)
        if (nodes[kids[i]].left >= 0 && nodes[kids[i]].box.half_area() > area) {
          area = nodes[kids[i]].box.half_area();
          pick = (int)i;
        }
      if (pick < 0) break;
      const int nd = kids[pick];
      kids[pick] = nodes[nd].left;
      kids.push_back(nodes[nd].right);
    }
    std::vector<Box> boxes;
    Box nb;
    nb.reset();
    for (int k : kids) {
      boxes.push_back(nodes[k].box);
      nb.grow(nodes[k].box);
    }
    int slot_of[8];
    assign_slots(boxes, nb, slot_of);
    int kid_at[8];
    for (int sl = 0; sl < 8; ++sl) kid_at[sl] = -1;
    for (size_t i = 0; i < kids.size(); ++i) kid_at[slot_of[i]] = kids[i];
    // Node words (layout in tt_bvh.h).
    uint32_t w[20] = {0};
    int e[3];
    for (int a = 0; a < 3; ++a) {
      std::memcpy(&w[a], &nb.lo[a], 4);
      e[a] = quant_exponent(nb.hi[a] - nb.lo[a]);
    }
    uint32_t imask = 0;
    const uint32_t child_base = (uint32_t)(out->nodes.size() / 20);
    const uint32_t tri_base = (uint32_t)(out->tris.size() / 12);
    uint32_t inner_rank = 0, tri_off = 0;
    uint8_t meta[8] = {0}, qlo[3][8], qhi[3][8];
    for (int sl = 0; sl < 8; ++sl)
      for (int a = 0; a < 3; ++a) { qlo[a][sl] = 255; qhi[a][sl] = 0; }
    std::vector<std::pair<int, uint32_t>> new_children;
    for (int sl = 0; sl < 8; ++sl) {
      const int k = kid_at[sl];
      if (k < 0) continue;
      const BuildNode& c = nodes[k];
      for (int a = 0; a < 3; ++a) {
        const double scale = std::ldexp(1.0, e[a]);
        const double lo = std::floor(((double)c.box.lo[a] - nb.lo[a]) / scale);
        const double hi = std::ceil(((double)c.box.hi[a] - nb.lo[a]) / scale);
        qlo[a][sl] = (uint8_t)std::min(255.0, std::max(0.0, lo));
        qhi[a][sl] = (uint8_t)std::min(255.0, std::max(0.0, hi));
      }
      if (c.left >= 0) {
        imask |= 1u << sl;
        new_children.push_back({k, child_base + inner_rank});
        ++inner_rank;
      } else {
        meta[sl] = (uint8_t)((tri_off << 2) | (uint32_t)c.count);
        for (int i = 0; i < c.count; ++i) {
          out->tris.resize(out->tris.size() + 12, 0.f);
          write_slot(in, b.order[c.start + i], &out->tris[out->tris.size() - 12]);
        }
        tri_off += (uint32_t)c.count;
      }
    }
    w[3] = (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) | (imask << 24);
    w[4] = child_base;
    w[5] = tri_base;
    std::memcpy(&w[6], meta, 8);
    for (int a = 0; a < 3; ++a) {
      std::memcpy(&w[8 + 2 * a], qlo[a], 8);
      std::memcpy(&w[14 + 2 * a], qhi[a], 8);
    }
    // Breadth-first allocation: queue item qi is node qi, and its inner children take the
    // next indices in slot order.
    std::memcpy(&out->nodes[20 * qi], w, sizeof(w));
    out->nodes.resize(out->nodes.size() + 20 * new_children.size(), 0u);
    for (auto& ch : new_children) queue.push_back({ch.first, it.depth + 1});
  }
  out->num_nodes = (uint32_t)(out->nodes.size() / 20);
  if (out->tris.empty()) {
    out->tris.assign(12, 0.f);
    const int32_t none = -1;
    std::memcpy(&out->tris[3], &none, 4);
  }
  return true;
}

}  // namespace tt
