// Wavefront kernels of the forward path tracer with next-event estimation.
//
// The per-sample loop of PathTracingWorker::RenderPixel
// (renderingalgorithms_pathtracing.hxx:731-817) is split into stages that each process a
// queue of path slots:
//   generate  - wavelength selection, next-event estimation at the camera vertex
//               (splatted to the pixel the light sample projects to), camera ray.
//   extend    - closest hit of the queued extension rays (BVH traversal).
//   shade     - MIS-weighted emission at the hit, Russian roulette, next-event estimation
//               (emits a shadow ray), BSDF sampling (emits the next extension ray).
//   shadow    - occlusion test; adds the NEE contribution of unoccluded rays.
//   guide     - (guided scenes) the network on the vertices shade queued for guiding, then
//               one-sample MIS of the BSDF and the learned mixture (emits the next ray).
//   flush     - converts finished paths to RGB and adds them to the framebuffer; commits
//               the path's training record when the guide is being trained.
// Queues are appended with warp-aggregated atomics.  All kernels loop grid-stride over a
// device-side count, so launch shapes are fixed (a multiple of the SM count).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <type_traits>

#include "tt_device.cuh"
#include "tt_guide.cuh"
#include "tt_guide_tc.cuh"
#include "tt_internal.h"
#include "tt_tables.h"

namespace tt {

// ----------------------------------------------------------------------------------------
__device__ __forceinline__ int warp_append(int* counter) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  const int rank = __popc(mask & ((1u << lane) - 1u));
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + rank;
}

// Per bounce: queue lengths of extension rays, shadow rays and finished paths.
__device__ __forceinline__ int* ext_count(const PathState& p, int b) { return &p.counters[kCountersPerBounce * b]; }
__device__ __forceinline__ int* sh_count(const PathState& p, int b) { return &p.counters[kCountersPerBounce * b + 1]; }
__device__ __forceinline__ int* done_count(const PathState& p, int b) { return &p.counters[kCountersPerBounce * b + 2]; }
__device__ __forceinline__ int* guide_count(const PathState& p, int b) { return &p.counters[kCountersPerBounce * b + 3]; }
__device__ __forceinline__ int* key_count(const PathState& p, int b) { return &p.counters[kCountersPerBounce * b + 4]; }
__device__ __forceinline__ int* key_cursor(const PathState& p, int b) {
  return &p.counters[kCountersPerBounce * b + 4 + kShadeKeys];
}

// Pending training record of a guided path (PathState::grec, 6 float4 per slot):
//   0: position normalised to the scene box (xyz), shading normal x
//   1: shading normal yz, outgoing direction xy
//   2: outgoing direction z, sampled direction xyz
//   3: BSDF pdf of the sampled direction, vertex depth (int bits), guided vertices seen on
//      the path (int bits), valid flag
//   4: path contribution before the vertex (spectral, 3)
//   5: throughput before the vertex (spectral, 3)
constexpr int kRecF4 = 6;


// ----------------------------------------------------------------------------------------
// BVH traversal (layout in tt_bvh.h) with the watertight ray/triangle test of Woop,
// Benthin and Wald (2013), replacing rtcIntersect1 / rtcOccluded1
// (embreeaccelerator.cxx:111, :302).  Hits count for tnear < t <= tfar.
struct RayPre {
  float3 o, d, id, ood;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

__device__ __forceinline__ float safe_inv(float x) {
  const float ax = fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x;
  return 1.f / ax;
}

__device__ __forceinline__ RayPre prepare_ray(float3 o, float3 d) {
  RayPre r;
  r.o = o;
  r.d = d;
  r.id = f3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
  r.ood = f3(o.x * r.id.x, o.y * r.id.y, o.z * r.id.z);
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = 0;
  if (ay > ax) kz = 1;
  if (az > fmaxf(ax, ay)) kz = 2;
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (comp(d, kz) < 0.f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx; r.ky = ky; r.kz = kz;
  const float dz = comp(d, kz);
  r.Sx = comp(d, kx) / dz;
  r.Sy = comp(d, ky) / dz;
  r.Sz = 1.f / dz;
  return r;
}

// Returns true with t and the barycentric weights (b1, b2) of v1 and v2.  Inside/outside
// is decided with the watertight sheared edge functions of Woop, Benthin and Wald (2013),
// so rays cannot slip through shared edges.  The hit distance comes from the plane
// equation, t = Ng.(v0 - o) / Ng.d: a ray starting on the triangle's plane gets t = 0
// exactly whenever the plane offset is exact (axis-aligned walls), so with tnear = 0 it
// cannot re-hit the surface it leaves even when the anti-self-intersection offset is 0.
__device__ __forceinline__ bool intersect_tri(const RayPre& r, float3 v0, float3 v1, float3 v2, float tnear,
                                              float tfar, float* tout, float* b1out, float* b2out) {
  const float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
  const float Az_ = comp(A, r.kz), Bz_ = comp(B, r.kz), Cz_ = comp(C, r.kz);
  const float Ax = comp(A, r.kx) - r.Sx * Az_, Ay = comp(A, r.ky) - r.Sy * Az_;
  const float Bx = comp(B, r.kx) - r.Sx * Bz_, By = comp(B, r.ky) - r.Sy * Bz_;
  const float Cx = comp(C, r.kx) - r.Sx * Cz_, Cy = comp(C, r.ky) - r.Sy * Cz_;
  // Rounded products without fused multiply-add: the edge function of an edge shared by
  // two triangles must come out as exact negatives in both for the test to be watertight.
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.f || V == 0.f || W == 0.f) {
    // Edge case: recompute the edge functions in double precision (Woop et al., sec. 4).
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  const float det = U + V + W;
  if (det == 0.f) return false;
  const float3 ng = cross3(v1 - v0, v2 - v0);
  const float den = dot3(ng, r.d);
  if (den == 0.f) return false;
  // Axis-aligned planes: the distance along that axis alone, so that coplanar faces of
  // any size yield bitwise-equal distances and the primitive-id tie rule applies.
  float t;
  if (ng.y == 0.f && ng.z == 0.f) t = A.x / r.d.x;
  else if (ng.x == 0.f && ng.z == 0.f) t = A.y / r.d.y;
  else if (ng.x == 0.f && ng.y == 0.f) t = A.z / r.d.z;
  else t = dot3(ng, A) / den;
  if (!(t > tnear && t <= tfar)) return false;
  const float inv = 1.f / det;
  *tout = t;
  *b1out = V * inv;
  *b2out = W * inv;
  return true;
}

// Ray/sphere test of a sphere slot (centre a.xyz, radius b.x) in double precision: the
// roots of t^2 |d|^2 + 2 t (v.d) + |v|^2 - r^2 = 0, v = o - centre, from the
// cancellation-free pair q = -(b + sign(b) sqrt(D)), t = q / a and c / q (PBRT's
// Quadratic, util.hxx:131-144).  The nearer root in (tnear, tfar] is the hit.  (The
// reference tests spheres in single precision with error bounds,
// embreeaccelerator.cxx:307-427; single precision loses planet-sized spheres near the
// ground.)
__device__ __forceinline__ bool intersect_sphere(const RayPre& r, float4 a, float4 b, float tnear, float tfar,
                                                 float* tout) {
  const double vx = (double)r.o.x - a.x, vy = (double)r.o.y - a.y, vz = (double)r.o.z - a.z;
  const double dx = r.d.x, dy = r.d.y, dz = r.d.z;
  const double A = dx * dx + dy * dy + dz * dz;
  const double B = vx * dx + vy * dy + vz * dz;
  const double C = vx * vx + vy * vy + vz * vz - (double)b.x * b.x;
  const double D = B * B - A * C;
  if (D < 0.0) return false;
  const double q = -(B + copysign(sqrt(D), B));
  double t0 = q / A, t1 = q != 0.0 ? C / q : 0.0;
  if (t0 > t1) { const double x = t0; t0 = t1; t1 = x; }
  float t = (float)t0;
  if (!(t > tnear && t <= tfar)) {
    t = (float)t1;
    if (!(t > tnear && t <= tfar)) return false;
  }
  *tout = t;
  return true;
}

struct TraceCounters {
  unsigned int nodes;
  unsigned int tris;
};

// Traversal state of one ray.  A step processes one inner node (both child boxes) or one
// leaf.
struct TraceState {
  RayPre r;
  float tnear, best_t, b1, b2;
  int best, best_prim, cur, sp;
};

// Closest-hit acceptance for a candidate at t <= best_t: nearer, or at the same distance
// with a lower primitive id.  Coplanar overlapping faces (a box standing on the floor) then
// resolve the same way whatever the traversal order or tree shape.
__device__ __forceinline__ bool closer(float t, int prim, float best_t, int best_prim) {
  return t < best_t || prim < best_prim;
}

__device__ __forceinline__ void trace_init(TraceState& s, float3 o, float3 d, float tnear, float tfar) {
  s.r = prepare_ray(o, d);
  s.tnear = tnear;
  s.best_t = tfar;
  s.b1 = s.b2 = 0.f;
  s.best = -1;
  s.best_prim = 0x7fffffff;
  s.cur = 0;  // the root is always an inner node
  s.sp = 0;
}

// One traversal step.  Returns true when the ray is finished (closest hit found, or for
// ANY the first hit), with the result in s.best / best_t / b1 / b2.
// A BVH in device layout: the surface BVH or the medium-boundary BVH.
struct BvhRef {
  const float4* nodes;
  const float4* tris;
};
__device__ __forceinline__ BvhRef surface_bvh(const DevScene& sc) { return BvhRef{sc.nodes, sc.tris}; }
__device__ __forceinline__ BvhRef volume_bvh(const DevScene& sc) { return BvhRef{sc.vnodes, sc.vtris}; }

template <bool ANY, bool COUNT, bool SPH>
__device__ __forceinline__ bool trace_step(const BvhRef& bvh, TraceState& s, int* stack, unsigned int* err,
                                           TraceCounters* cnt) {
  const RayPre& r = s.r;
  if (s.cur >= 0) {
    const float4* np = bvh.nodes + 4 * (size_t)s.cur;
    const float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
    const int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
    if (COUNT) cnt->nodes++;
    const float lim = s.best_t * 1.0000004f;  // 1 + 2 gamma(3): conservative slabs
    float tx0 = fmaf(n0.x, r.id.x, -r.ood.x), tx1 = fmaf(n0.y, r.id.x, -r.ood.x);
    float ty0 = fmaf(n0.z, r.id.y, -r.ood.y), ty1 = fmaf(n0.w, r.id.y, -r.ood.y);
    float tz0 = fmaf(n2.x, r.id.z, -r.ood.z), tz1 = fmaf(n2.y, r.id.z, -r.ood.z);
    const float c0min = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), s.tnear));
    const float c0max = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), lim));
    tx0 = fmaf(n1.x, r.id.x, -r.ood.x); tx1 = fmaf(n1.y, r.id.x, -r.ood.x);
    ty0 = fmaf(n1.z, r.id.y, -r.ood.y); ty1 = fmaf(n1.w, r.id.y, -r.ood.y);
    tz0 = fmaf(n2.z, r.id.z, -r.ood.z); tz1 = fmaf(n2.w, r.id.z, -r.ood.z);
    const float c1min = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), s.tnear));
    const float c1max = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), lim));
    const bool h0 = c0min <= c0max, h1 = c1min <= c1max;
    if (h0 && h1) {
      int near = n3.x, far = n3.y;
      if (c1min < c0min) { near = n3.y; far = n3.x; }
      if (s.sp >= BVH_STACK) {
        atomicOr(err, ERR_STACK);
        s.best = -1;
        return true;
      }
      stack[s.sp++] = far;
      s.cur = near;
      return false;
    }
    if (h0) { s.cur = n3.x; return false; }
    if (h1) { s.cur = n3.y; return false; }
  } else {
    const unsigned v = ~(unsigned)s.cur;
    const int start = (int)(v >> 3), count = (int)(v & 7u) + 1;
    for (int i = start; i < start + count; ++i) {
      const float4 a = __ldg(&bvh.tris[3 * i]);
      const float4 b = __ldg(&bvh.tris[3 * i + 1]);
      const float4 c = __ldg(&bvh.tris[3 * i + 2]);
      if (COUNT) cnt->tris++;
      float t, b1 = 0.f, b2 = 0.f;
      bool hit;
      if (SPH && __float_as_int(c.w) != 0) hit = intersect_sphere(r, a, b, s.tnear, s.best_t, &t);
      else hit = intersect_tri(r, xyz(a), xyz(b), xyz(c), s.tnear, s.best_t, &t, &b1, &b2);
      if (hit && (ANY || closer(t, __float_as_int(a.w), s.best_t, s.best_prim))) {
        s.best = i;
        s.best_prim = __float_as_int(a.w);
        s.best_t = t;
        s.b1 = b1;
        s.b2 = b2;
        if (ANY) return true;
      }
    }
  }
  if (s.sp == 0) return true;
  s.cur = stack[--s.sp];
  return false;
}

// No node: larger than any node index and not a leaf reference (leaf references are
// negative, -1 included).
constexpr int kNoNode = 0x7fffffff;

// Both child boxes of binary node `node` against the ray, culled beyond best_t: returns
// the child to visit next (kNoNode when neither is hit) and, when both are hit, the
// farther one in *far_out (else kNoNode).
__device__ __forceinline__ int visit_node2(const float4* __restrict__ nodes, const RayPre& r, int node, float tnear,
                                           float best_t, int* far_out) {
  const float4* np = nodes + 4 * (size_t)node;
  const float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
  const int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
  const float lim = best_t * 1.0000004f;  // 1 + 2 gamma(3): conservative slabs
  float tx0 = fmaf(n0.x, r.id.x, -r.ood.x), tx1 = fmaf(n0.y, r.id.x, -r.ood.x);
  float ty0 = fmaf(n0.z, r.id.y, -r.ood.y), ty1 = fmaf(n0.w, r.id.y, -r.ood.y);
  float tz0 = fmaf(n2.x, r.id.z, -r.ood.z), tz1 = fmaf(n2.y, r.id.z, -r.ood.z);
  const float c0min = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tnear));
  const float c0max = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), lim));
  tx0 = fmaf(n1.x, r.id.x, -r.ood.x); tx1 = fmaf(n1.y, r.id.x, -r.ood.x);
  ty0 = fmaf(n1.z, r.id.y, -r.ood.y); ty1 = fmaf(n1.w, r.id.y, -r.ood.y);
  tz0 = fmaf(n2.z, r.id.z, -r.ood.z); tz1 = fmaf(n2.w, r.id.z, -r.ood.z);
  const float c1min = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tnear));
  const float c1max = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), lim));
  const bool h0 = c0min <= c0max, h1 = c1min <= c1max;
  *far_out = kNoNode;
  if (h0 && h1) {
    const bool swap = c1min < c0min;
    *far_out = swap ? n3.x : n3.y;
    return swap ? n3.y : n3.x;
  }
  return h0 ? n3.x : (h1 ? n3.y : kNoNode);
}

// Binary-BVH traversal in the "speculative while-while" form of Aila and Laine (2009,
// "Understanding the efficiency of ray traversal on GPUs"): a lane that reaches a leaf
// postpones it and keeps descending inner nodes until every active lane of the warp holds
// a leaf (or has finished); then the lanes test their leaves' primitives together, so inner
// and leaf work run in separate loops instead of splitting the warp every step.  A
// postponed leaf is tested after the inner nodes visited meanwhile (their culling used the
// older best_t, which only adds work); the closest hit and its tie-break are unchanged.
template <bool ANY, bool COUNT, bool SPH>
__device__ __forceinline__ void trace_ww(const BvhRef& bvh, TraceState& s, int* stack, unsigned int* err,
                                         TraceCounters* cnt) {
  const RayPre& r = s.r;
  int cur = 0;         // the root is always an inner node
  int leaf = kNoNode;  // postponed leaf reference, or kNoNode
  int sp = 0;
  while (cur != kNoNode || leaf != kNoNode) {
    // Inner nodes (0 <= cur < kNoNode).
    while ((unsigned)cur < (unsigned)kNoNode) {
      int far;
      const int next = visit_node2(bvh.nodes, r, cur, s.tnear, s.best_t, &far);
      if (COUNT) cnt->nodes++;
      if (next == kNoNode) {
        cur = sp > 0 ? stack[--sp] : kNoNode;
      } else {
        if (far != kNoNode) {
          if (sp >= BVH_STACK) {
            atomicOr(err, ERR_STACK);
            s.best = -1;
            return;
          }
          stack[sp++] = far;
        }
        cur = next;
      }
      // Postpone the first leaf met and carry on with the stack.
      if (cur < 0 && leaf == kNoNode) {
        leaf = cur;
        cur = sp > 0 ? stack[--sp] : kNoNode;
      }
      if (!__any_sync(__activemask(), leaf == kNoNode)) break;
    }
    // Leaves: the postponed one, then cur while it is a leaf.
    while (leaf != kNoNode) {
      const unsigned v = ~(unsigned)leaf;
      const int start = (int)(v >> 3), count = (int)(v & 7u) + 1;
      for (int i = start; i < start + count; ++i) {
        const float4 a = __ldg(&bvh.tris[3 * i]);
        const float4 b = __ldg(&bvh.tris[3 * i + 1]);
        const float4 c = __ldg(&bvh.tris[3 * i + 2]);
        if (COUNT) cnt->tris++;
        float t, b1 = 0.f, b2 = 0.f;
        bool hit;
        if (SPH && __float_as_int(c.w) != 0) hit = intersect_sphere(r, a, b, s.tnear, s.best_t, &t);
        else hit = intersect_tri(r, xyz(a), xyz(b), xyz(c), s.tnear, s.best_t, &t, &b1, &b2);
        if (hit && (ANY || closer(t, __float_as_int(a.w), s.best_t, s.best_prim))) {
          s.best = i;
          s.best_prim = __float_as_int(a.w);
          s.best_t = t;
          s.b1 = b1;
          s.b2 = b2;
          if (ANY) return;
        }
      }
      leaf = kNoNode;
      if (cur < 0) {
        leaf = cur;
        cur = sp > 0 ? stack[--sp] : kNoNode;
      }
    }
  }
}

// Traversal of the 4-wide layout (the binary tree collapsed to nodes of up to four
// children: tt_build.h).  A node's four boxes are tested together (structure of arrays),
// the hit children sorted by entry distance: the nearest is visited next, the others pushed
// farthest first.  Closest hit postpones leaves as trace_ww does (speculative while-while);
// any hit tests a leaf as soon as it reaches it.  Half the binary tree's depth means half
// the chain of dependent node fetches that bounds the traversal.  (Used for closest hit;
// the ANY form, leaves tested as soon as reached, measured slower than the binary per-step
// traversal for shadow rays.)
__device__ __forceinline__ void sort2(float& da, int& ra, float& db, int& rb) {
  if (db < da) {
    const float t = da;
    da = db;
    db = t;
    const int u = ra;
    ra = rb;
    rb = u;
  }
}
template <bool ANY, bool COUNT, bool SPH>
__device__ __forceinline__ void trace4(const float4* __restrict__ nodes4, const float4* __restrict__ tris,
                                       TraceState& s, int* stack, unsigned int* err, TraceCounters* cnt) {
  const RayPre& r = s.r;
  int cur = 0;
  int leaf = kNoNode;
  int sp = 0;
  while (cur != kNoNode || leaf != kNoNode) {
    while ((unsigned)cur < (unsigned)kNoNode) {
      const float4* np = nodes4 + 8 * (size_t)cur;
      const float4 lx = __ldg(np), hx = __ldg(np + 1), ly = __ldg(np + 2), hy = __ldg(np + 3);
      const float4 lz = __ldg(np + 4), hz = __ldg(np + 5);
      const int4 rf = __ldg(reinterpret_cast<const int4*>(np + 6));
      if (COUNT) cnt->nodes++;
      const float lim = s.best_t * 1.0000004f;  // 1 + 2 gamma(3): conservative slabs
      const float lxs[4] = {lx.x, lx.y, lx.z, lx.w}, hxs[4] = {hx.x, hx.y, hx.z, hx.w};
      const float lys[4] = {ly.x, ly.y, ly.z, ly.w}, hys[4] = {hy.x, hy.y, hy.z, hy.w};
      const float lzs[4] = {lz.x, lz.y, lz.z, lz.w}, hzs[4] = {hz.x, hz.y, hz.z, hz.w};
      float d[4];
      int c[4] = {rf.x, rf.y, rf.z, rf.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float tx0 = fmaf(lxs[j], r.id.x, -r.ood.x), tx1 = fmaf(hxs[j], r.id.x, -r.ood.x);
        const float ty0 = fmaf(lys[j], r.id.y, -r.ood.y), ty1 = fmaf(hys[j], r.id.y, -r.ood.y);
        const float tz0 = fmaf(lzs[j], r.id.z, -r.ood.z), tz1 = fmaf(hzs[j], r.id.z, -r.ood.z);
        const float tmin = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), s.tnear));
        const float tmax = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), lim));
        d[j] = (tmin <= tmax && c[j] != kNoNode) ? tmin : INFINITY;  // empty slots never hit
      }
      sort2(d[0], c[0], d[1], c[1]);
      sort2(d[2], c[2], d[3], c[3]);
      sort2(d[0], c[0], d[2], c[2]);
      sort2(d[1], c[1], d[3], c[3]);
      sort2(d[1], c[1], d[2], c[2]);
      if (d[0] == INFINITY) {
        cur = sp > 0 ? stack[--sp] : kNoNode;
      } else {
        if (sp + 3 > BVH_STACK) {
          atomicOr(err, ERR_STACK);
          s.best = -1;
          return;
        }
        if (d[3] != INFINITY) stack[sp++] = c[3];
        if (d[2] != INFINITY) stack[sp++] = c[2];
        if (d[1] != INFINITY) stack[sp++] = c[1];
        cur = c[0];
      }
      if (cur < 0 && leaf == kNoNode) {
        leaf = cur;
        cur = sp > 0 ? stack[--sp] : kNoNode;
        if (ANY) break;
      }
      if (!ANY && !__any_sync(__activemask(), leaf == kNoNode)) break;
    }
    while (leaf != kNoNode) {
      const unsigned v = ~(unsigned)leaf;
      const int start = (int)(v >> 3), count = (int)(v & 7u) + 1;
      for (int i = start; i < start + count; ++i) {
        const float4 a = __ldg(&tris[3 * i]);
        const float4 b = __ldg(&tris[3 * i + 1]);
        const float4 cc = __ldg(&tris[3 * i + 2]);
        if (COUNT) cnt->tris++;
        float t, b1 = 0.f, b2 = 0.f;
        bool hit;
        if (SPH && __float_as_int(cc.w) != 0) hit = intersect_sphere(r, a, b, s.tnear, s.best_t, &t);
        else hit = intersect_tri(r, xyz(a), xyz(b), xyz(cc), s.tnear, s.best_t, &t, &b1, &b2);
        if (hit && (ANY || closer(t, __float_as_int(a.w), s.best_t, s.best_prim))) {
          s.best = i;
          s.best_prim = __float_as_int(a.w);
          s.best_t = t;
          s.b1 = b1;
          s.b2 = b2;
          if (ANY) return;
        }
      }
      leaf = kNoNode;
      if (cur < 0) {
        leaf = cur;
        cur = sp > 0 ? stack[--sp] : kNoNode;
      }
    }
  }
}

// Recomputes the distance of the closest hit from the plane equation in double precision
// (float rounding of Ng.(v0 - o) is amplified by 1/|cos| at grazing incidence).
__device__ __forceinline__ float refine_t(const float4* tris, const RayPre& r, int slot) {
  const float4 a = __ldg(&tris[3 * slot]);
  const float4 b = __ldg(&tris[3 * slot + 1]);
  const float4 c = __ldg(&tris[3 * slot + 2]);
  const double e1x = (double)b.x - a.x, e1y = (double)b.y - a.y, e1z = (double)b.z - a.z;
  const double e2x = (double)c.x - a.x, e2y = (double)c.y - a.y, e2z = (double)c.z - a.z;
  const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
  const double ax = (double)a.x - r.o.x, ay = (double)a.y - r.o.y, az = (double)a.z - r.o.z;
  const double den = nx * r.d.x + ny * r.d.y + nz * r.d.z;
  return (float)((nx * ax + ny * ay + nz * az) / den);
}

// ----------------------------------------------------------------------------------------
// 8-wide BVH traversal (layout in tt_bvh.h), after the compressed wide BVH of Ylitie, Karras
// and Laine (2017): one 80-byte node gives the quantised boxes of eight children; hit
// inner children form a "node group" (first child index, inner mask, hit bits in
// octant-permuted order) that is consumed nearest-first, with the rest pushed on a short
// stack; hit leaf children form a primitive group tested right away.  Slab distances are
// (p - o) / d + q * 2^e / d per axis, widened by 1 + 2 gamma(3) for conservative culling.

// Maps bit s of an 8-bit mask to bit s ^ oct.
__device__ __forceinline__ unsigned permute8(unsigned m, unsigned oct) {
  if (oct & 1u) m = ((m & 0x55u) << 1) | ((m & 0xAAu) >> 1);
  if (oct & 2u) m = ((m & 0x33u) << 2) | ((m & 0xCCu) >> 2);
  if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m & 0xF0u) >> 4);
  return m;
}

// Three-input minimum and maximum (PTX ISA 8.8, sm_100+).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

struct Trace8State {
  uint2 ng;     // node group: x = first child node, y = inner mask << 8 | permuted hit bits
  uint2 pg;     // primitive group: x = first slot, y = slots still to test (bit i = x + i)
  int best, best_prim, sp;
  float tnear, best_t, b1, b2;
};

template <bool COUNT>
__device__ __forceinline__ void visit_node8(const uint4* __restrict__ nodes, const RayPre& r, unsigned oct,
                                            unsigned node, Trace8State& s, TraceCounters* cnt) {
  const uint4* np = nodes + 5 * (size_t)node;
  const uint4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
  if (COUNT) cnt->nodes++;
  const float ax = (__uint_as_float(n0.x) - r.o.x) * r.id.x;
  const float ay = (__uint_as_float(n0.y) - r.o.y) * r.id.y;
  const float az = (__uint_as_float(n0.z) - r.o.z) * r.id.z;
  const float sx = __uint_as_float((n0.w & 0xffu) << 23) * r.id.x;
  const float sy = __uint_as_float(((n0.w >> 8) & 0xffu) << 23) * r.id.y;
  const float sz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23) * r.id.z;
  // Far planes carry the 1 + 2 gamma(3) widening through their per-node constants.
  constexpr float kWiden = 1.0000011f;
  const float fax = ax * kWiden, fay = ay * kWiden, faz = az * kWiden;
  const float fsx = sx * kWiden, fsy = sy * kWiden, fsz = sz * kWiden;
  const float lim = s.best_t * kWiden;
  const unsigned imask = n0.w >> 24;
  // Near and far planes per axis follow the ray direction's signs.
  const uint2 lox = make_uint2(n2.x, n2.y), loy = make_uint2(n2.z, n2.w), loz = make_uint2(n3.x, n3.y);
  const uint2 hix = make_uint2(n3.z, n3.w), hiy = make_uint2(n4.x, n4.y), hiz = make_uint2(n4.z, n4.w);
  const uint2 nx = (oct & 1u) ? hix : lox, fx = (oct & 1u) ? lox : hix;
  const uint2 ny = (oct & 2u) ? hiy : loy, fy = (oct & 2u) ? loy : hiy;
  const uint2 nz = (oct & 4u) ? hiz : loz, fz = (oct & 4u) ? loz : hiz;
  unsigned hits = 0u;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const unsigned sh = 8u * (unsigned)(c & 3);
    const unsigned wnx = c < 4 ? nx.x : nx.y, wny = c < 4 ? ny.x : ny.y, wnz = c < 4 ? nz.x : nz.y;
    const unsigned wfx = c < 4 ? fx.x : fx.y, wfy = c < 4 ? fy.x : fy.y, wfz = c < 4 ? fz.x : fz.y;
    const float tnx = fmaf((float)((wnx >> sh) & 0xffu), sx, ax);
    const float tny = fmaf((float)((wny >> sh) & 0xffu), sy, ay);
    const float tnz = fmaf((float)((wnz >> sh) & 0xffu), sz, az);
    const float tfx = fmaf((float)((wfx >> sh) & 0xffu), fsx, fax);
    const float tfy = fmaf((float)((wfy >> sh) & 0xffu), fsy, fay);
    const float tfz = fmaf((float)((wfz >> sh) & 0xffu), fsz, faz);
    const float tmin = fmax3(tnx, tny, fmaxf(tnz, s.tnear));
    const float tmax = fmin3(tfx, tfy, fminf(tfz, lim));
    hits |= (tmin <= tmax ? 1u : 0u) << c;
  }
  // Leaf children (nonzero meta bytes) that were hit contribute their primitive slots.
  unsigned prims = 0u;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const unsigned m = ((c < 4 ? n1.z : n1.w) >> (8u * (unsigned)(c & 3))) & 0xffu;
    if (m != 0u && ((hits >> c) & 1u)) prims |= ((1u << (m & 3u)) - 1u) << (m >> 2);
  }
  s.ng = make_uint2(n1.x, (imask << 8) | permute8(hits & imask, oct));
  s.pg = make_uint2(n1.y, prims);
}

template <bool ANY, bool COUNT, bool SPH>
__device__ __forceinline__ void trace8_run(const uint4* __restrict__ nodes, const float4* __restrict__ tris,
                                           const RayPre& r, Trace8State& s, unsigned int* err, TraceCounters* cnt) {
  // Octant from the signs of the reciprocal direction, which carry the sign of a -0
  // component (safe_inv), so near and far planes are chosen consistently with it.
  const unsigned oct = (r.id.x < 0.f ? 1u : 0u) | (r.id.y < 0.f ? 2u : 0u) | (r.id.z < 0.f ? 4u : 0u);
  uint2 stack[BVH8_STACK];
  s.ng = make_uint2(0u, (1u << 8) | (1u << oct));  // the root as the single inner child of slot 0
  s.pg = make_uint2(0u, 0u);
  s.sp = 0;
  for (;;) {
    if (s.ng.y & 0xffu) {
      const unsigned p = (unsigned)__ffs(s.ng.y & 0xffu) - 1u;
      const unsigned slot = p ^ oct;
      const unsigned node = s.ng.x + (unsigned)__popc((s.ng.y >> 8) & ((1u << slot) - 1u));
      s.ng.y &= ~(1u << p);
      if (s.ng.y & 0xffu) {
        if (s.sp >= BVH8_STACK) {
          atomicOr(err, ERR_STACK);
          s.best = -1;
          return;
        }
        stack[s.sp++] = s.ng;
      }
      visit_node8<COUNT>(nodes, r, oct, node, s, cnt);
    }
    while (s.pg.y) {
      const int k = __ffs(s.pg.y) - 1;
      s.pg.y &= s.pg.y - 1u;
      const int i = (int)s.pg.x + k;
      const float4 a = __ldg(&tris[3 * i]);
      const float4 b = __ldg(&tris[3 * i + 1]);
      const float4 c = __ldg(&tris[3 * i + 2]);
      if (COUNT) cnt->tris++;
      float t, b1 = 0.f, b2 = 0.f;
      bool hit;
      if (SPH && __float_as_int(c.w) != 0) hit = intersect_sphere(r, a, b, s.tnear, s.best_t, &t);
      else hit = intersect_tri(r, xyz(a), xyz(b), xyz(c), s.tnear, s.best_t, &t, &b1, &b2);
      if (hit && (ANY || closer(t, __float_as_int(a.w), s.best_t, s.best_prim))) {
        s.best = i;
        s.best_prim = __float_as_int(a.w);
        s.best_t = t;
        s.b1 = b1;
        s.b2 = b2;
        if (ANY) return;
      }
    }
    if (!(s.ng.y & 0xffu)) {
      if (s.sp == 0) return;
      s.ng = stack[--s.sp];
    }
  }
}

// Whole traversal of one ray (batch queries).  Returns the triangle slot or -1.
template <bool ANY, bool COUNT, bool SPH, bool WIDE>
__device__ __forceinline__ int trace(const DevScene& sc, const RayPre& r, float tnear, float tfar, float* t_out,
                                     float* b1_out, float* b2_out, unsigned int* err, TraceCounters* cnt) {
  if (WIDE) {
    Trace8State s;
    s.tnear = tnear;
    s.best_t = tfar;
    s.best = -1;
    s.best_prim = 0x7fffffff;
    s.b1 = s.b2 = 0.f;
    trace8_run<ANY, COUNT, SPH>(sc.nodes8, sc.tris, r, s, err, cnt);
    if (s.best >= 0) {
      *t_out = (ANY || (SPH && is_sphere_slot(sc.tris, s.best))) ? s.best_t : refine_t(sc.tris, r, s.best);
      *b1_out = s.b1;
      *b2_out = s.b2;
    }
    return s.best;
  }
  const BvhRef bvh = surface_bvh(sc);
  TraceState s;
  int stack[BVH_STACK];
  s.r = r;
  s.tnear = tnear;
  s.best_t = tfar;
  s.b1 = s.b2 = 0.f;
  s.best = -1;
  s.best_prim = 0x7fffffff;
  s.cur = 0;
  s.sp = 0;
  if (!ANY && sc.nodes4) {
    // Closest hit on the 4-wide nodes (6 % less closest-hit time than the binary while-while
    // traversal on the terrain workload).
    trace4<ANY, COUNT, SPH>(sc.nodes4, sc.tris, s, stack, err, cnt);
  } else if (ANY) {
    // Any hit: one binary node or leaf per step, so that a lane meets its first hit as early
    // as the tree order allows (postponing leaves measured 3.5 % slower for shadow rays, the
    // 4-wide nodes 7 % slower).
    while (!trace_step<ANY, COUNT, SPH>(bvh, s, stack, err, cnt)) {
    }
  } else {
    // Closest hit: while-while traversal (6.5 % less closest-hit time on the bench frame).
    trace_ww<ANY, COUNT, SPH>(bvh, s, stack, err, cnt);
  }
  if (s.best >= 0) {
    *t_out = (ANY || (SPH && is_sphere_slot(sc.tris, s.best))) ? s.best_t : refine_t(sc.tris, r, s.best);
    *b1_out = s.b1;
    *b2_out = s.b2;
  }
  return s.best;
}

// Nearest hit with tnear < t <= tfar in `bvh`, with the single-precision plane distance
// (no refinement, so that the next query can start exactly at the returned t).  Returns
// the triangle slot or -1.
template <bool SPH>
__device__ __forceinline__ int next_hit8(const uint4* nodes, const float4* tris, const RayPre& r, float tnear,
                                         float tfar, float* t_out, unsigned int* err) {
  Trace8State s;
  s.tnear = tnear;
  s.best_t = tfar;
  s.best = -1;
  s.best_prim = 0x7fffffff;
  s.b1 = s.b2 = 0.f;
  trace8_run<false, false, SPH>(nodes, tris, r, s, err, nullptr);
  *t_out = s.best_t;
  return s.best;
}

template <bool SPH>
__device__ __forceinline__ int next_hit(const BvhRef& bvh, const RayPre& r, float tnear, float tfar, float* t_out,
                                        unsigned int* err) {
  TraceState s;
  int stack[BVH_STACK];
  s.r = r;
  s.tnear = tnear;
  s.best_t = tfar;
  s.b1 = s.b2 = 0.f;
  s.best = -1;
  s.best_prim = 0x7fffffff;
  s.cur = 0;
  s.sp = 0;
  while (!trace_step<false, false, SPH>(bvh, s, stack, err, nullptr)) {
  }
  *t_out = s.best_t;
  return s.best;
}

// Nearest medium-boundary crossing after tnear: the next entry of
// EmbreeAccelerator::IntersectionsInOrder (embreeaccelerator.cxx:134-213).  Walking the
// crossings one query at a time with tnear = the previous crossing drops repeated hits at
// the same distance, as the reference's (geometry, t) de-duplication does for the two
// triangles that share an edge the ray passes through.
template <bool SPH, bool WIDE>
__device__ __forceinline__ int next_crossing(const DevScene& sc, const RayPre& r, float tnear, float tfar,
                                             float* t_out, unsigned int* err) {
  if (sc.num_vol_tris == 0) return -1;
  if (WIDE) return next_hit8<SPH>(sc.vnodes8, sc.vtris, r, tnear, tfar, t_out, err);
  return next_hit<SPH>(volume_bvh(sc), r, tnear, tfar, t_out, err);
}

// Winding normal (a sphere's: outward at o + t d) and material of a slot.
__device__ __forceinline__ void crossing_info(const float4* tris, int slot, float3 o, float3 d, float t, float3* ng,
                                              int* material) {
  const float4 a = __ldg(&tris[3 * slot]);
  const float4 b = __ldg(&tris[3 * slot + 1]);
  const float4 c = __ldg(&tris[3 * slot + 2]);
  *ng = __float_as_int(c.w) != 0 ? (o + d * t) - xyz(a) : cross3(xyz(b) - xyz(a), xyz(c) - xyz(a));
  *material = __float_as_int(b.w);
}

// ----------------------------------------------------------------------------------------
// Light sampling and connection (TrivialLightPicker::PickLight, EmitterSampleVisitor,
// CalculateConnection, PdfConversionFactor; rendering_randomwalk_impl.hxx:192-250,
// 373-409, 493-513).
enum { LIGHT_NONE = -1, LIGHT_ENV = 0, LIGHT_AREA = 1, LIGHT_POINT = 2 };

struct LightNode {
  int type;
  float3 coord;      // area: position; env: direction of travel; point: position
  float3 ng;         // area: raw winding normal
  float3 bounds;     // area: position error bound
  float3 radiance;   // env radiance / point spectrum
  int prim;
  float pdf;
  bool delta;
};

__device__ __forceinline__ float tri_area(float3 p0, float3 p1, float3 p2) {
  return 0.5f * len3(cross3(p1 - p0, p2 - p0));
}

struct Connection {
  float3 org, dir;
  float len;
  float3 weight;    // scatter * target * DFactors * r2 (transmittance excluded)
  float pdf_due;    // pdf of sampling the light vertex by scattering, light's measure
  float pdf_eye;    // scatter density of the direction at the eye (solid angle)
  float conv;       // pdf_due / pdf_eye: DFactor(light) / distance^2 (DFactor alone for an env light)
  bool valid;       // nonzero weight: a shadow ray is needed
  int unit;         // camera eye: pixel the connection lands in
};

struct Eye {
  bool is_camera;
  bool is_volume;   // a scattering event inside a medium
  float3 pos;       // camera or volume-vertex position
  Surf surf;        // surface eye
  float3 wi;        // reverse incident direction (surface and volume eyes)
  const DevMaterial* mat;
  const DevMedium* med;  // volume eye: its medium
  float3 sigma_s;        // volume eye: scattering coefficient at the vertex
  const DevCamera* cam;  // camera eye: its camera
};

__device__ __forceinline__ Connection connect(const DevScene& sc, const Eye& eye, const LightNode& L, Lambda l) {
  Connection c;
  c.valid = false;
  c.unit = -1;
  c.pdf_due = 0.f;
  c.pdf_eye = 0.f;
  c.conv = 0.f;
  c.weight = f3(0.f, 0.f, 0.f);
  const bool light_env = L.type == LIGHT_ENV;
  const bool point_eye = eye.is_camera || eye.is_volume;  // no surface offset, DFactor 1
  float3 cs = point_eye ? eye.pos : eye.surf.pos;
  float3 ct = L.coord;
  // CalculateSegmentToTarget: direction, offsets on surface nodes, recompute.
  float3 d;
  float len;
  if (!light_env) {
    const float3 dd = ct - cs;
    len = len3(dd);
    d = dd * (1.f / len);
  } else {
    d = -ct;
    len = sc.long_distance;
  }
  if (!point_eye) cs = cs + offset_at(eye.surf, d);
  if (L.type == LIGHT_AREA) {
    const float delta = dot3(L.bounds, abs3(L.ng));
    ct = ct + (delta * (dot3(-d, L.ng) > 0.f ? 1.f : -1.f)) * L.ng;
  }
  if (!light_env) {
    const float3 dd = ct - cs;
    len = len3(dd);
    d = dd * (1.f / len);
  }
  c.org = cs;
  c.dir = d;
  c.len = len;
  // Eye factor.
  float3 sf;
  float pdf_eye = 0.f;
  if (eye.is_camera) {
    const int unit = camera_evaluate(*eye.cam, d, &pdf_eye);
    c.unit = unit;
    sf = unit >= 0 ? f3(pdf_eye, pdf_eye, pdf_eye) : f3(0.f, 0.f, 0.f);
  } else if (eye.is_volume) {
    // EvaluateScatterCoordinateOfScatterer, volume branch: sigma_s x phase function.
    sf = mul(eye.sigma_s, medium_phase_eval(*eye.med, eye.pos, eye.wi, d, l, &pdf_eye));
  } else {
    sf = eval_bsdf(*eye.mat, eye.wi, eye.surf, d, l, &pdf_eye) * bsdf_correction(eye.surf, d);
  }
  // Light factor and DFactor of the light vertex.
  float3 tf;
  float dfac_light = 1.f;
  if (L.type == LIGHT_AREA) {
    const DevMaterial& lm = sc.materials[__ldg(&sc.tri_idx[L.prim]).w];
    const float vis = dot3(L.ng, -d) > 0.f ? 1.f : 0.f;
    tf = take(lm.emission, l) * (vis / (2.f * kPi));
    dfac_light = fabsf(dot3(L.ng, d));
  } else {
    tf = L.radiance;
  }
  // PdfConversionFactor(eye, light): DFactor(light) / (len^2 + eps) unless the light is at
  // infinity.
  c.conv = light_env ? dfac_light : dfac_light / (len * len + kEps);
  c.pdf_eye = pdf_eye;
  c.pdf_due = pdf_eye * c.conv;
  if (is_zero(sf) || is_zero(tf)) return c;
  const float dfac_eye = point_eye ? 1.f : fabsf(dot3(eye.surf.ng, d));
  const float r2 = light_env ? 1.f : 1.f / (len * len);
  c.weight = mul(sf * dfac_eye, tf * dfac_light) * r2;
  c.valid = true;
  return c;
}

// Completes an area light sample: position, winding normal, error bound and pdf.  The
// vertices come from the per-light table (area light order), not from the leaf slots.  A
// sphere light (a.w = 1: centre a.xyz, radius b.x) takes L.coord as a uniform direction
// (Spheres::SampleUniformPosition, primitive.cxx:193-203).
__device__ __forceinline__ void resolve_area(const DevScene& sc, int light_index, LightNode& L) {
  const float4 a = __ldg(&sc.area_verts[3 * light_index]);
  const float4 b = __ldg(&sc.area_verts[3 * light_index + 1]);
  const float4 c = __ldg(&sc.area_verts[3 * light_index + 2]);
  if (a.w != 0.f) {
    const float3 off = L.coord * b.x;
    L.coord = xyz(a) + off;
    L.ng = normalize3(off);
    L.bounds = abs3(L.coord) * gamma5();
    L.pdf = (sc.type_probs[1] / sc.num_area_lights) * (1.f / (b.x * b.x * 4.f * kPi));
    return;
  }
  const float3 p0 = xyz(a), p1 = xyz(b), p2 = xyz(c);
  const float3 w = L.coord;
  L.coord = p0 * w.x + p1 * w.y + p2 * w.z;
  L.ng = normalize3(cross3(p1 - p0, p2 - p0));
  L.bounds = (abs3(p0 * w.x) + abs3(p1 * w.y) + abs3(p2 * w.z)) * gamma7();
  const float area = tri_area(p0, p1, p2);
  L.pdf = (sc.type_probs[1] / sc.num_area_lights) * (1.f / area);
}

// ----------------------------------------------------------------------------------------
__device__ __forceinline__ float mis_weight(const DevScene& sc, float pdf_taken, bool delta, float pdf_other) {
  if (!delta && sc.sample_bsdf && sc.sample_lights) return power_heuristic(pdf_taken, pdf_other);
  return 1.f;
}

__device__ __forceinline__ LightNode pick_light(const DevScene& sc, Rng& rng, Lambda l) {
  LightNode L;
  L.type = LIGHT_NONE;
  L.delta = false;
  L.pdf = 0.f;
  // A scene without lights has none to pick: no draw, no connection.
  if (sc.num_env == 0 && sc.num_area_lights == 0 && sc.num_point_lights == 0) return L;
  const int which = tower_sampling4(sc.type_probs, rng.uniform());
  if (which == LIGHT_ENV) {
    const int i = rng.uniform_int(0, sc.num_env - 1);
    DirSample s = env_sample_one(sc.env[i], rng, l);
    L.type = LIGHT_ENV;
    L.coord = s.dir;
    L.radiance = s.value;
    L.pdf = sc.type_probs[0] * (s.pdf * (1.f / sc.num_env));
    L.delta = s.delta;
  } else if (which == LIGHT_POINT) {
    const int n = sc.num_point_lights;
    const int i = rng.uniform_int(0, n - 1);
    const float* pl = sc.point_lights + (size_t)i * (NBINS + 3);
    L.type = LIGHT_POINT;
    L.coord = f3(pl[NBINS], pl[NBINS + 1], pl[NBINS + 2]);
    L.radiance = take(pl, l) * (1.f / (4.f * kPi));
    L.pdf = sc.type_probs[2] / n;
    L.delta = true;
  } else if (which == LIGHT_AREA) {
    const int n = sc.num_area_lights;
    const int i = rng.uniform_int(0, n - 1);
    float r[2];
    rng.square(r);
    L.type = LIGHT_AREA;
    L.prim = __ldg(&sc.area_lights[i]);
    L.coord = __ldg(&sc.area_verts[3 * i]).w != 0.f ? to_uniform_sphere(r) : to_triangle_barycentric(r);
    resolve_area(sc, i, L);
  }
  return L;
}

// ----------------------------------------------------------------------------------------
// Queues a shadow ray for the connection c.  Without media the MIS weight is final here;
// with media it depends on the transmittance pdf factor of the segment, which the shadow
// kernel computes, so the light pdf and the scatter pdf travel with the ray.
template <bool MEDIA>
__device__ __forceinline__ void emit_shadow(const DevScene& sc, const PathState& p, int qbounce, int slot,
                                            const Connection& c, const LightNode& L, float3 beta, float scale,
                                            int target, const MTracker& mt, const Rng& rng,
                                            bool defer_mis = false) {
  float3 contrib;
  if (defer_mis) {
    // Guided vertex: the scatter density is the one-sample-MIS mixture, known only after
    // the network ran; k_guide completes the weight.
    const bool mis_on = !L.delta && sc.sample_bsdf && sc.sample_lights;
    p.gnee[slot] = make_float4(mis_on ? L.pdf : -1.f, c.conv, c.pdf_eye, 1.f);
  }
  if (MEDIA) {
    contrib = mul(c.weight, beta) * (scale / L.pdf);
    const bool mis_on = !L.delta && sc.sample_bsdf && sc.sample_lights;
    // The path's random state here seeds the shadow ray's own stream for ratio tracking.
    p.sh_med[slot] = make_float4(mis_on ? L.pdf : -1.f, c.pdf_due, __uint_as_float((unsigned)(rng.state & 0xffffffffu)),
                                 __uint_as_float((unsigned)(rng.state >> 32)));
    p.sh_track[slot] = store_tracker(mt);
  } else {
    const float mis = defer_mis ? 1.f : mis_weight(sc, L.pdf, L.delta, c.pdf_due);
    contrib = mul(c.weight, beta) * (mis * scale / L.pdf);
  }
  const int q = warp_append(sh_count(p, qbounce));
  p.sh_q[q] = slot;
  p.sh_o[slot] = make_float4(c.org.x, c.org.y, c.org.z, c.len * 0.9999f);
  p.sh_d[slot] = make_float4(c.dir.x, c.dir.y, c.dir.z, __int_as_float(target));
  p.sh_c[slot] = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
}

// One camera sample: wavelength selection, next-event estimation at the camera vertex
// (splatted to the pixel the light sample projects to, scaled by splat_scale), camera ray.
// `slot` is the path's slot, `pixel` its index in the framebuffer, `unit` the pixel within
// the camera, `sample` the sample's index in its pixel (the quasi-random point index); the
// random stream is (seed, path_id).
template <bool MEDIA>
__device__ __forceinline__ void generate_one(const DevScene& sc, const PathState& p, int slot, int pixel, int unit,
                                             unsigned long long seed, unsigned long long path_id,
                                             unsigned long long sample, const DevCamera& cam, uint2 cam_track,
                                             float splat_scale, int splat_base) {
  const int i = slot;
  Smp2 smp;
  Rng& rng = smp.rng;
  rng.seed_path(seed, path_id);
  smp.mats = sc.sobol;
  // LambdaSelectionStrategy::WithWeights (shader_util.hxx:83-91).
  const int main_idx = rng.uniform_int(0, 11);
  int idx[3] = {main_idx, main_idx + 12, main_idx + 24};
  const int rot = rng.uniform_int(0, 2);
  { const int t = idx[0]; idx[0] = idx[rot]; idx[rot] = t; }
  // SampleWavelengthStrata: its values are not used; quasi-random draws leave the PCG32
  // stream untouched.
  if (!smp.mats) { rng.uniform(); rng.uniform(); rng.uniform(); }
  const Lambda l{idx[0], idx[1], idx[2]};
  const float3 beta = f3(12.f, 12.f, 12.f);
  const float3 cam_pos = f3(cam.pos[0], cam.pos[1], cam.pos[2]);
  const MTracker cam_mt = load_tracker(cam_track);
  p.accum[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sc.guide_record) p.grec[(size_t)kRecF4 * i + 3] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sc.guide) p.rr[i] = 1.f;
  const bool pt2 = sc.algo == TT_ALGO_PT2;
  if (pt2) {
    // CameraRenderWorker::InitializePathState (renderingalgorithms_pathtracing2.cxx:378-405):
    // node count 2, unit track weights, no roughness; no next-event estimation at the camera.
    p.rough[i] = 0.f;
    if (MEDIA)
      for (int k = 0; k < 9; ++k) p.wt2[9 * (size_t)i + k] = 1.f;
  }
  // Next-event estimation at the camera vertex: a light sample seen directly by the
  // camera is splatted to the pixel it projects to, scaled by 1/(xres*yres).
  if (sc.sample_lights && !pt2) {
    LightNode L = pick_light(sc, rng, l);
    if (L.type != LIGHT_NONE) {
      Eye eye;
      eye.is_camera = true;
      eye.is_volume = false;
      eye.pos = cam_pos;
      eye.cam = &cam;
      Connection c = connect(sc, eye, L, l);
      if (c.valid && c.unit >= 0)
        emit_shadow<MEDIA>(sc, p, 0, i, c, L, beta, splat_scale, splat_base + c.unit, cam_mt, rng);
    }
  }
  // Camera ray (TakeRandomWalkStep from the camera node; pt2: subsequence 2, node count 1).
  DirSample s;
  if (smp.mats) {
    const int py = unit / cam.xres, px = unit - py * cam.xres;
    const int r = (px % kRotationBlock) + (py % kRotationBlock) * kRotationBlock;
    smp.q = make_uint4((uint32_t)sample, rotation_fixed(__ldg(&sc.rotations[2 * r])),
                       rotation_fixed(__ldg(&sc.rotations[2 * r + 1])), 0u);
    smp.prep(2u);
    s = camera_sample(cam, unit, smp);
    p.qmc[i] = smp.q;
  } else {
    s = camera_sample(cam, unit, rng);
  }
  const float3 bf = s.value * (1.f / s.pdf);
  // meta.z: node count; meta.w bit 0: last scatter was a delta (pt2: bit 1 = has one).
  p.meta[i] = make_uint4((unsigned)pixel, pack_lambda(l), pt2 ? 2u : 1u, pt2 ? 0u : (s.delta ? 1u : 0u));
  p.rng_state[i] = rng.state;
  p.rng_inc[i] = rng.inc;
  if (MEDIA) p.track[i] = cam_track;
  if (is_zero(bf)) {
    const int q = warp_append(done_count(p, 0));
    p.done_q[q] = i;
    return;
  }
  const float3 nb = mul(beta, bf);
  p.beta[i] = make_float4(nb.x, nb.y, nb.z, s.pdf);
  p.ray_o[i] = make_float4(cam_pos.x, cam_pos.y, cam_pos.z, 0.f);
  p.ray_d[i] = make_float4(s.dir.x, s.dir.y, s.dir.z, kLargeNumber);
  const int q = warp_append(ext_count(p, 0));
  p.ext_q[0][q] = i;
}

template <bool MEDIA>
__global__ void __launch_bounds__(256) k_generate(DevScene sc, PathState p, Framebuffer fb, WaveArgs w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.wave_paths; i += gridDim.x * blockDim.x) {
    const long long g = w.wave_start + i;
    const int pix_local = (int)(g % w.npix_range);
    const unsigned long long sample = w.sample_offset + (unsigned long long)(g / w.npix_range);
    const int pixel = w.pixel_begin + pix_local;
    generate_one<MEDIA>(sc, p, i, pixel, pixel, w.seed, sample * (unsigned long long)w.npix_total + (unsigned long long)pixel,
                        sample, sc.cam, sc.cam_track, 1.f / (float)w.npix_total, 0);
  }
}

// Multi-view batches: the wave's paths are numbered over the concatenation of the views'
// (pixel, sample) ranges; a path finds its view by binary search over the views' first
// path indices (staged in shared memory).  View v's paths use the random streams that a
// single-view pass of that camera with seed views[v].seed would use.  The wave arguments
// come from device memory (waves[*wave_idx]) so that one captured graph serves every wave.
constexpr int kMaxViewsSmem = 1024;

template <bool MEDIA>
__global__ void __launch_bounds__(256) k_generate_views(DevScene sc, PathState p, const ViewWave* waves,
                                                        const int* wave_idx, const DevView* views, int nviews) {
  __shared__ long long sbeg[kMaxViewsSmem];
  const bool staged = nviews <= kMaxViewsSmem;
  if (staged)
    for (int v = threadIdx.x; v < nviews; v += blockDim.x) sbeg[v] = views[v].path_begin;
  __syncthreads();
  const ViewWave w = waves[*wave_idx];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.wave_paths; i += gridDim.x * blockDim.x) {
    const long long g = w.wave_start + i;
    int lo = 0, hi = nviews - 1;
    while (lo < hi) {  // last view whose first path <= g
      const int mid = (lo + hi + 1) >> 1;
      const long long b = staged ? sbeg[mid] : views[mid].path_begin;
      if (b <= g) lo = mid;
      else hi = mid - 1;
    }
    const DevView& V = views[lo];
    const long long li = g - V.path_begin;
    const int pix = (int)(li % V.npix);
    const unsigned long long sample = (unsigned long long)(li / V.npix);
    generate_one<MEDIA>(sc, p, i, V.pix_begin + pix, pix, V.seed, sample * (unsigned long long)V.npix + (unsigned long long)pix,
                        sample, V.cam, V.cam_track, 1.f / (float)V.npix, V.pix_begin);
  }
}

__global__ void k_wave_advance(int* wave_idx) {
  if (blockIdx.x == 0 && threadIdx.x == 0) ++*wave_idx;
}

// rgb = (accum + splats) / spp of the pixel's view.
__global__ void k_resolve_views(const float* accum, const float* light, const DevView* views, int nviews, int npix,
                                float* rgb) {
  for (int px = blockIdx.x * blockDim.x + threadIdx.x; px < npix; px += gridDim.x * blockDim.x) {
    int lo = 0, hi = nviews - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (views[mid].pix_begin <= px) lo = mid;
      else hi = mid - 1;
    }
    const float inv = 1.f / (float)views[lo].spp;
    for (int k = 0; k < 3; ++k) rgb[3 * px + k] = (accum[3 * px + k] + light[3 * px + k]) * inv;
  }
}

// Material-sorted shading.  The shading key of a hit: 0 escaped, 1 volume vertex, 2 + the
// shader kind of the hit surface's material.  k_sort_count (or k_extend itself) keys the
// bounce's hit queue and counts the keys (a shared-memory histogram per block);
// k_sort_scatter writes every entry into its key's range of sort_q (ranges in key order,
// entries of a key in queue order within each block's share), so that the warps of k_shade
// meet one material kind each.  The sorted order interleaves the path slots of different
// keys: in a scene of two shader kinds k_shade fetched 1.8x the DRAM bytes sorted, and a
// partition within windows of 1,024 queue entries (which keeps the slots a block touches)
// did not recover the loss, so the library sorts by default only where the divergence it
// removes is larger (three or more shader kinds).
__device__ __forceinline__ int hit_key(const DevScene& sc, int tri) {
  if (tri <= -2) return 1;
  if (tri < 0) return 0;
  const int mat = __float_as_int(__ldg(&sc.tris[3 * tri + 1]).w);
  return 2 + min(sc.materials[mat].shader, kShadeKeys - 3);
}
__device__ __forceinline__ int shade_key(const DevScene& sc, const PathState& p, int slot) {
  return hit_key(sc, __float_as_int(p.hit[slot].w));
}
// Bounce 0 (camera rays, whose hits are coherent in image order) is shaded unsorted.
__host__ __device__ __forceinline__ bool sorted_bounce(const DevScene& sc, const PathState& p, int bounce) {
  return sc.sort_shading && p.sort_q && bounce >= 1;
}

// Per-block key histogram in shared memory: lanes with the same key share one shared
// atomic per warp, and the block adds its counts to the bounce's global counters once at
// the end (one global atomic per key and block; one per key and warp serialised on the few
// counter addresses).
struct KeyHistogram {
  int* h;  // kShadeKeys shared ints
  __device__ void clear() {
    if (threadIdx.x < kShadeKeys) h[threadIdx.x] = 0;
  }
  __device__ void add(int key) {
    const unsigned peers = __match_any_sync(__activemask(), key);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[key], __popc(peers));
  }
  // After a __syncthreads that follows every add.
  __device__ void flush(int* global) {
    if (threadIdx.x < kShadeKeys && h[threadIdx.x] != 0) atomicAdd(&global[threadIdx.x], h[threadIdx.x]);
  }
};

// Closest hit of the queued extension rays, one ray per thread over a grid-stride loop
// sized to the SM count times the kernel's resident blocks.  (A persistent variant that
// refilled finished lanes after every traversal step measured 20 % slower.)
template <bool COUNT, bool SPH, bool WIDE>
__global__ void __launch_bounds__(256) k_extend(DevScene sc, PathState p, int bounce, unsigned long long* counters) {
  const int n = *ext_count(p, bounce);
  const int* q = p.ext_q[bounce & 1];
  const bool keyed = sc.algo == TT_ALGO_PT && sc.num_media == 0 && sorted_bounce(sc, p, bounce);
  __shared__ int hist_mem[kShadeKeys];
  KeyHistogram hist{hist_mem};
  if (keyed) {
    hist.clear();
    __syncthreads();
  }
  TraceCounters cnt{0u, 0u};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = q[i];
    const float4 o = p.ray_o[slot], d = p.ray_d[slot];
    const RayPre r = prepare_ray(xyz(o), xyz(d));
    float t = 0.f, b1 = 0.f, b2 = 0.f;
    const int hit = trace<false, COUNT, SPH, WIDE>(sc, r, 0.f, d.w, &t, &b1, &b2, p.err, &cnt);
    p.hit[slot] = make_float4(t, b1, b2, __int_as_float(hit));
    if (keyed) {
      // Material sort, scenes without media: key and count the hit here.
      const int key = hit_key(sc, hit);
      p.sort_key[i] = (unsigned char)key;
      hist.add(key);
    }
  }
  if (keyed) {  // uniform over the grid
    __syncthreads();
    hist.flush(key_count(p, bounce));
  }
  if (COUNT) {
    atomicAdd(&counters[0], (unsigned long long)cnt.nodes);
    atomicAdd(&counters[1], (unsigned long long)cnt.tris);
  }
}

// Media scenes, after k_extend: TrackToNextInteraction (rendering_util.hxx:215-269).  The
// medium-boundary crossings in front of the surface hit (up to 0.9999 of its distance) are
// walked in order; in each segment spectral tracking samples a collision in the current
// medium.  A collision turns the hit into a volume vertex (hit.w = -2 - medium, hit.x =
// distance, vol.xyz = sigma_s); otherwise the tracker ends past every crossing.  The
// tracking weight multiplies the throughput, and vol.w receives the product of the
// segments' mean transmittances (the pdf factor of PdfConversionFactor).
template <bool SPH, bool WIDE>
__global__ void __launch_bounds__(256) k_track(DevScene sc, PathState p, int bounce) {
  const int n = *ext_count(p, bounce);
  const int* q = p.ext_q[bounce & 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = q[i];
    float4 h = p.hit[slot];
    const float4 o = p.ray_o[slot], d = p.ray_d[slot];
    const int tri = __float_as_int(h.w);
    const float vend = (tri >= 0 ? h.x : kLargeNumber) * 0.9999f;
    MTracker mt = load_tracker(p.track[slot]);
    const Lambda l = unpack_lambda(p.meta[slot].y);
    Rng rng{p.rng_state[slot], p.rng_inc[slot]};
    const RayPre r = prepare_ray(xyz(o), xyz(d));
    float3 weight = f3(1.f, 1.f, 1.f);
    float ctr = 1.f;
    float snear = 0.f;
    bool interacted = false;
    float3 sig_s = f3(0.f, 0.f, 0.f);
    for (int k = 0;; ++k) {
      float tc;
      const int cs = next_crossing<SPH, WIDE>(sc, r, snear, vend, &tc, p.err);
      const float sfar = cs >= 0 ? tc : vend;
      const int m = mt.cur;
      if (m >= 0) {
        const DevMedium& M = sc.media[m];
        const float3 sorg = xyz(o) + xyz(d) * snear;
        const InteractionSample ms = medium_interaction(M, sorg, xyz(d), sfar - snear, weight, rng, l);
        weight = mul(weight, ms.weight);
        interacted = ms.t < sfar - snear;
        ctr *= medium_segment_tr(M, sorg, xyz(d), interacted ? ms.t : sfar - snear, l);
        if (interacted) {
          h = make_float4(snear + ms.t, 0.f, 0.f, __int_as_float(-2 - m));
          sig_s = ms.sigma_s;
          break;
        }
      }
      if (cs < 0) break;
      if (k >= kMaxCrossings) {
        atomicOr(p.err, ERR_CROSSINGS);
        weight = f3(0.f, 0.f, 0.f);
        break;
      }
      float3 ng;
      int mat;
      crossing_info(sc.vtris, cs, xyz(o), xyz(d), sfar, &ng, &mat);
      going_through(sc, mt, xyz(d), ng, mat);
      snear = sfar;
    }
    if (interacted) p.hit[slot] = h;
    p.vol[slot] = make_float4(sig_s.x, sig_s.y, sig_s.z, ctr);
    p.track[slot] = store_tracker(mt);
    p.rng_state[slot] = rng.state;
    const float4 b = p.beta[slot];
    p.beta[slot] = make_float4(b.x * weight.x, b.y * weight.y, b.z * weight.z, b.w);
  }
}

__global__ void __launch_bounds__(256) k_sort_count(DevScene sc, PathState p, int bounce) {
  const int n = *ext_count(p, bounce);
  const int* q = p.ext_q[bounce & 1];
  __shared__ int hist_mem[kShadeKeys];
  KeyHistogram hist{hist_mem};
  hist.clear();
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int key = shade_key(sc, p, q[i]);
    p.sort_key[i] = (unsigned char)key;
    hist.add(key);
  }
  __syncthreads();
  hist.flush(key_count(p, bounce));
}

__global__ void __launch_bounds__(256) k_sort_scatter(PathState p, int bounce) {
  // Per block and iteration of blockDim queue entries: each warp ranks its lanes per key
  // (match_any), the block adds up the warps' counts per key in shared memory and reserves
  // its range of every key's segment with one global atomic per key, and every entry is
  // written at segment start + block range + warp offset + lane rank.
  constexpr int kWarps = 256 / 32;
  __shared__ int base[kShadeKeys];
  __shared__ int wcount[kWarps][kShadeKeys];
  __shared__ int block_off[kShadeKeys];
  if (threadIdx.x == 0) {
    const int* counts = key_count(p, bounce);
    int acc = 0;
    for (int k = 0; k < kShadeKeys; ++k) {
      base[k] = acc;
      acc += counts[k];
    }
  }
  const int n = *ext_count(p, bounce);
  const int* q = p.ext_q[bounce & 1];
  int* cursor = key_cursor(p, bounce);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const int i = i0 + threadIdx.x;
    const int key = i < n ? (int)p.sort_key[i] : -1;
    for (int k = threadIdx.x; k < kWarps * kShadeKeys; k += blockDim.x) (&wcount[0][0])[k] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (key >= 0 && lane == __ffs(peers) - 1) wcount[warp][key] = __popc(peers);
    __syncthreads();
    if (threadIdx.x < kShadeKeys) {
      const int k = threadIdx.x;
      int acc = 0;
      for (int w = 0; w < nwarps; ++w) {
        const int c = wcount[w][k];
        wcount[w][k] = acc;
        acc += c;
      }
      block_off[k] = acc > 0 ? atomicAdd(&cursor[k], acc) : 0;
    }
    __syncthreads();
    if (key >= 0) p.sort_q[base[key] + block_off[key] + wcount[warp][key] + rank] = q[i];
    __syncthreads();
  }
}

template <bool MEDIA>
__global__ void __launch_bounds__(256, MEDIA ? 2 : 3) k_shade(DevScene sc, PathState p, int bounce) {
  const int n = *ext_count(p, bounce);
  const int* q = sorted_bounce(sc, p, bounce) ? p.sort_q : p.ext_q[bounce & 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = q[i];
    const float4 h = p.hit[slot];
    const float4 d4 = p.ray_d[slot];
    const float3 dir = xyz(d4);
    uint4 meta = p.meta[slot];
    const Lambda l = unpack_lambda(meta.y);
    float4 b4 = p.beta[slot];
    float3 beta = xyz(b4);
    const float prev_pdf = b4.w;
    const bool prev_delta = meta.w & 1u;
    float4 acc4 = p.accum[slot];
    float3 acc = xyz(acc4);
    Rng rng{p.rng_state[slot], p.rng_inc[slot]};
    const int count = (int)meta.z + 1;
    const int tri = __float_as_int(h.w);
    bool done = false;
    Surf s;
    // Media: the step's transmittance pdf factor and, at a volume vertex, sigma_s.
    const float4 vol = MEDIA ? p.vol[slot] : make_float4(0.f, 0.f, 0.f, 1.f);
    const float ctr = vol.w;
    const bool is_volume = MEDIA && tri <= -2;
    const int medium = is_volume ? -2 - tri : -1;
    float3 vpos = f3(0.f, 0.f, 0.f);
    if (is_volume) {
      vpos = xyz(p.ray_o[slot]) + dir * h.x;
    } else if (tri >= 0) {
      const float u = h.y, v = h.z;
      const bool sphere = sc.num_spheres > 0 && is_sphere_slot(sc.tris, tri);
      s = sphere ? sphere_hit_surface(sc.tris, tri, xyz(p.ray_o[slot]), dir, h.x)
                 : make_surface(sc, tri, 1.f - u - v, u, v, f3(u, v, 1.f - u - v));
      orient(s, dir);
      const DevMaterial& m = sc.materials[s.material];
      if (sc.sample_bsdf && m.emissive) {
        // Emission at an emitter hit, MIS against area-light sampling.
        const float vis = dot3(s.ng, -dir) > 0.f ? 1.f : 0.f;
        const float3 end_weight = take(m.emission, l) * (vis / (2.f * kPi));
        const float4 a = __ldg(&sc.tris[3 * tri]), b = __ldg(&sc.tris[3 * tri + 1]), c = __ldg(&sc.tris[3 * tri + 2]);
        const float area = __float_as_int(c.w) != 0 ? b.x * b.x * 4.f * kPi : tri_area(xyz(a), xyz(b), xyz(c));
        const float pdf_direct = (1.f / area) * sc.type_probs[1] * sc.in_class_area;
        const float dfac = fabsf(dot3(s.ng, dir));
        float pdf_due = prev_delta ? dfac * prev_pdf : dfac / (h.x * h.x + kEps) * prev_pdf;
        if (MEDIA) pdf_due *= ctr;
        const float mis = mis_weight(sc, pdf_due, prev_delta, pdf_direct);
        acc = acc + mul(end_weight, beta) * mis;
      }
    } else {
      // Escaped: environment emission with MIS, then the walk ends.
      if (sc.sample_bsdf && sc.num_env > 0) {
        const float3 end_weight = env_eval_total(sc, -dir, l);
        const float pdf_direct = env_pdf_total(sc, -dir) * sc.type_probs[0];
        const float mis = mis_weight(sc, MEDIA ? prev_pdf * ctr : prev_pdf, prev_delta, pdf_direct);
        acc = acc + mul(end_weight, beta) * mis;
      }
      done = true;
    }
    // Russian roulette (SurvivalAtNthScatterNode, rendering_randomwalk_impl.hxx:736-755).
    // In guided scenes the survival probability uses the throughput the path would have
    // had with the BSDF densities in place of the one-sample-MIS mixture (beta times
    // p.rr): sampling half the time from the BSDF divides its samples' weights by (1 - c),
    // which would keep beta high and let paths run to the depth cap.  Any survival
    // probability leaves the estimator unbiased.
    if (!done) {
      if (count < sc.max_path_nodes) {
        if (count > 5) {
          const float pr = fminf(0.9f, max3(beta) * (sc.guide ? p.rr[slot] : 1.f));
          if (rng.uniform() > pr) done = true;
          else beta = beta * (1.f / pr);
        }
      } else {
        done = true;
      }
    }
    if (!done) {
      const float3 wi = -dir;
      MTracker mt;
      if (MEDIA) mt = load_tracker(p.track[slot]);
      // Guided scattering at diffuse and microfacet surfaces.
      const bool guided = sc.guide && bounce < sc.guide_depth && !is_volume &&
                          (sc.materials[s.material].shader == TT_SHADER_DIFFUSE ||
                           sc.materials[s.material].shader == TT_SHADER_MICROFACET);
      if (guided) p.gnee[slot].w = 0.f;
      if (sc.sample_lights) {
        LightNode L = pick_light(sc, rng, l);
        if (L.type != LIGHT_NONE) {
          Eye eye;
          eye.is_camera = false;
          eye.is_volume = is_volume;
          eye.wi = wi;
          if (is_volume) {
            eye.pos = vpos;
            eye.med = &sc.media[medium];
            eye.sigma_s = xyz(vol);
          } else {
            eye.surf = s;
            eye.mat = &sc.materials[s.material];
          }
          Connection c = connect(sc, eye, L, l);
          if (c.valid) {
            MTracker smt;
            if (MEDIA) {
              // MaybeHandlePassageThroughSurface at the eye (rendering_randomwalk_impl.hxx:517-527).
              smt = mt;
              if (!is_volume && dot3(c.dir, s.n) < 0.f) going_through(sc, smt, c.dir, s.ng, s.material);
            }
            emit_shadow<MEDIA>(sc, p, bounce + 1, slot, c, L, beta, 1.f, -1, smt, rng, guided);
          }
        }
      }
      // At a guided vertex the network inputs are queued, and k_guide evaluates the network
      // and samples the mixture.
      if (guided) {
        const int qg = warp_append(guide_count(p, bounce));
        p.guide_q[qg] = slot;
        const float3 p01 = f3((s.pos.x - sc.box_lo[0]) * sc.box_inv[0], (s.pos.y - sc.box_lo[1]) * sc.box_inv[1],
                              (s.pos.z - sc.box_lo[2]) * sc.box_inv[2]);
        float4* gi = p.ginp + 3 * (size_t)qg;
        gi[0] = make_float4(p01.x, p01.y, p01.z, s.ns.x);
        gi[1] = make_float4(s.ns.y, s.ns.z, wi.x, wi.y);
        gi[2] = make_float4(wi.z, 0.f, 0.f, 0.f);
        p.beta[slot] = make_float4(beta.x, beta.y, beta.z, b4.w);
        meta.z = (unsigned)count;
        p.meta[slot] = meta;
        p.accum[slot] = make_float4(acc.x, acc.y, acc.z, 0.f);
        p.rng_state[slot] = rng.state;
        continue;
      }
      // Scatter: BSDF sample at a surface, phase-function sample at a volume vertex
      // (TakeRandomWalkStep from a scatter node).
      float3 ndir, bf, org;
      float pdf;
      bool delta;
      if (is_volume) {
        const DevMedium& M = sc.media[medium];
        float3 pval;
        ndir = medium_phase_sample(M, vpos, wi, rng, l, &pval, &pdf);
        // sigma_s x phase value / pdf; a single phase function's value is its pdf.
        bf = M.kind == TT_MEDIUM_ATMOSPHERE ? mul(xyz(vol), pval) * (1.f / pdf) : xyz(vol);
        delta = false;
        org = vpos;
      } else {
        const DevMaterial& m = sc.materials[s.material];
        ScatterSample ss = sample_bsdf(m, wi, s, rng, l);
        const float3 val = ss.value * (bsdf_correction(s, ss.dir) * fabsf(dot3(s.ng, ss.dir)));
        bf = val * (1.f / ss.pdf);
        pdf = ss.pdf;
        delta = ss.delta;
        ndir = ss.dir;
        org = s.pos + offset_at(s, ss.dir);
      }
      if (is_zero(bf) || !(pdf > 0.f)) {
        done = true;
      } else {
        beta = mul(beta, bf);
        if (MEDIA && !is_volume && dot3(ndir, s.n) < 0.f) {
          going_through(sc, mt, ndir, s.ng, s.material);
          p.track[slot] = store_tracker(mt);
        }
        p.ray_o[slot] = make_float4(org.x, org.y, org.z, 0.f);
        p.ray_d[slot] = make_float4(ndir.x, ndir.y, ndir.z, kLargeNumber);
        p.beta[slot] = make_float4(beta.x, beta.y, beta.z, pdf);
        meta.z = (unsigned)count;
        meta.w = delta ? 1u : 0u;
        p.meta[slot] = meta;
        const int qe = warp_append(ext_count(p, bounce + 1));
        p.ext_q[(bounce + 1) & 1][qe] = slot;
      }
    }
    p.accum[slot] = make_float4(acc.x, acc.y, acc.z, 0.f);
    p.rng_state[slot] = rng.state;
    if (done) {
      const int qd = warp_append(done_count(p, bounce + 1));
      p.done_q[qd] = slot;
    }
  }
}

// One guided vertex with network outputs `gout`: one-sample MIS of the BSDF and the learned
// vMF mixture, as SampleWithBinaryMixtureDensity (renderingalgorithms_pathtracing_guided.cxx:
// 474-524): with probability c the mixture is sampled, else the BSDF; the density is
// (1 - c) p_bsdf + c p_mixture either way.  NEE from the vertex gets its MIS weight against
// the same density (the reference's MaybeAddNeeLighting evaluates the same binary mixture,
// :1824-1840).  A reservoir of size one keeps one training record per path.
// Per-slot path state a guided vertex needs, loaded before the network runs so that the
// loads' latency overlaps the tensor-core work.
struct GuidePre {
  int slot;
  float rr;
  float4 h, d4, b4, nee;
  uint4 meta;
  unsigned long long rs, ri;
};

__device__ __forceinline__ GuidePre guide_prefetch(const PathState& p, int slot) {
  GuidePre g;
  g.slot = slot;
  g.h = p.hit[slot];
  g.d4 = p.ray_d[slot];
  g.b4 = p.beta[slot];
  g.nee = p.gnee[slot];
  g.rr = p.rr[slot];
  g.meta = p.meta[slot];
  g.rs = p.rng_state[slot];
  g.ri = p.rng_inc[slot];
  return g;
}

// One-sample MIS between the BSDF and a guiding distribution `dist` (sample(rng), pdf(x),
// and c, the probability of sampling it) at a queued guided vertex.
template <bool MEDIA, class Dist>
__device__ __forceinline__ void guide_scatter_dist(const DevScene& sc, const PathState& p, int bounce,
                                                   const GuidePre& pre, const Dist& dist) {
  const int slot = pre.slot;
  const float4 h = pre.h;
  const float3 dir = xyz(pre.d4);
  uint4 meta = pre.meta;
  const Lambda l = unpack_lambda(meta.y);
  const float4 b4 = pre.b4;
  float3 beta = xyz(b4);
  Rng rng{pre.rs, pre.ri};
  const int tri = __float_as_int(h.w);
  const bool sphere = sc.num_spheres > 0 && is_sphere_slot(sc.tris, tri);
  Surf s = sphere ? sphere_hit_surface(sc.tris, tri, xyz(p.ray_o[slot]), dir, h.x)
                  : make_surface(sc, tri, 1.f - h.y - h.z, h.y, h.z, f3(h.y, h.z, 1.f - h.y - h.z));
  orient(s, dir);
  const DevMaterial& m = sc.materials[s.material];
  const float3 wi = -dir;
  float3 ndir, val;
  float pb = 0.f;
  // An untrained network is not sampled: selection probability 0 gives plain BSDF sampling
  // with the BSDF density, while the records for the first training step are collected.
  const float c = sc.guide_cold ? 0.f : dist.c;
  if (rng.uniform() < c) {
    ndir = dist.sample(rng);
    val = eval_bsdf(m, wi, s, ndir, l, &pb);
  } else {
    const ScatterSample ss = sample_bsdf(m, wi, s, rng, l);
    ndir = ss.dir;
    val = ss.value;
    pb = ss.pdf;
  }
  const float pg = dist.pdf(ndir);
  const float pdf = (1.f - c) * pb + c * pg;
  const float4 nee = pre.nee;
  if (nee.w != 0.f) {
    const float3 sd = xyz(p.sh_d[slot]);
    const float pdf_due = ((1.f - c) * nee.z + c * dist.pdf(sd)) * nee.y;
    if (MEDIA) {
      p.sh_med[slot].y = pdf_due;
    } else if (nee.x > 0.f) {
      const float w = power_heuristic(nee.x, pdf_due);
      const float4 c4 = p.sh_c[slot];
      p.sh_c[slot] = make_float4(c4.x * w, c4.y * w, c4.z * w, c4.w);
    }
  }
  const float3 f = val * (bsdf_correction(s, ndir) * fabsf(dot3(s.ng, ndir)));
  const float3 bf = f * (1.f / pdf);
  const bool done = !(pdf > 0.f) || is_zero(bf) || !isfinite(bf.x + bf.y + bf.z);
  if (!done && sc.guide_record) {
    // Reservoir sampling over the path's guided vertices.
    float4* r = p.grec + (size_t)kRecF4 * slot;
    const float4 r3 = r[3];
    const int seen = (r3.w != 0.f ? __float_as_int(r3.z) : 0) + 1;
    const bool take = rng.uniform() * (float)seen < 1.f;
    if (take) {
      const float3 p01 = f3((s.pos.x - sc.box_lo[0]) * sc.box_inv[0], (s.pos.y - sc.box_lo[1]) * sc.box_inv[1],
                            (s.pos.z - sc.box_lo[2]) * sc.box_inv[2]);
      const float4 a = p.accum[slot];
      r[0] = make_float4(p01.x, p01.y, p01.z, s.ns.x);
      r[1] = make_float4(s.ns.y, s.ns.z, wi.x, wi.y);
      r[2] = make_float4(wi.z, ndir.x, ndir.y, ndir.z);
      r[3] = make_float4(pb, __int_as_float(bounce), __int_as_float(seen), 1.f);
      r[4] = make_float4(a.x, a.y, a.z, 0.f);
      r[5] = make_float4(beta.x, beta.y, beta.z, 0.f);
    } else {
      r[3] = make_float4(r3.x, r3.y, __int_as_float(seen), 1.f);
    }
  }
  if (done) {
    const int qd = warp_append(done_count(p, bounce + 1));
    p.done_q[qd] = slot;
  } else {
    beta = mul(beta, bf);
    if (MEDIA && dot3(ndir, s.n) < 0.f) {
      MTracker mt = load_tracker(p.track[slot]);
      going_through(sc, mt, ndir, s.ng, s.material);
      p.track[slot] = store_tracker(mt);
    }
    const float3 org = s.pos + offset_at(s, ndir);
    p.ray_o[slot] = make_float4(org.x, org.y, org.z, 0.f);
    p.ray_d[slot] = make_float4(ndir.x, ndir.y, ndir.z, kLargeNumber);
    p.beta[slot] = make_float4(beta.x, beta.y, beta.z, pdf);
    // Roulette throughput: the BSDF weight f / p_bsdf in place of f / pdf.
    if (pb > 0.f) p.rr[slot] = pre.rr * (pdf / pb);
    meta.w = 0u;
    p.meta[slot] = meta;
    const int qe = warp_append(ext_count(p, bounce + 1));
    p.ext_q[(bounce + 1) & 1][qe] = slot;
  }
  p.rng_state[slot] = rng.state;
}

// The learned or fitted vMF mixture as a guiding distribution.
struct MixDist {
  const GuideMixture& m;
  float c;
  __device__ __forceinline__ float3 sample(Rng& rng) const { return guide_mixture_sample(m, rng); }
  __device__ __forceinline__ float pdf(float3 x) const { return guide_mixture_pdf(m, x); }
};
template <bool MEDIA>
__device__ __forceinline__ void guide_scatter_mix(const DevScene& sc, const PathState& p, int bounce,
                                                  const GuidePre& pre, const GuideMixture& mix) {
  guide_scatter_dist<MEDIA>(sc, p, bounce, pre, MixDist{mix, mix.c});
}

template <bool MEDIA>
__device__ __forceinline__ void guide_scatter_one(const DevScene& sc, const PathState& p, int bounce,
                                                  const GuidePre& pre, const float* gout) {
  guide_scatter_mix<MEDIA>(sc, p, bounce, pre, guide_decode(gout));
}

// Cell of a normalised position in the tree guider's kd-tree (kdtree::Tree::Lookup,
// path_guiding_tree.hxx:129-150: left when the coordinate is below the split).
__device__ __forceinline__ int tree_cell(const DevScene& sc, float x, float y, float z) {
  int ref = sc.tree_root;
  for (int d = 0; d < 64 && ref >= 0; ++d) {
    const float4 nd = __ldg(&sc.tree_nodes[ref]);
    const int axis = __float_as_int(nd.y);
    const float c = axis == 0 ? x : (axis == 1 ? y : z);
    ref = __float_as_int(c < nd.x ? nd.z : nd.w);
  }
  return ref < 0 ? ~ref : 0;
}

// Quadtree distribution of a cell (layout in tt_quadtree.h): hierarchical warping of two
// uniforms down the tree (quadtree::Sample, path_guiding_quadtree.cxx:178-244, after
// Clarberg et al. 2005, section 5.1: at every node the column is chosen by the first
// uniform against the left and right sums of the children's weights and the row by the
// second against the chosen column's bottom and top weights, each uniform rescaled to the
// chosen part), then a point uniform in the leaf's square, mapped to the sphere with
// u = phi / 2 pi + 1/2, v = (z + 1) / 2.  Density per solid angle: leaf weight / (root
// weight x leaf area) / 4 pi.  At most kQuadMaxDepth levels; the loop stops at 16.
__device__ __forceinline__ float3 quad_square_to_dir(float u, float v) {
  const float z = 2.f * v - 1.f;
  const float rho = sqrtf(fmaxf(0.f, 1.f - z * z));
  float sn, cs;
  sincospif(2.f * u - 1.f, &sn, &cs);
  return f3(rho * cs, rho * sn, z);
}
__device__ __forceinline__ float3 quad_sample(const int4* __restrict__ child, const float* __restrict__ prob, int root,
                                              float u0, float u1, float* pdf) {
  constexpr float kLt1 = 0.99999994f;  // the largest float below 1
  constexpr float kEpsF = 1.1920929e-07f;
  u0 = fminf(u0, kLt1);
  u1 = fminf(u1, kLt1);
  float lo0 = 0.f, lo1 = 0.f, hi0 = 1.f, hi1 = 1.f;
  int node = root;
  for (int d = 0; d < 16; ++d) {
    const int4 c = __ldg(&child[node]);
    if (c.x < 0) break;
    const float w0 = __ldg(&prob[c.x]), w1 = __ldg(&prob[c.y]), w2 = __ldg(&prob[c.z]), w3 = __ldg(&prob[c.w]);
    const float wl = w0 + w2, wr = w1 + w3;
    const float s0 = u0 * (wl + wr);
    int q = s0 < wl ? 0 : 1;
    u0 = s0 < wl ? s0 / (wl + kEpsF) : (s0 - wl) / (wr + kEpsF);
    const float wb = q ? w1 : w0, wt = q ? w3 : w2;
    const float s1 = u1 * (wb + wt);
    q |= s1 < wb ? 0 : 2;
    u1 = s1 < wb ? s1 / (wb + kEpsF) : (s1 - wb) / (wt + kEpsF);
    u0 = fminf(u0, kLt1);
    u1 = fminf(u1, kLt1);
    const float c0 = 0.5f * (lo0 + hi0), c1 = 0.5f * (lo1 + hi1);
    if (q & 1) lo0 = c0; else hi0 = c0;
    if (q & 2) lo1 = c1; else hi1 = c1;
    node = q == 0 ? c.x : (q == 1 ? c.y : (q == 2 ? c.z : c.w));
  }
  const float a0 = hi0 - lo0, a1 = hi1 - lo1;
  *pdf = __ldg(&prob[node]) / (__ldg(&prob[root]) * a0 * a1) * (1.f / (4.f * kPi));
  const float pu = fmaxf(fminf(a0 * u0 + lo0, hi0 * kLt1), lo0);
  const float pv = fmaxf(fminf(a1 * u1 + lo1, hi1 * kLt1), lo1);
  return quad_square_to_dir(pu, pv);
}
__device__ __forceinline__ float quad_pdf(const int4* __restrict__ child, const float* __restrict__ prob, int root,
                                          float3 x) {
  const float u = (atan2f(x.y, x.x) * (1.f / kPi) + 1.f) * 0.5f, v = (x.z + 1.f) * 0.5f;
  float lo0 = 0.f, lo1 = 0.f, hi0 = 1.f, hi1 = 1.f;
  int node = root;
  for (int d = 0; d < 16; ++d) {
    const int4 c = __ldg(&child[node]);
    if (c.x < 0) break;
    const float c0 = 0.5f * (lo0 + hi0), c1 = 0.5f * (lo1 + hi1);
    const int q = (u < c0 ? 0 : 1) | (v < c1 ? 0 : 2);
    if (q & 1) lo0 = c0; else hi0 = c0;
    if (q & 2) lo1 = c1; else hi1 = c1;
    node = q == 0 ? c.x : (q == 1 ? c.y : (q == 2 ? c.z : c.w));
  }
  return __ldg(&prob[node]) / (__ldg(&prob[root]) * (hi0 - lo0) * (hi1 - lo1)) * (1.f / (4.f * kPi));
}
// A cell's quadtree as a guiding distribution (c = 0: not sampled, when the tree carries no
// weight).
struct QuadGuide {
  const int4* child;
  const float* prob;
  int root;
  float c;
  __device__ __forceinline__ float3 sample(Rng& rng) const {
    const float u0 = rng.uniform(), u1 = rng.uniform();
    float pdf;
    return quad_sample(child, prob, root, u0, u1, &pdf);
  }
  __device__ __forceinline__ float pdf(float3 x) const { return quad_pdf(child, prob, root, x); }
};

// Tree-guided scattering: the cell's fitted distribution (vMF mixture or quadtree) against
// the BSDF by the same one-sample MIS, the distribution chosen with probability 0.5
// (PROB_BSDF, renderingalgorithms_pathtracing_guided.cxx:470).
template <bool MEDIA>
__global__ void __launch_bounds__(256) k_guide_tree(DevScene sc, PathState p, int bounce) {
  const int n = *guide_count(p, bounce);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const GuidePre pre = guide_prefetch(p, p.guide_q[i]);
    const float4 a = p.ginp[3 * (size_t)i];
    const int cell = tree_cell(sc, a.x, a.y, a.z);
    if (sc.tree_quad) {
      const int root = __ldg(&sc.tree_qroot[cell]);
      const float w = __ldg(&sc.tree_qprob[root]);
      guide_scatter_dist<MEDIA>(sc, p, bounce, pre,
                                QuadGuide{sc.tree_qchild, sc.tree_qprob, root, (w > 0.f && isfinite(w)) ? 0.5f : 0.f});
      continue;
    }
    const float* cm = sc.tree_mix + 40 * (size_t)cell;
    GuideMixture mix;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
      mix.w[k] = __ldg(&cm[k]);
      mix.mu[k] = f3(__ldg(&cm[8 + 3 * k]), __ldg(&cm[9 + 3 * k]), __ldg(&cm[10 + 3 * k]));
      mix.kappa[k] = __ldg(&cm[32 + k]);
    }
    mix.c = 0.5f;
    guide_scatter_mix<MEDIA>(sc, p, bounce, pre, mix);
  }
}

// Guided scattering of the vertices k_shade queued this bounce: a persistent kernel whose
// warps take 32 queue entries at a time, evaluate the network on them (two 16-row tiles
// with the weights in shared memory, guide_mlp_tile) and then scatter one entry per lane.
constexpr int kGuideWarps = 8;
constexpr int kGuideSmem = kGSmBytes + kGuideWarps * 32 * (kGInputs + kGOutStride) * 4;

template <bool MEDIA>
__global__ void __launch_bounds__(kGuideWarps * 32) k_guide(DevScene sc, PathState p, int bounce) {
  extern __shared__ __align__(16) unsigned char gsm[];
  __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(gsm);
  float* sb = reinterpret_cast<float*>(gsm + kGSmW * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* q = reinterpret_cast<float*>(gsm + kGSmBytes) + warp * 32 * kGInputs;
  float* o = reinterpret_cast<float*>(gsm + kGSmBytes) + kGuideWarps * 32 * kGInputs + warp * 32 * kGOutStride;
  const int n = *guide_count(p, bounce);
  if (blockIdx.x * kGuideWarps * 32 >= n) return;
  guide_smem_load(sc.guide_w16, sc.guide_w32, sw, sb);
  __syncthreads();
  for (int base = (blockIdx.x * kGuideWarps + warp) * 32; base < n; base += gridDim.x * kGuideWarps * 32) {
    const int i = base + lane;
    float* r = q + lane * kGInputs;
    GuidePre pre;
    if (i < n) pre = guide_prefetch(p, p.guide_q[i]);
    if (i < n) {
      const float4* gi = p.ginp + 3 * (size_t)i;
      const float4 a = gi[0], b = gi[1], c = gi[2];
      r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w; r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w; r[8] = c.x;
    } else {
#pragma unroll
      for (int k = 0; k < kGInputs; ++k) r[k] = 0.f;
    }
    __syncwarp();
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
      uint32_t xf[6][4];
      guide_tile_features(q + mt * 16 * kGInputs, kGInputs, xf);
      guide_mlp_tile(sw, sb, xf, o + mt * 16 * kGOutStride, kGOutStride, nullptr);
    }
    __syncwarp();
    if (i < n) guide_scatter_one<MEDIA>(sc, p, bounce, pre, o + lane * kGOutStride);
    __syncwarp();
  }
}

// The same on the tcgen05 tensor cores (tt_guide_tc.cuh): each CTA runs kTcChains chains of
// 128 queue entries; a thread encodes its entry's features into the chain's tile, the chain
// runs the network with the accumulators in tensor memory, and each thread then decodes its
// row's outputs and scatters its entry.
template <bool MEDIA>
__global__ void __launch_bounds__(kTcThreads) k_guide_tc(DevScene sc, PathState p, int bounce) {
  extern __shared__ __align__(128) unsigned char tsm[];
  const int n = *guide_count(p, bounce);
  if ((long long)blockIdx.x * kTcThreads >= n) return;  // uniform over the CTA
  const TcChain c = tc_setup(tsm);
  tc_load_weights(sc.guide_w16, sc.guide_w32, tsm);
  __syncthreads();
  uint32_t phase = 0;
  bool ok = true;
  const int g = threadIdx.x / kTcRows;
  for (int base = (blockIdx.x * kTcChains + g) * kTcRows; base < n; base += gridDim.x * kTcThreads) {
    const int i = base + c.row;
    GuidePre pre;
    float q[kGInputs];
    if (i < n) {
      pre = guide_prefetch(p, p.guide_q[i]);
      const float4* gi = p.ginp + 3 * (size_t)i;
      const float4 a = gi[0], b = gi[1], d = gi[2];
      q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = a.w; q[4] = b.x; q[5] = b.y; q[6] = b.z; q[7] = b.w; q[8] = d.x;
    } else {
#pragma unroll
      for (int k = 0; k < kGInputs; ++k) q[k] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < kGIn; k += 8)
      *reinterpret_cast<uint4*>(tsm + c.xo + tc_off(c.row, k, kGIn)) =
          make_uint4(guide_feature_pair(q, k), guide_feature_pair(q, k + 2), guide_feature_pair(q, k + 4),
                     guide_feature_pair(q, k + 6));
    if (!tc_mlp_tile(tsm, c, phase)) {  // the same on every thread of the chain
      ok = false;
      break;
    }
    float o[kGOut];
#pragma unroll
    for (int k = 0; k < kGOut / 4; ++k) {
      const float4 v = *tc_out_slot(tsm, c.xo, c.row, k);
      o[4 * k] = v.x; o[4 * k + 1] = v.y; o[4 * k + 2] = v.z; o[4 * k + 3] = v.w;
    }
    tc_chain_sync(c);  // the outputs are read out before the next entries' features land there
    if (i < n) guide_scatter_one<MEDIA>(sc, p, bounce, pre, o);
  }
  if (!ok) {
    atomicOr(p.err, ERR_TENSOR);
    tc_drain(c, phase);
  }
  tc_teardown(tsm);
}

// Occlusion test of the queued shadow rays.  Unoccluded rays add their contribution to
// the path (or, for camera-vertex samples, splat it to the pixel they project to).  In
// media scenes the contribution is multiplied by the transmittance through the media
// between the medium-boundary crossings (TransmittanceEstimate, rendering_util.cxx:40-67)
// and by the MIS weight that the segment's transmittance pdf factor completes.
template <bool MEDIA, bool COUNT, bool SPH, bool WIDE>
__global__ void __launch_bounds__(256) k_shadow(DevScene sc, PathState p, Framebuffer fb, int bounce,
                                                unsigned long long* counters) {
  const int n = *sh_count(p, bounce);
  TraceCounters cnt{0u, 0u};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = p.sh_q[i];
    const float4 o = p.sh_o[slot], d = p.sh_d[slot];
    const RayPre r = prepare_ray(xyz(o), xyz(d));
    float t, b1, b2;
    const int hit = trace<true, COUNT, SPH, WIDE>(sc, r, 0.f, o.w, &t, &b1, &b2, p.err, &cnt);
    if (hit >= 0) continue;
    const float4 c4 = p.sh_c[slot];
    float3 c = xyz(c4);
    const int target = __float_as_int(d.w);
    if (MEDIA) {
      const Lambda l = unpack_lambda(p.meta[slot].y);
      MTracker mt = load_tracker(p.sh_track[slot]);
      const float4 med = p.sh_med[slot];
      Rng srng;
      srng.seed_path(((unsigned long long)__float_as_uint(med.w) << 32) | __float_as_uint(med.z), p.rng_inc[slot]);
      float3 T = f3(1.f, 1.f, 1.f);
      float ctr = 1.f, snear = 0.f;
      for (int k = 0;; ++k) {
        float tc;
        const int cs = next_crossing<SPH, WIDE>(sc, r, snear, o.w, &tc, p.err);
        const float sfar = cs >= 0 ? tc : o.w;
        if (mt.cur >= 0) {
          const DevMedium& M = sc.media[mt.cur];
          const float3 sorg = xyz(o) + xyz(d) * snear;
          ctr *= medium_segment_tr(M, sorg, xyz(d), sfar - snear, l);
          T = mul(T, medium_transmission(M, sorg, xyz(d), sfar - snear, srng, l, p.err));
        }
        if (cs < 0) break;
        if (k >= kMaxCrossings) {
          atomicOr(p.err, ERR_CROSSINGS);
          T = f3(0.f, 0.f, 0.f);
          break;
        }
        float3 ng;
        int mat;
        crossing_info(sc.vtris, cs, xyz(o), xyz(d), sfar, &ng, &mat);
        going_through(sc, mt, xyz(d), ng, mat);
        snear = sfar;
      }
      const float mis = med.x < 0.f ? 1.f : power_heuristic(med.x, med.y * ctr);
      c = mul(c, T) * mis;
    }
    if (target < 0) {
      const float4 a = p.accum[slot];
      p.accum[slot] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, 0.f);
      if (sc.guide_record) {
        // Direct light at the recorded vertex is not radiance along its sampled direction.
        const float4 r3 = p.grec[(size_t)kRecF4 * slot + 3];
        if (r3.w != 0.f && __float_as_int(r3.y) == bounce - 1) {
          const float4 r4 = p.grec[(size_t)kRecF4 * slot + 4];
          p.grec[(size_t)kRecF4 * slot + 4] = make_float4(r4.x + c.x, r4.y + c.y, r4.z + c.z, 0.f);
        }
      }
    } else {
      const Lambda l = unpack_lambda(p.meta[slot].y);
      const float3 rgb = selection_to_rgb(c, l);
      atomicAdd(&fb.light[3 * target], rgb.x);
      atomicAdd(&fb.light[3 * target + 1], rgb.y);
      atomicAdd(&fb.light[3 * target + 2], rgb.z);
    }
  }
  if (COUNT) {
    atomicAdd(&counters[0], (unsigned long long)cnt.nodes);
    atomicAdd(&counters[1], (unsigned long long)cnt.tris);
  }
}

// MediumTracker::initializePosition (rendering_util.cxx:13-38): walks a ray from outside
// the scene bounds (+x side) to `pos` through every medium boundary, then every surface,
// updating the tracker at each crossing.  One thread.
__global__ void k_init_tracker(DevScene sc, float3 pos, float3 lo, float3 hi, uint2* out, unsigned int* err) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  MTracker mt{0xffffffffu, -1};
  const bool inside = pos.x >= lo.x && pos.x <= hi.x && pos.y >= lo.y && pos.y <= hi.y && pos.z >= lo.z &&
                      pos.z <= hi.z;
  if (inside) {
    const float go = 2.f * fmaxf(hi.x - lo.x, fmaxf(hi.y - lo.y, hi.z - lo.z));
    const float3 dir = f3(-1.f, 0.f, 0.f);
    const RayPre r = prepare_ray(f3(pos.x + go, pos.y, pos.z), dir);
    for (int pass = 0; pass < 2; ++pass) {
      const BvhRef bvh = pass == 0 ? volume_bvh(sc) : surface_bvh(sc);
      const uint4* nodes8 = pass == 0 ? sc.vnodes8 : sc.nodes8;
      float t = 0.f;
      for (int k = 0; k < kMaxCrossings; ++k) {
        float tc;
        const int slot = sc.wide ? next_hit8<true>(nodes8, bvh.tris, r, t, go, &tc, err)
                                 : next_hit<true>(bvh, r, t, go, &tc, err);
        if (slot < 0) break;
        float3 ng;
        int mat;
        crossing_info(bvh.tris, slot, r.o, dir, tc, &ng, &mat);
        going_through(sc, mt, dir, ng, mat);
        t = tc;
      }
    }
  }
  out[0] = store_tracker(mt);
}

__global__ void __launch_bounds__(256) k_flush(DevScene sc, PathState p, Framebuffer fb, int bounce) {
  const int n = *done_count(p, bounce);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = p.done_q[i];
    const uint4 meta = p.meta[slot];
    if (sc.guide_record) {
      // Commit the path's pending record if it carries light (a record with F = 0 adds
      // nothing to the loss or its gradient), kept with probability guide_keep: F / q =
      // (contribution after the vertex) / (throughput before it), averaged over the
      // wavelengths with nonzero throughput.  The pool is a ring: the oldest records give way.
      const float4* r = p.grec + (size_t)kRecF4 * slot;
      const float4 r3 = r[3];
      Rng krng{p.rng_state[slot], p.rng_inc[slot]};
      if (r3.w != 0.f && (sc.guide_keep >= 1.f || krng.uniform() < sc.guide_keep)) {
        const float4 r0 = r[0], r1 = r[1], r2 = r[2], r4 = r[4], r5 = r[5];
        const float4 a = p.accum[slot];
        float fq = 0.f;
        int nz = 0;
        const float da[3] = {a.x - r4.x, a.y - r4.y, a.z - r4.z}, bb[3] = {r5.x, r5.y, r5.z};
        for (int k = 0; k < 3; ++k)
          if (bb[k] > 0.f) {
            fq += fmaxf(da[k], 0.f) / bb[k];
            ++nz;
          }
        fq = nz > 0 ? fq / nz : 0.f;
        if (fq > 0.f && isfinite(fq)) {
          const unsigned idx = atomicAdd(reinterpret_cast<unsigned*>(p.rec_count), 1u) % (unsigned)p.rec_cap;
          GuideRecord rec;
          rec.pos[0] = r0.x; rec.pos[1] = r0.y; rec.pos[2] = r0.z;
          rec.n[0] = r0.w; rec.n[1] = r1.x; rec.n[2] = r1.y;
          rec.wo[0] = r1.z; rec.wo[1] = r1.w; rec.wo[2] = r2.x;
          rec.wi[0] = r2.y; rec.wi[1] = r2.z; rec.wi[2] = r2.w;
          rec.p_bsdf = r3.x;
          rec.f_over_q = fq;
          p.records[idx] = rec;
        }
      }
    }
    const float3 rgb = selection_to_rgb(xyz(p.accum[slot]), unpack_lambda(meta.y));
    const int px = (int)meta.x;
    atomicAdd(&fb.accum[3 * px], rgb.x);
    atomicAdd(&fb.accum[3 * px + 1], rgb.y);
    atomicAdd(&fb.accum[3 * px + 2], rgb.z);
  }
}

__global__ void __launch_bounds__(256) k_gather(PathState p, Framebuffer fb, WaveArgs w) {
  const int off = (int)(w.wave_start % w.npix_range);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < w.npix_range; j += gridDim.x * blockDim.x) {
    // Slot i holds pixel (wave_start + i) mod npix_range.
    int i = j - off;
    if (i < 0) i += w.npix_range;
    float3 sum = f3(0.f, 0.f, 0.f);
    for (; i < w.wave_paths; i += w.npix_range)
      sum = sum + selection_to_rgb(xyz(p.accum[i]), unpack_lambda(p.meta[i].y));
    float* a = fb.accum + 3 * (size_t)(w.pixel_begin + j);
    a[0] += sum.x;
    a[1] += sum.y;
    a[2] += sum.z;
  }
}

__global__ void k_accumulate(Framebuffer fb, double* acc, double* light, int n3) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    acc[i] += (double)fb.accum[i];
    light[i] += (double)fb.light[i];
    fb.accum[i] = 0.f;
    fb.light[i] = 0.f;
  }
}

// ----------------------------------------------------------------------------------------
// Batch queries and shader sampling for the parity tests.
template <bool SPH, bool WIDE>
__global__ void k_intersect_rays(DevScene sc, const float* rays, int n, int* prim, float* t, float* u, float* v,
                                 unsigned int* err) {
  TraceCounters cnt{0u, 0u};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* r = rays + 8 * (size_t)i;
    const RayPre rp = prepare_ray(f3(r[0], r[1], r[2]), f3(r[4], r[5], r[6]));
    float tt = -1.f, b1 = 0.f, b2 = 0.f;
    const int slot = trace<false, false, SPH, WIDE>(sc, rp, r[3], r[7], &tt, &b1, &b2, err, &cnt);
    prim[i] = slot >= 0 ? __float_as_int(__ldg(&sc.tris[3 * slot]).w) : -1;
    t[i] = slot >= 0 ? tt : -1.f;
    u[i] = b1;
    v[i] = b2;
  }
}

template <bool SPH, bool WIDE>
__global__ void k_occluded_rays(DevScene sc, const float* rays, int n, unsigned char* occ, unsigned int* err) {
  TraceCounters cnt{0u, 0u};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* r = rays + 8 * (size_t)i;
    const RayPre rp = prepare_ray(f3(r[0], r[1], r[2]), f3(r[4], r[5], r[6]));
    float tt, b1, b2;
    occ[i] = trace<true, false, SPH, WIDE>(sc, rp, r[3], r[7], &tt, &b1, &b2, err, &cnt) >= 0 ? 1 : 0;
  }
}

template <bool SPH, bool WIDE>
__global__ void k_count_rays(DevScene sc, const float* rays, int n, unsigned long long* counters,
                             unsigned int* err) {
  TraceCounters cnt{0u, 0u};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* r = rays + 8 * (size_t)i;
    const RayPre rp = prepare_ray(f3(r[0], r[1], r[2]), f3(r[4], r[5], r[6]));
    float tt, b1, b2;
    trace<false, true, SPH, WIDE>(sc, rp, r[3], r[7], &tt, &b1, &b2, err, &cnt);
  }
  atomicAdd(&counters[0], (unsigned long long)cnt.nodes);
  atomicAdd(&counters[1], (unsigned long long)cnt.tris);
}

__device__ __forceinline__ Surf zup_surface(float3 wi) {
  Surf s;
  s.prim = 0;
  s.material = 0;
  s.pos = f3(0.f, 0.f, 0.f);
  s.ng = f3(0.f, 0.f, 1.f);
  s.ns_raw = s.ng;
  s.bounds = f3(0.f, 0.f, 0.f);
  s.uv = make_float2(0.f, 0.f);
  orient(s, -wi);
  return s;
}

__global__ void k_sample_bsdf(DevScene sc, int material, float3 wi, int3 li, int n, unsigned long long seed,
                              float* dir, float* val, float* pdf) {
  const Lambda l{li.x, li.y, li.z};
  const Surf s = zup_surface(wi);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Rng rng;
    rng.seed_path(seed, (unsigned long long)i);
    ScatterSample ss = sample_bsdf(sc.materials[material], wi, s, rng, l);
    dir[3 * i] = ss.dir.x; dir[3 * i + 1] = ss.dir.y; dir[3 * i + 2] = ss.dir.z;
    val[3 * i] = ss.value.x; val[3 * i + 1] = ss.value.y; val[3 * i + 2] = ss.value.z;
    pdf[i] = ss.delta ? -ss.pdf : ss.pdf;
  }
}

__global__ void k_eval_bsdf(DevScene sc, int material, float3 wi, int3 li, const float* dirs, int n, float* val,
                            float* pdf) {
  const Lambda l{li.x, li.y, li.z};
  const Surf s = zup_surface(wi);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float pp = 0.f;
    const float3 v = eval_bsdf(sc.materials[material], wi, s, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]), l, &pp);
    val[3 * i] = v.x; val[3 * i + 1] = v.y; val[3 * i + 2] = v.z;
    pdf[i] = pp;
  }
}

// Phase-function sampling and evaluation at a volume vertex at pos in medium `medium`
// (the sampling-test hooks of the PhaseFunctionTests fixture, tests_sampling.cxx:1202-1259):
// sample i draws from the PCG32 stream (seed, i), as the render kernels do per path.
__global__ void k_sample_phase(DevScene sc, int medium, float3 pos, float3 wi, int3 li, int n, unsigned long long seed,
                               float* dir, float* val, float* pdf) {
  const Lambda l{li.x, li.y, li.z};
  const DevMedium& m = sc.media[medium];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Rng rng;
    rng.seed_path(seed, (unsigned long long)i);
    float3 v;
    float pp;
    const float3 d = medium_phase_sample(m, pos, wi, rng, l, &v, &pp);
    dir[3 * i] = d.x; dir[3 * i + 1] = d.y; dir[3 * i + 2] = d.z;
    val[3 * i] = v.x; val[3 * i + 1] = v.y; val[3 * i + 2] = v.z;
    pdf[i] = pp;
  }
}

__global__ void k_eval_phase(DevScene sc, int medium, float3 pos, float3 wi, int3 li, const float* dirs, int n,
                             float* val, float* pdf) {
  const Lambda l{li.x, li.y, li.z};
  const DevMedium& m = sc.media[medium];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float pp = 0.f;
    const float3 v = medium_phase_eval(m, pos, wi, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]), l, &pp);
    val[3 * i] = v.x; val[3 * i + 1] = v.y; val[3 * i + 2] = v.z;
    pdf[i] = pp;
  }
}

// ----------------------------------------------------------------------------------------
// Host launchers.


void upload_constant_tables() {
  float m[3][NBINS], smits[7][NBINS];
  for (int i = 0; i < 3; ++i)
    for (int b = 0; b < NBINS; ++b) m[i][b] = (float)kSpectrumToRgb[i][b];
  for (int i = 0; i < 7; ++i)
    for (int b = 0; b < NBINS; ++b) smits[i][b] = (float)kSmitsBasis[i][b];
  cudaMemcpyToSymbol(c_spec_to_rgb, m, sizeof(m));
  cudaMemcpyToSymbol(c_smits, smits, sizeof(smits));
}

#include "tt_pt2.cuh"

constexpr int kBlock = 256;

// Calls f with std::integral_constant<bool, b>: picks a kernel instantiation at run time.
template <class F>
static void with_bool(bool b, F&& f) {
  if (b) f(std::true_type{});
  else f(std::false_type{});
}

// Launch grids depend on the device's SM count, so they are cached per device ordinal
// (the current device of the calling thread).  Concurrent first calls compute the same value.
constexpr int kGridCacheDevices = 64;
static int current_device_slot() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev >= 0 && dev < kGridCacheDevices ? dev : kGridCacheDevices - 1;
}

// Threads per block of the wavefront launches: the autotuner's choice (128 or 256), else
// kBlock.  Every wavefront kernel loops grid-stride and takes any size up to kBlock.
static int blk(const DevScene& s) { return (s.block > 0 && s.block <= kBlock && kBlock % s.block == 0) ? s.block : kBlock; }

// Blocks of `fn` that stay resident on one SM at `block` threads, cached per device,
// kernel and block size (a short list under a mutex; the first launch of each kernel pays
// one occupancy query).
static int resident_blocks(const void* fn, int block) {
  struct Entry {
    const void* fn;
    int dev, block, blocks;
  };
  static std::mutex mu;
  static Entry cache[512];
  static int used = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < used; ++i)
    if (cache[i].fn == fn && cache[i].dev == dev && cache[i].block == block) return cache[i].blocks;
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, block, 0);
  if (b < 1) b = 1;
  if (used < 512) cache[used++] = Entry{fn, dev, block, b};
  return b;
}
static int sm_count() {
  static int g[kGridCacheDevices] = {};
  int& gg = g[current_device_slot()];
  if (gg == 0) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    gg = sms > 0 ? sms : 1;
  }
  return gg;
}
// Grid of a grid-stride wavefront launch: every SM filled to the launched kernel's own
// occupancy limit (traversal kernels).  A kernel whose variants differ in registers (the
// sphere and media instantiations) would otherwise get a grid sized for another variant
// and run a last partial round of blocks on a third of the SMs' slots.
template <class K>
static int full_grid(K* kernel, int block) {
  return sm_count() * resident_blocks(reinterpret_cast<const void*>(kernel), block);
}
// A requested grid (the context's default or the autotuner's choice) cut down to whole
// rounds of resident blocks of this kernel: no partial last round.
template <class K>
static int fit_grid(K* kernel, int grid, int block) {
  const int cap = full_grid(kernel, block);
  return grid > cap ? grid / cap * cap : grid;
}

void launch_generate(const DevScene& s, const PathState& p, const Framebuffer& fb, const WaveArgs& w, int grid,
                     cudaStream_t st) {
  const int b = blk(s);
  if (s.num_media > 0) k_generate<true><<<fit_grid(k_generate<true>, grid, b), b, 0, st>>>(s, p, fb, w);
  else k_generate<false><<<fit_grid(k_generate<false>, grid, b), b, 0, st>>>(s, p, fb, w);
}
void launch_extend(const DevScene& s, const PathState& p, int bounce, bool count, unsigned long long* stats, int grid,
                   cudaStream_t st) {
  (void)grid;
  const int b = blk(s);
  with_bool(count, [&](auto C) {
    with_bool(s.num_spheres > 0, [&](auto S) {
      with_bool(s.wide != 0, [&](auto W) {
        auto* k = k_extend<decltype(C)::value, decltype(S)::value, decltype(W)::value>;
        k<<<full_grid(k, b), b, 0, st>>>(s, p, bounce, stats);
      });
    });
  });
}
int shade_launches(const DevScene& s, const PathState& p, int bounce) {
  if (s.algo != TT_ALGO_PT || !sorted_bounce(s, p, bounce)) return 1;
  return s.num_media > 0 ? 3 : 2;  // without media k_extend keys and counts the hits
}
void launch_shade(const DevScene& s, const PathState& p, int bounce, int grid, cudaStream_t st) {
  const int b = blk(s);
  if (s.algo == TT_ALGO_PT && sorted_bounce(s, p, bounce)) {
    if (s.num_media > 0) k_sort_count<<<fit_grid(k_sort_count, grid, b), b, 0, st>>>(s, p, bounce);
    k_sort_scatter<<<fit_grid(k_sort_scatter, grid, b), b, 0, st>>>(p, bounce);
  }
  if (s.algo == TT_ALGO_PT2) {
    if (s.num_media == 0) {
      auto* k = k_shade2<false, false, false>;
      k<<<fit_grid(k, grid, b), b, 0, st>>>(s, p, bounce);
      return;
    }
    with_bool(s.num_spheres > 0, [&](auto S) {
      with_bool(s.wide != 0, [&](auto W) {
        auto* k = k_shade2<true, decltype(S)::value, decltype(W)::value>;
        k<<<fit_grid(k, grid, b), b, 0, st>>>(s, p, bounce);
      });
    });
    return;
  }
  if (s.num_media > 0) k_shade<true><<<fit_grid(k_shade<true>, grid, b), b, 0, st>>>(s, p, bounce);
  else k_shade<false><<<fit_grid(k_shade<false>, grid, b), b, 0, st>>>(s, p, bounce);
}
void launch_shadow(const DevScene& s, const PathState& p, const Framebuffer& fb, int bounce, bool count,
                   unsigned long long* stats, int grid, cudaStream_t st) {
  (void)grid;
  const int b = blk(s);
  if (s.algo == TT_ALGO_PT2 && s.num_media > 0) {
    with_bool(s.num_spheres > 0, [&](auto S) {
      with_bool(s.wide != 0, [&](auto W) {
        auto* k = k_shadow2<decltype(S)::value, decltype(W)::value>;
        k<<<full_grid(k, b), b, 0, st>>>(s, p, bounce);
      });
    });
    return;
  }
  // Media, sphere and layout variants are instantiated separately so that the surface-only,
  // triangle-only traversal stays lean for mesh scenes.
  with_bool(s.num_media > 0, [&](auto M) {
    with_bool(count, [&](auto C) {
      with_bool(s.num_spheres > 0, [&](auto S) {
        with_bool(s.wide != 0, [&](auto W) {
          auto* k = k_shadow<decltype(M)::value, decltype(C)::value, decltype(S)::value, decltype(W)::value>;
          k<<<full_grid(k, b), b, 0, st>>>(s, p, fb, bounce, stats);
        });
      });
    });
  });
}
void launch_track(const DevScene& s, const PathState& p, int bounce, int grid, cudaStream_t st) {
  if (s.algo == TT_ALGO_PT2) return;  // the null-path tracer tracks inside its shade stage
  with_bool(s.num_spheres > 0, [&](auto S) {
    with_bool(s.wide != 0, [&](auto W) {
      auto* k = k_track<decltype(S)::value, decltype(W)::value>;
      k<<<fit_grid(k, grid, blk(s)), blk(s), 0, st>>>(s, p, bounce);
    });
  });
}
void launch_init_tracker(const DevScene& s, float3 pos, float3 bb_lo, float3 bb_hi, uint2* out, unsigned int* err,
                         cudaStream_t st) {
  k_init_tracker<<<1, 32, 0, st>>>(s, pos, bb_lo, bb_hi, out, err);
}
void launch_flush(const DevScene& s, const PathState& p, const Framebuffer& fb, int bounce, int grid,
                  cudaStream_t st) {
  k_flush<<<fit_grid(k_flush, grid, blk(s)), blk(s), 0, st>>>(s, p, fb, bounce);
}

void launch_gather(const DevScene& s, const PathState& p, const Framebuffer& fb, const WaveArgs& w, int grid,
                   cudaStream_t st) {
  k_gather<<<fit_grid(k_gather, grid, 256), 256, 0, st>>>(p, fb, w);
}

void launch_generate_views(const DevScene& s, const PathState& p, const ViewWave* waves, const int* wave_idx,
                           const DevView* views, int nviews, int grid, cudaStream_t st) {
  const int b = blk(s);
  if (s.num_media > 0)
    k_generate_views<true><<<fit_grid(k_generate_views<true>, grid, b), b, 0, st>>>(s, p, waves, wave_idx, views, nviews);
  else
    k_generate_views<false><<<fit_grid(k_generate_views<false>, grid, b), b, 0, st>>>(s, p, waves, wave_idx, views, nviews);
}

void launch_wave_advance(int* wave_idx, cudaStream_t st) { k_wave_advance<<<1, 32, 0, st>>>(wave_idx); }

void launch_resolve_views(const float* accum, const float* light, const DevView* views, int nviews, int npix,
                          float* rgb, cudaStream_t st) {
  const int grid = std::max(1, std::min(65535, (npix + 255) / 256));
  k_resolve_views<<<grid, 256, 0, st>>>(accum, light, views, nviews, npix, rgb);
}

// Grids of the guided-scattering kernels, per device: [0] k_guide, [1] k_guide_tc, [2] k_guide_tree.
static int g_guide_grids[kGridCacheDevices][3] = {};

void prepare_guide_launch() {
  int* grids = g_guide_grids[current_device_slot()];
  if (grids[0] != 0) return;
  cudaFuncSetAttribute(k_guide<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGuideSmem);
  cudaFuncSetAttribute(k_guide<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGuideSmem);
  cudaFuncSetAttribute(k_guide_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  cudaFuncSetAttribute(k_guide_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_guide_tc<true>, kTcThreads, kTcSmem);
  grids[1] = sms * (per_sm > 0 ? per_sm : 1);
  per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_guide_tree<true>, kBlock, 0);
  grids[2] = sms * (per_sm > 0 ? per_sm : 1);
  per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_guide<true>, kGuideWarps * 32, kGuideSmem);
  grids[0] = sms * (per_sm > 0 ? per_sm : 1);  // last: marks the entry complete
}

void launch_guide(const DevScene& s, const PathState& p, int bounce, cudaStream_t st) {
  prepare_guide_launch();
  const int* grids = g_guide_grids[current_device_slot()];
  if (s.guide_method == TT_GUIDE_TREE) {
    if (s.num_media > 0) k_guide_tree<true><<<grids[2], kBlock, 0, st>>>(s, p, bounce);
    else k_guide_tree<false><<<grids[2], kBlock, 0, st>>>(s, p, bounce);
    return;
  }
  if (s.guide_net == TT_GUIDE_NET_TCGEN05) {
    if (s.num_media > 0) k_guide_tc<true><<<grids[1], kTcThreads, kTcSmem, st>>>(s, p, bounce);
    else k_guide_tc<false><<<grids[1], kTcThreads, kTcSmem, st>>>(s, p, bounce);
    return;
  }
  const int grid = grids[0];
  if (s.num_media > 0) k_guide<true><<<grid, kGuideWarps * 32, kGuideSmem, st>>>(s, p, bounce);
  else k_guide<false><<<grid, kGuideWarps * 32, kGuideSmem, st>>>(s, p, bounce);
}
void launch_accumulate(const Framebuffer& fb, double* acc, double* light, int n3, cudaStream_t st) {
  const int grid = (n3 + kBlock - 1) / kBlock;
  if (grid > 0) k_accumulate<<<grid < 65535 ? grid : 65535, kBlock, 0, st>>>(fb, acc, light, n3);
}
static int grid_for(int n) {
  int g = (n + kBlock - 1) / kBlock;
  return g < 1 ? 1 : (g > 65535 ? 65535 : g);
}
void launch_intersect_rays(const DevScene& s, const float* rays, int n, int* prim, float* t, float* u, float* v,
                           unsigned int* err, cudaStream_t st) {
  if (n <= 0) return;
  with_bool(s.num_spheres > 0, [&](auto S) {
    with_bool(s.wide != 0, [&](auto W) {
      k_intersect_rays<decltype(S)::value, decltype(W)::value><<<grid_for(n), kBlock, 0, st>>>(s, rays, n, prim, t, u, v,
                                                                                               err);
    });
  });
}
void launch_occluded_rays(const DevScene& s, const float* rays, int n, unsigned char* occ, unsigned int* err,
                          cudaStream_t st) {
  if (n <= 0) return;
  with_bool(s.num_spheres > 0, [&](auto S) {
    with_bool(s.wide != 0, [&](auto W) {
      k_occluded_rays<decltype(S)::value, decltype(W)::value><<<grid_for(n), kBlock, 0, st>>>(s, rays, n, occ, err);
    });
  });
}
void launch_count_rays(const DevScene& s, const float* rays, int n, unsigned long long* counters, unsigned int* err,
                       cudaStream_t st) {
  if (n <= 0) return;
  with_bool(s.num_spheres > 0, [&](auto S) {
    with_bool(s.wide != 0, [&](auto W) {
      k_count_rays<decltype(S)::value, decltype(W)::value><<<grid_for(n), kBlock, 0, st>>>(s, rays, n, counters, err);
    });
  });
}
void launch_sample_bsdf(const DevScene& s, int material, float3 wi, int3 lambda, int n, unsigned long long seed,
                        float* dir, float* val, float* pdf, cudaStream_t st) {
  if (n > 0) k_sample_bsdf<<<grid_for(n), kBlock, 0, st>>>(s, material, wi, lambda, n, seed, dir, val, pdf);
}
void launch_eval_bsdf(const DevScene& s, int material, float3 wi, int3 lambda, const float* dirs, int n, float* val,
                      float* pdf, cudaStream_t st) {
  if (n > 0) k_eval_bsdf<<<grid_for(n), kBlock, 0, st>>>(s, material, wi, lambda, dirs, n, val, pdf);
}
void launch_sample_phase(const DevScene& s, int medium, float3 pos, float3 wi, int3 lambda, int n,
                         unsigned long long seed, float* dir, float* val, float* pdf, cudaStream_t st) {
  if (n > 0) k_sample_phase<<<grid_for(n), kBlock, 0, st>>>(s, medium, pos, wi, lambda, n, seed, dir, val, pdf);
}
void launch_eval_phase(const DevScene& s, int medium, float3 pos, float3 wi, int3 lambda, const float* dirs, int n,
                       float* val, float* pdf, cudaStream_t st) {
  if (n > 0) k_eval_phase<<<grid_for(n), kBlock, 0, st>>>(s, medium, pos, wi, lambda, dirs, n, val, pdf);
}
__global__ void k_resolve(const double* accum, const double* light, const double* inv_spp_px, double inv_spp,
                          double splat_weight, int npix, float* rgb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * npix; i += gridDim.x * blockDim.x) {
    const double inv = inv_spp_px ? inv_spp_px[i / 3] : inv_spp;
    rgb[i] = (float)(accum[i] * inv + splat_weight * light[i]);
  }
}
// The tree guider's quadtree sampler on given uniforms (test hook).
__global__ void k_quadtree_sample(const int4* child, const float* prob, const float* u, int n, float* dir, float* pdf,
                                  float* pdf_eval) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float pd;
    const float3 d = quad_sample(child, prob, 0, u[2 * i], u[2 * i + 1], &pd);
    dir[3 * i] = d.x;
    dir[3 * i + 1] = d.y;
    dir[3 * i + 2] = d.z;
    pdf[i] = pd;
    pdf_eval[i] = quad_pdf(child, prob, 0, d);
  }
}
void launch_quadtree_sample(const int4* child, const float* prob, const float* u, int n, float* dir, float* pdf,
                            float* pdf_eval, cudaStream_t st) {
  if (n > 0) k_quadtree_sample<<<grid_for(n), kBlock, 0, st>>>(child, prob, u, n, dir, pdf, pdf_eval);
}
void launch_resolve(const double* accum, const double* light, const double* inv_spp_px, double inv_spp,
                    double splat_weight, int npix, float* rgb, cudaStream_t st) {
  if (npix > 0) k_resolve<<<grid_for(3 * npix), kBlock, 0, st>>>(accum, light, inv_spp_px, inv_spp, splat_weight, npix, rgb);
}

int kernel_blocks_per_sm() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<false>, kBlock, 0);
  return b < 1 ? 1 : b;
}

}  // namespace tt
