// Device-side building blocks of the path tracer: vector math, the PCG32 stream, the
// sampling warps, spectral conversions, shaders, lights and cameras.  Single precision;
// each function names the reference code whose semantics it reproduces.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "tt_internal.h"

namespace tt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kEps = 2.220446049250313e-16f;   // double epsilon, as added in denominators
constexpr float kEpsF = 1.1920928955078125e-07f; // float epsilon
constexpr float kLargeNumber = 3.4028234663852886e+38f / 16.f;

// Spectrum -> RGB matrix and Smits basis, uploaded by upload_constant_tables().  This
// header is compiled into exactly one translation unit (tt_kernels.cu), which owns them.
__constant__ float c_spec_to_rgb[3][NBINS];
__constant__ float c_smits[7][NBINS];

// ----------------------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 mul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 normalize3(float3 a) { return a * (1.f / len3(a)); }
__device__ __forceinline__ float3 abs3(float3 a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }
__device__ __forceinline__ float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ bool is_zero(float3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
__device__ __forceinline__ float max3(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }

// OrthogonalSystemZAligned (vec3f.hxx:240-258): Duff et al. 2017, listing 3.
struct Frame {
  float3 X, Y, Z;
  __device__ __forceinline__ float3 to_world(float3 v) const { return X * v.x + Y * v.y + Z * v.z; }
  __device__ __forceinline__ float3 to_local(float3 w) const { return f3(dot3(X, w), dot3(Y, w), dot3(Z, w)); }
};
__device__ __forceinline__ Frame frame_z(float3 z) {
  Frame f;
  f.Z = z;
  const float sign = copysignf(1.f, z.z);
  const float a = -1.f / (sign + z.z);
  const float b = z.x * z.y * a;
  f.X = f3(1.f + sign * z.x * z.x * a, sign * b, -sign * z.x);
  f.Y = f3(b, sign + z.y * z.y * a, -z.y);
  return f;
}

// ----------------------------------------------------------------------------------------
// PCG32 (O'Neill 2014) with the pcg32 interface used by RandGen (sampler.cxx:366-393).
struct Rng {
  unsigned long long state, inc;
  __device__ __forceinline__ uint32_t next() {
    unsigned long long old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
  }
  __device__ __forceinline__ void seed(unsigned long long initstate, unsigned long long initseq) {
    state = 0ull;
    inc = (initseq << 1u) | 1u;
    next();
    state += initstate;
    next();
  }
  // Per-path stream: PCG32 streams with nearby increments are strongly correlated, so the
  // (seed, path index) pair is scrambled with the SplitMix64 finalizer (Steele, Lea and
  // Flood 2014) into the initial state and the stream selector.
  __device__ __forceinline__ static unsigned long long splitmix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  __device__ __forceinline__ void seed_path(unsigned long long seed, unsigned long long path) {
    const unsigned long long s1 = splitmix64(seed ^ splitmix64(path));
    const unsigned long long s2 = splitmix64(s1 ^ 0xd1b54a32d192ed03ULL);
    this->seed(s1, s2);
  }
  // 23 random mantissa bits (pcg32::nextFloat): the single-precision twin of nextDouble.
  __device__ __forceinline__ float uniform() { return __uint_as_float((next() >> 9) | 0x3f800000u) - 1.0f; }
  __device__ __forceinline__ void square(float r[2]) { r[0] = uniform(); r[1] = uniform(); }
  // RandGen::UniformInt via pcg32::nextUInt(bound); the rejection loop is bounded.
  __device__ __forceinline__ int uniform_int(int a, int b_inclusive) {
    const uint32_t bound = (uint32_t)(b_inclusive + 1 - a);
    const uint32_t threshold = (~bound + 1u) % bound;
    uint32_t r = next();
    for (int k = 0; k < 64 && r < threshold; ++k) r = next();
    return a + (int)(r % bound);
  }
};

// ----------------------------------------------------------------------------------------
// QuasiRandomSequence (sampler.cxx:254-331) for pt2 with qmc, else the path's PCG32
// stream.  The k-th one-dimensional draw of subsequence `id` is Sobol dimension
// (id << 6) + 2 + k for k < 62 (later draws come from the PCG32 stream); two-dimensional
// draws are dimensions (id << 6) and (id << 6) + 1.  The point index is the sample's index
// in its pixel; every draw is shifted by the pixel's Cranley-Patterson rotation (x for 1D
// draws, (x, y) for 2D draws) modulo 1, here in 32-bit fixed point.  Integer draws always
// come from PCG32 (Sampler::UniformInt).  The subsequence is set per vertex as
// PrepSamplerDimension does: (node count << 1) | 1 for next-event estimation, | 0 for
// scattering; distance sampling continues the subsequence of the scatter before it.
__device__ __forceinline__ uint32_t sobol_mult(uint32_t point, const uint32_t* m) {
  uint32_t c = 0u;
  for (int k = 0; k < 32 && point != 0u; ++k, point >>= 1)
    if (point & 1u) c ^= __ldg(m + k);
  return c;
}
__device__ __forceinline__ float fixed01(uint32_t u) { return (float)(u >> 8) * (1.f / 16777216.f); }

struct Smp2 {
  Rng rng;
  const uint32_t* mats;  // null: pseudo-random
  uint4 q;               // point, rotation x, rotation y, dimension offset | draw counter << 16
  __device__ __forceinline__ void prep(uint32_t id) { q.w = id << 6; }
  __device__ __forceinline__ float uniform() {
    if (!mats) return rng.uniform();
    const uint32_t base = q.w & 0xffffu, sub = q.w >> 16;
    const uint32_t c = sub < 62u ? sobol_mult(q.x, mats + 32u * (base + 2u + sub)) : rng.next();
    q.w = base | ((sub < 0xffffu ? sub + 1u : sub) << 16);
    return fixed01(c + q.y);
  }
  __device__ __forceinline__ void square(float r[2]) {
    if (!mats) {
      rng.square(r);
      return;
    }
    const uint32_t base = q.w & 0xffffu;
    r[0] = fixed01(sobol_mult(q.x, mats + 32u * base) + q.y);
    r[1] = fixed01(sobol_mult(q.x, mats + 32u * (base + 1u)) + q.z);
  }
  __device__ __forceinline__ int uniform_int(int a, int b_inclusive) { return rng.uniform_int(a, b_inclusive); }
};

// Rotation of a pixel in 32-bit fixed point.
__device__ __forceinline__ uint32_t rotation_fixed(float r) { return (uint32_t)fminf(r * 4294967296.f, 4294967040.f); }

// ----------------------------------------------------------------------------------------
// Warps, sampler.cxx:6-124.
__device__ __forceinline__ float3 to_uniform_sphere(const float r[2]) {
  float z = 1.f - 2.f * r[1];
  float s = sqrtf(r[1] * (1.f - r[1]));
  float sn, cs;
  sincosf(2.f * kPi * r[0], &sn, &cs);
  return f3(2.f * cs * s, 2.f * sn * s, z);
}
__device__ __forceinline__ float3 to_uniform_hemisphere(const float r[2]) {
  float3 v = to_uniform_sphere(r);
  v.z = v.z >= 0.f ? v.z : -v.z;
  return v;
}
__device__ __forceinline__ float3 to_sphere_section(float cos_open, const float r[2]) {
  float z = 1.f - r[1] * (1.f - cos_open);
  float s = sqrtf(fmaxf(0.f, 1.f - z * z));
  float sn, cs;
  sincosf(2.f * kPi * r[0], &sn, &cs);
  return f3(cs * s, sn * s, z);
}
__device__ __forceinline__ float3 to_sphere_section(const float r[2], float phi0, float z0, float phi1, float z1) {
  const float z = z0 + r[1] * (z1 - z0);
  float s = sqrtf(1.f - z * z);
  s = isnan(s) ? 0.f : s;
  float sn, cs;
  sincosf(phi0 + (phi1 - phi0) * r[0], &sn, &cs);
  return f3(cs * s, sn * s, z);
}
__device__ __forceinline__ float3 to_cos_hemisphere(const float r[2]) {
  float rho = sqrtf(1.f - r[0]);
  float z = sqrtf(r[0]);
  float sn, cs;
  sincosf(2.f * kPi * r[1], &sn, &cs);
  return f3(cs * rho, sn * rho, z);
}
__device__ __forceinline__ float3 to_triangle_barycentric(const float r[2]) {
  float s = sqrtf(r[0]);
  return f3(1.f - s, (1.f - r[1]) * s, r[1] * s);
}
__device__ __forceinline__ float power_heuristic(float p, float o) {
  float pp = p * p;
  return pp / (pp + o * o + kEps);
}
__device__ __forceinline__ int tower_sampling4(const float* probs, float r) {
  int n = 3;
  while (r >= probs[n] && n > 0) { r -= probs[n]; --n; }
  return n;
}
__device__ __forceinline__ int tower_bisection(const float* cmf, int size, float r) {
  int upper;
  if (r < cmf[0]) upper = 0;
  else if (r >= cmf[size - 1]) upper = size;
  else {
    int first = 0, last = size - 1;
    while (last > first + 1) {
      int center = (first + last) / 2;
      if (r < cmf[center]) last = center; else first = center;
    }
    upper = last;
  }
  return upper >= size ? size - 1 : upper;
}
// tower_bisection's index (the first i with cmf[i] > r, at most size - 1) for r in [0, 1],
// searched only between the guide entries that bracket r: the index is non-decreasing in r,
// so it lies in [guide[g], guide[g + 1]] for g = floor(r kEnvGuide).
__device__ __forceinline__ int guided_bisection(const float* __restrict__ cmf, const int* __restrict__ guide, int size,
                                                float r) {
  const int g = min((int)(r * (float)kEnvGuide), kEnvGuide - 1);
  int lo = __ldg(&guide[g]), hi = __ldg(&guide[g + 1]);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&cmf[mid]) > r) hi = mid;
    else lo = mid + 1;
  }
  return lo >= size ? size - 1 : lo;
}
__device__ __forceinline__ float prob_from_cmf(const float* cmf, int idx) {
  return cmf[idx] - (idx > 0 ? cmf[idx - 1] : 0.f);
}

// ----------------------------------------------------------------------------------------
// Spectral selections (spectral.cxx:81-140, shader_util.hxx:47-92).
struct Lambda {
  int i0, i1, i2;
};
__device__ __forceinline__ unsigned pack_lambda(Lambda l) { return (unsigned)l.i0 | ((unsigned)l.i1 << 8) | ((unsigned)l.i2 << 16); }
__device__ __forceinline__ Lambda unpack_lambda(unsigned p) {
  return Lambda{(int)(p & 255u), (int)((p >> 8) & 255u), (int)((p >> 16) & 255u)};
}
__device__ __forceinline__ float3 take(const float* spec, Lambda l) { return f3(spec[l.i0], spec[l.i1], spec[l.i2]); }
__device__ __forceinline__ float3 selection_to_rgb(float3 v, Lambda l) {
  float3 rgb;
  rgb.x = v.x * c_spec_to_rgb[0][l.i0] + v.y * c_spec_to_rgb[0][l.i1] + v.z * c_spec_to_rgb[0][l.i2];
  rgb.y = v.x * c_spec_to_rgb[1][l.i0] + v.y * c_spec_to_rgb[1][l.i1] + v.z * c_spec_to_rgb[1][l.i2];
  rgb.z = v.x * c_spec_to_rgb[2][l.i0] + v.y * c_spec_to_rgb[2][l.i1] + v.z * c_spec_to_rgb[2][l.i2];
  return rgb;
}
__device__ __forceinline__ float3 lincomb_sel(float a, int ia, float b, int ib, float c, int ic, Lambda l) {
  return f3(a * c_smits[ia][l.i0] + b * c_smits[ib][l.i0] + c * c_smits[ic][l.i0],
            a * c_smits[ia][l.i1] + b * c_smits[ib][l.i1] + c * c_smits[ic][l.i1],
            a * c_smits[ia][l.i2] + b * c_smits[ib][l.i2] + c * c_smits[ic][l.i2]);
}
// RGBToSpectralSelection (spectral.cxx:142-174); basis order white, red, green, blue,
// yellow, cyan, magenta.
__device__ __forceinline__ float3 rgb_to_selection(float r, float g, float b, Lambda l) {
  if (r <= g && r <= b) {
    if (g <= b) return lincomb_sel(r, 0, g - r, 5, b - g, 3, l);
    return lincomb_sel(r, 0, b - r, 5, g - b, 2, l);
  } else if (g <= r && g <= b) {
    if (r <= b) return lincomb_sel(g, 0, r - g, 6, b - r, 3, l);
    return lincomb_sel(g, 0, b - g, 6, r - b, 1, l);
  } else {
    if (r <= g) return lincomb_sel(b, 0, r - b, 4, g - r, 2, l);
    return lincomb_sel(b, 0, g - b, 4, r - g, 1, l);
  }
}

// ----------------------------------------------------------------------------------------
// Physics helpers, shader_physics.hxx:10-148, normaldistributionfunction.hxx:8-127.
__device__ __forceinline__ float3 reflected(float3 wi, float3 n) { return 2.f * dot3(wi, n) * n - wi; }
__device__ __forceinline__ bool refracted(float3 wi, float3 m, float eta, float3* out) {
  const float c = dot3(m, wi);
  const float t2 = 1.f - eta * eta * (1.f - c * c);
  if (t2 < 0.f) return false;
  const float s = c >= 0.f ? 1.f : -1.f;
  *out = (eta * c - s * sqrtf(t2)) * m - eta * wi;
  return true;
}
__device__ __forceinline__ float fresnel_reflectivity(float cs_i, float cs_t, float eta) {
  float rs = (eta * cs_i - cs_t) / (eta * cs_i + cs_t);
  float rp = (eta * cs_t - cs_i) / (eta * cs_t + cs_i);
  return 0.5f * (rs * rs + rp * rp);
}
__device__ __forceinline__ float beckmann_d(float alpha, float cs) {
  if (cs <= 0.f) return 0.f;
  const float t1 = (cs * cs - 1.f) / (cs * cs * alpha * alpha);
  const float t2 = alpha * alpha * cs * cs * cs * cs * kPi;
  return expf(t1) / t2;
}
__device__ __forceinline__ float3 beckmann_sample_wh(float alpha, const float r[2]) {
  const float t1 = -alpha * alpha * logf(r[0]);
  const float t = 1.f / (t1 + 1.f);
  const float z = sqrtf(t);
  const float rho = sqrtf(1.f - t);
  float sn, cs;
  sincosf(2.f * kPi * r[1], &sn, &cs);
  return f3(cs * rho, sn * rho, z);
}
__device__ __forceinline__ float g1_vcavity(float cos_v_m, float cos_v_n, float cos_n_m) {
  if (cos_v_m * cos_v_n < 0.f) return 0.f;
  return fminf(1.f, 2.f * fabsf(cos_n_m * cos_v_n) / (fabsf(cos_v_m) + kEps));
}
__device__ __forceinline__ float g2_vcavity(float wh_in, float wh_out, float ns_in, float ns_out, float ns_wh) {
  return fminf(g1_vcavity(wh_in, ns_in, ns_wh), g1_vcavity(wh_out, ns_out, ns_wh));
}
// G2VCavityTransmissive (normaldistributionfunction.hxx:87-94).
__device__ __forceinline__ float g2_vcavity_transmissive(float wh_in, float wh_out, float ns_in, float ns_out,
                                                         float ns_wh) {
  return fmaxf(g1_vcavity(wh_in, ns_in, ns_wh) + g1_vcavity(wh_out, ns_out, ns_wh) - 1.f, 0.f);
}
// FresnelReflectivity from the incident cosine alone (Walter et al. 2007; shader_physics.hxx:132-148).
__device__ __forceinline__ float fresnel_reflectivity_walter(float cos_n_wi, float eta_i_over_t) {
  const float c = fabsf(cos_n_wi);
  const float tmp = 1.f / (eta_i_over_t * eta_i_over_t) - 1.f + c * c;
  if (tmp < 0.f) return 1.f;
  const float g = sqrtf(tmp);
  if (g == 0.f && c == 0.f) return 1.f;
  const float nom = c * (g + c) - 1.f, den = c * (g - c) + 1.f;
  const float a = (g - c) / (g + c), b = nom / den;
  return 0.5f * a * a * (1.f + b * b);
}
__device__ __forceinline__ float clamp_dot(float3 a, float3 b) { return fmaxf(0.f, dot3(a, b)); }
constexpr float kWiBelowHorizonFix = 1.e-6f;
__device__ __forceinline__ float vndf_pdf(float d, float3 wh, float3 wi) {
  float3 whp = f3(-wh.x, -wh.y, wh.z);
  const float a = clamp_dot(wi, whp), b = clamp_dot(wh, wi);
  return d * fabsf(wh.z) * ((2.f * b + kWiBelowHorizonFix) / (b + a + kWiBelowHorizonFix));
}

// ----------------------------------------------------------------------------------------
// Surface interaction (scene.hxx:77-95).
struct Surf {
  int prim;
  int material;
  float3 pos;
  float3 ng;        // geometry_normal (winding)
  float3 ns_raw;    // smooth_normal
  float3 n;         // oriented geometry normal
  float3 ns;        // oriented shading normal
  float3 bounds;    // pos_bounds
  float2 uv;        // texture coordinates (SurfaceInteraction::tex_coord)
};

// util::Gamma<float>(7) (util.hxx:124-127) with the full float epsilon.
__device__ __forceinline__ float gamma7() { return (7.f * kEpsF) / (1.f - 7.f * kEpsF); }

// AntiSelfIntersectionOffset (scene.cxx:256-261).
__device__ __forceinline__ float3 offset_at(const Surf& s, float3 exitant) {
  const float delta = dot3(s.bounds, abs3(s.ng));
  return (delta * (dot3(exitant, s.ng) > 0.f ? 1.f : -1.f)) * s.ng;
}

// Builds the interaction for barycentrics (w0, w1, w2) of the triangle at leaf slot `slot`.
// FirstIntersectionTriangle (embreeaccelerator.cxx:216-244) passes (u, v, 1-u-v) as the
// HitId barycentrics to FillPosBoundsTriangle while interpolating with (1-u-v, u, v);
// `bw` carries the weights used for the bound.
__device__ __forceinline__ Surf make_surface(const DevScene& sc, int slot, float w0, float w1, float w2, float3 bw) {
  const float4 a = __ldg(&sc.tris[3 * slot]);
  const float4 b = __ldg(&sc.tris[3 * slot + 1]);
  const float4 c = __ldg(&sc.tris[3 * slot + 2]);
  Surf s;
  s.prim = __float_as_int(a.w);
  s.material = __float_as_int(b.w);
  const float3 p0 = xyz(a), p1 = xyz(b), p2 = xyz(c);
  s.pos = p0 * w0 + p1 * w1 + p2 * w2;
  s.ng = normalize3(cross3(p1 - p0, p2 - p0));
  if (sc.normals) {
    const uint4 ti = __ldg(&sc.tri_idx[s.prim]);
    const float* N = sc.normals;
    float3 na = f3(N[3 * ti.x], N[3 * ti.x + 1], N[3 * ti.x + 2]);
    float3 nb = f3(N[3 * ti.y], N[3 * ti.y + 1], N[3 * ti.y + 2]);
    float3 nc = f3(N[3 * ti.z], N[3 * ti.z + 1], N[3 * ti.z + 2]);
    s.ns_raw = normalize3(na * w0 + nb * w1 + nc * w2);
  } else {
    s.ns_raw = s.ng;
  }
  s.bounds = (abs3(p0 * bw.x) + abs3(p1 * bw.y) + abs3(p2 * bw.z)) * gamma7();
  s.n = s.ng;
  s.ns = s.ns_raw;
  // Texture coordinates interpolated like the position (rtcInterpolate1 of the uv vertex
  // attribute, embreeaccelerator.cxx:226-228); only textured materials read them.
  s.uv = make_float2(0.f, 0.f);
  if (sc.uvs && sc.materials[s.material].tex) {
    const uint4 ti = __ldg(&sc.tri_idx[s.prim]);
    const float2 ua = __ldg(&sc.uvs[ti.x]), ub = __ldg(&sc.uvs[ti.y]), uc = __ldg(&sc.uvs[ti.z]);
    s.uv = make_float2(ua.x * w0 + ub.x * w1 + uc.x * w2, ua.y * w0 + ub.y * w1 + uc.y * w2);
  }
  return s;
}

// KartesianToSpherical (third component up, vec3f.hxx:298-321) then SphericalToUv
// (vec3f.hxx:286-295) of a direction: a sphere hit's texture coordinates from its normal
// (EmbreeAccelerator::FirstIntersectionSphere, embreeaccelerator.cxx:258).
__device__ __forceinline__ float2 direction_uv(float3 d) {
  const float x = d.x, z = d.y, y = d.z;
  const float ax = fabsf(x), az = fabsf(z);
  const float theta = acosf(fminf(1.f, fmaxf(-1.f, y / len3(d))));
  float phi;
  if (ax > az) {
    phi = atan2f(z, ax);
    phi = (x > 0.f) ? phi : kPi - phi;
  } else {
    phi = atan2f(x, az);
    phi = (z > 0.f) ? (kPi / 2.f) - phi : (3.f / 2.f * kPi) + phi;
  }
  return make_float2(phi / (2.f * kPi), theta / kPi);
}

// UvToPixel (texture.hxx:37-55) and Texture::GetPixel (texture.hxx:94-117): the texel under
// the coordinates wrapped to [0, 1), v up, row 0 at the top; linear RGB.
__device__ __forceinline__ float3 texture_rgb(const DevMaterial& m, float2 uv) {
  float dummy;
  float u = modff(uv.x, &dummy), v = modff(uv.y, &dummy);
  if (u < 0.f) u = 1.f + u;
  if (v < 0.f) v = 1.f + v;
  if (u > 1.f - kEpsF) u -= kEpsF;
  if (v > 1.f - kEpsF) v -= kEpsF;
  const int x = min(max((int)(u * m.tex_w), 0), m.tex_w - 1);
  const int y = min(max(m.tex_h - (int)(v * m.tex_h) - 1, 0), m.tex_h - 1);
  const float* p = m.tex + 3 * ((size_t)y * m.tex_w + x);
  return f3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

__device__ __forceinline__ void orient(Surf& s, float3 incident) {
  const float sign = -copysignf(1.f, dot3(incident, s.ng));
  s.n = sign * s.ng;
  s.ns = sign * s.ns_raw;
}

// ----------------------------------------------------------------------------------------
// Shaders (shader.cxx).
struct ScatterSample {
  float3 dir;
  float3 value;
  float pdf;
  bool delta;
};

// pt2's path regularisation (ShaderQuery::minimum_roughness): a dielectric met after a
// rough bounce spreads its specular lobes into uniform cones of cos opening 1 - r
// (SpecularTransmissiveDielectricShader::Sample/EvaluateBsdfMollified, shader.cxx:482-605).
__device__ __forceinline__ float3 eval_dielectric_mollified(const DevMaterial& m, float3 wi, const Surf& s, float3 wo,
                                                            float rough, float* pdf) {
  const float opening_cos = 1.f - rough;
  const bool entering = dot3(s.ng, wi) > 0.f;
  const float eta = entering ? 1.f / m.ior_ratio : m.ior_ratio;
  const float abs_i = fabsf(dot3(s.ns, wi));
  float fr = 1.f;
  float3 wt;
  const bool has_wt = refracted(wi, s.ns, eta, &wt);
  if (has_wt) fr = fresnel_reflectivity(abs_i, fabsf(dot3(wt, s.ns)), eta);
  const float prob_reflection = has_wt ? fmaxf(0.1f, fminf(0.9f, fr)) : 1.f;
  const float section_pdf = 1.f / (2.f * kPi * (1.f - opening_cos));
  const bool maybe_reflected = dot3(reflected(wi, s.ns), wo) > opening_cos;
  float total_pdf = maybe_reflected ? section_pdf * prob_reflection : 0.f;
  float total_val = maybe_reflected ? prob_reflection * fr : 0.f;
  if (has_wt && dot3(wt, wo) > opening_cos) {
    total_val += (1.f - fr) * section_pdf;
    total_pdf += (1.f - prob_reflection) * section_pdf;
  }
  if (dot3(wo, s.n) < 0.f) total_val *= eta * eta;
  total_val /= fabsf(dot3(wo, s.ns));
  if (pdf) *pdf = total_pdf;
  return f3(total_val, total_val, total_val);
}

// DiffuseShader's reflectance at the hit: times the texture's RGB turned into the selected
// wavelengths' values when the material has a texture (MaybeMultiplyTextureLookup,
// shader.cxx:17-27).
__device__ __forceinline__ float3 diffuse_kr(const DevMaterial& m, const Surf& s, Lambda l) {
  float3 kr = take(m.reflectance, l);
  if (m.tex) {
    const float3 c = texture_rgb(m, s.uv);
    kr = mul(kr, rgb_to_selection(c.x, c.y, c.z, l));
  }
  return kr;
}

// SpecularDenseDielectricShader (shader.cxx:977-1081): Schlick reflectivity of the coating
// (SchlicksApproximation, shader_physics.hxx:95-101) and the diffuse attenuation
// (1 - R(w_in)) (1 - R(w_out)) / (1 - average albedo) of Kelemen and Szirmay-Kalos 2001
// (DiffuseAttenuationFactor), the average albedo k + (1 - k) 2 / 42
// (AverageOfProjectedSchlicksApproximationOverHemisphere).
__device__ __forceinline__ float schlick(float k, float cos_n) {
  const float x = 1.f - cos_n;
  return k + (1.f - k) * (x * x * x * x * x);
}
__device__ __forceinline__ float dense_attenuation(float k, float r_in, float r_out) {
  const float avg = k + (1.f - k) * (2.f / 42.f);
  return (1.f - r_in) * (1.f - r_out) / (1.f - avg);
}

// Shader::MyRoughness (shader.cxx:244-247, 666-670, 728-731): the alpha of the microfacet
// and of the glossy dielectric, 0 otherwise.
__device__ __forceinline__ float my_roughness(const DevMaterial& m) {
  return (m.shader == TT_SHADER_MICROFACET || m.shader == TT_SHADER_GLOSSY_DIELECTRIC) ? m.alpha : 0.f;
}

// GlossyTransmissiveDielectricShader (shader.cxx:710-787) with its wrapper
// GlossyTransmissiveDielectricWrapper (shader.cxx:126-190) and the sampling density
// TransmissiveMicrofacetDensity (normaldistributionfunction.hxx:149-197): a rough interface
// with a Beckmann distribution of roughness alpha; reflection and refraction are chosen by
// the Fresnel reflectivity at the sampled half vector, which is drawn from the Beckmann
// distribution of the broadened roughness alpha (1.2 - 0.2 |cos wi|).  Local frame on the
// oriented shading normal; eta_i_over_t from the winding normal's side of wi.
struct GlossyDielectric {
  Frame fr;
  float3 wi;     // local
  float3 ng;     // oriented geometry normal, local
  float eta;     // eta_i / eta_t, i = the side of wi
  float alpha, alpha_b;
};
__device__ __forceinline__ GlossyDielectric glossy_dielectric(const DevMaterial& m, float3 wi, const Surf& s,
                                                              float min_rough) {
  GlossyDielectric g;
  g.fr = frame_z(s.ns);
  g.wi = g.fr.to_local(wi);
  g.ng = g.fr.to_local(s.n);
  g.eta = dot3(s.ng, wi) < 0.f ? m.ior_ratio : 1.f / m.ior_ratio;
  g.alpha = fmaxf(min_rough, m.alpha);
  g.alpha_b = g.alpha * (1.2f - 0.2f * fabsf(g.wi.z));  // AlphaBroadeningFormula, shader.cxx:59-62
  return g;
}
// HalfVector (shader_physics.hxx:37-46); a vanishing sum falls back to the frame's x axis.
__device__ __forceinline__ float3 half_vector(float3 wi, float3 wo) {
  const float3 h = wi + wo;
  const float n = len3(h);
  return n > 0.f ? h * (1.f / n) : frame_z(wi).X;
}
// HalfVectorRefracted (shader_physics.hxx:50-66), Walter et al. 2007 eq. 16.
__device__ __forceinline__ bool half_vector_refracted(float3 wi, float3 wo, float eta, float3* out) {
  float3 h = -(eta * wi + wo);
  const float n = len3(h);
  h = n > 0.f ? h * (1.f / n) : wi;
  *out = h;
  return dot3(h, wi) * dot3(h, wo) < 0.f;
}
// HalfVectorPdfToTransmittedPdf (shader_physics.hxx:80-88).
__device__ __forceinline__ float half_pdf_to_transmitted(float pdf_wh, float eta, float wi_wh, float wo_wh) {
  float den = eta * wi_wh + wo_wh;
  if (den == 0.f) return pdf_wh;
  return pdf_wh * fabsf(wo_wh) / (den * den);
}
// TransmissiveMicrofacetDensity::Pdf with the broadened distribution.
__device__ __forceinline__ float glossy_dielectric_pdf(const GlossyDielectric& g, float3 wo) {
  float pdf_t = 0.f;
  float3 wht;
  if (half_vector_refracted(g.wi, wo, g.eta, &wht)) {
    const float fr = fresnel_reflectivity_walter(fabsf(dot3(wht, g.wi)), g.eta);
    const float d = beckmann_d(g.alpha_b, fabsf(wht.z)) * fabsf(wht.z);
    pdf_t = half_pdf_to_transmitted(d, g.eta, dot3(wht, g.wi), dot3(wht, wo)) * (1.f - fr);
  }
  const float3 whr = half_vector(g.wi, wo);
  const float fr = fresnel_reflectivity_walter(fabsf(dot3(whr, g.wi)), g.eta);
  const float d = beckmann_d(g.alpha_b, fabsf(whr.z)) * fabsf(whr.z);
  const float pdf_r = d * 0.25f / (fabsf(dot3(whr, g.wi)) + kEps) * fr;
  return pdf_r + pdf_t;
}
// GlossyTransmissiveDielectricWrapper::Evaluate: BRDF on the oriented geometry normal's
// side, BTDF below; monochromatic.
__device__ __forceinline__ float glossy_dielectric_eval(const GlossyDielectric& g, float3 wo, float* pdf) {
  if (pdf) *pdf = glossy_dielectric_pdf(g, wo);
  const float ns_out = wo.z, ns_in = g.wi.z;
  if (dot3(g.ng, wo) >= 0.f) {
    const float3 h = half_vector(g.wi, wo);
    const float wh_out = dot3(wo, h), wh_in = dot3(g.wi, h);
    const float fr = fresnel_reflectivity_walter(fabsf(wh_in), g.eta);
    const float d = beckmann_d(g.alpha, fabsf(h.z));
    const float gg = g2_vcavity(wh_in, wh_out, ns_in, ns_out, h.z);
    return fr * gg * d * 0.25f / (fabsf(ns_in * ns_out) + kEps);
  }
  float3 h;
  if (!half_vector_refracted(g.wi, wo, g.eta, &h)) return 0.f;
  if (h.z < 0.f) h = -h;
  const float wh_out = dot3(wo, h), wh_in = dot3(g.wi, h);
  const float fr = fresnel_reflectivity_walter(fabsf(wh_in), g.eta);
  const float d = beckmann_d(g.alpha, fabsf(h.z));
  const float j = half_pdf_to_transmitted(1.f, g.eta, wh_in, wh_out);
  const float gg = g2_vcavity_transmissive(wh_in, wh_out, ns_in, ns_out, h.z);
  return (1.f - fr) * fabsf(wh_in) * gg * d * j / (fabsf(ns_in * ns_out) + kEps);
}

// EvaluateBSDF of DiffuseShader (shader.cxx:280-297), the delta shaders, and
// MicrofacetShader (shader.cxx:676-689 with MicrofacetShaderWrapper::Evaluate :74-113).
// min_rough > 0 (pt2 only) raises the microfacet's alpha and mollifies the dielectric.
__device__ __forceinline__ float3 eval_bsdf(const DevMaterial& m, float3 wi, const Surf& s, float3 wo, Lambda l,
                                            float* pdf, float min_rough = 0.f) {
  if (m.shader == TT_SHADER_SPECULAR_DIELECTRIC && min_rough > 0.f)
    return eval_dielectric_mollified(m, wi, s, wo, min_rough, pdf);
  if (m.shader == TT_SHADER_DIFFUSE) {
    float3 ret = f3(0.f, 0.f, 0.f);
    if (dot3(s.n, wo) > 0.f) ret = diffuse_kr(m, s, l) * (1.f / kPi);
    if (pdf) *pdf = fmaxf(0.f, dot3(s.ns, wo)) / kPi;
    return ret;
  }
  if (m.shader == TT_SHADER_GLOSSY_DIELECTRIC) {
    const GlossyDielectric g = glossy_dielectric(m, wi, s, min_rough);
    const float v = glossy_dielectric_eval(g, g.fr.to_local(wo), pdf);
    return f3(v, v, v);
  }
  if (m.shader == TT_SHADER_SPECULAR_DENSE_DIELECTRIC) {
    // The diffuse part; the specular reflection is a delta lobe.
    if (!(dot3(s.n, wo) > 0.f)) {
      if (pdf) *pdf = 0.f;
      return f3(0.f, 0.f, 0.f);
    }
    const float r_in = schlick(m.spec, fmaxf(0.f, dot3(s.ns, wi)));
    const float r_out = schlick(m.spec, fmaxf(0.f, dot3(s.ns, wo)));
    if (pdf) *pdf = fmaxf(0.f, dot3(s.ns, wo)) / kPi * (1.f - r_in);
    return diffuse_kr(m, s, l) * ((1.f / kPi) * dense_attenuation(m.spec, r_in, r_out));
  }
  if (m.shader == TT_SHADER_MICROFACET) {
    const Frame fr = frame_z(s.ns);
    const float3 ng = fr.to_local(s.n);
    const float3 lwi = fr.to_local(wi), lwo = fr.to_local(wo);
    const float3 wh = normalize3(lwi + lwo);
    const float ns_out = lwo.z, ns_in = lwi.z, ns_wh = wh.z;
    const float wh_out = dot3(lwo, wh), wh_in = dot3(lwi, wh);
    const float d = beckmann_d(fmaxf(m.alpha, min_rough), fabsf(ns_wh));
    const float g = g2_vcavity(wh_in, wh_out, ns_in, ns_out, ns_wh);
    if (pdf) {
      const float3 whf = wh.z < 0.f ? -wh : wh;
      *pdf = vndf_pdf(d, whf, lwi) * 0.25f / (fabsf(dot3(whf, lwi)) + kEps);
    }
    if (dot3(ng, lwo) <= 0.f) return f3(0.f, 0.f, 0.f);
    const float3 kr = take(m.reflectance, l);
    const float x = 1.f - fabsf(wh_in);
    const float f5 = x * x * x * x * x;
    const float mono = g * d * 0.25f / (fabsf(ns_in * ns_out) + kEps);
    return f3(kr.x + (1.f - kr.x) * f5, kr.y + (1.f - kr.y) * f5, kr.z + (1.f - kr.z) * f5) * mono;
  }
  if (pdf) *pdf = 0.f;
  return f3(0.f, 0.f, 0.f);
}

// SampleBSDF: DiffuseShader (shader.cxx:300-318), SpecularReflectiveShader (:345-366),
// SpecularTransmissiveDielectricShader::SampleBsdfRegular (:401-473), MicrofacetShader
// (:692-707).  Draw order matches the reference: square, then single uniforms.
template <class R>
__device__ __forceinline__ ScatterSample sample_bsdf(const DevMaterial& m, float3 wi, const Surf& s, R& rng,
                                                     Lambda l, float min_rough = 0.f) {
  ScatterSample out;
  out.delta = false;
  if (m.shader == TT_SHADER_SPECULAR_DIELECTRIC && min_rough > 0.f) {
    // SampleBsdfMollified (shader.cxx:482-549): lobe choice, then a direction in its cone.
    const float opening_cos = 1.f - min_rough;
    const float abs_i = fabsf(dot3(s.ns, wi));
    const bool entering = dot3(s.ng, wi) > 0.f;
    const float eta = entering ? 1.f / m.ior_ratio : m.ior_ratio;
    float fr = 1.f;
    float3 wt;
    const bool has_wt = refracted(wi, s.ns, eta, &wt);
    if (has_wt) fr = fresnel_reflectivity(abs_i, fabsf(dot3(wt, s.ns)), eta);
    const float prob_reflection = has_wt ? fmaxf(0.1f, fminf(0.9f, fr)) : 1.f;
    const bool do_reflect = has_wt ? rng.uniform() < prob_reflection : true;
    const float section_pdf = 1.f / (2.f * kPi * (1.f - opening_cos));
    float r[2];
    rng.square(r);
    const float3 axis = do_reflect ? reflected(wi, s.ns) : wt;
    out.dir = frame_z(axis).to_world(to_sphere_section(opening_cos, r));
    float value;
    if (do_reflect) {
      out.pdf = prob_reflection * section_pdf;
      value = fr * section_pdf;
    } else {
      out.pdf = (1.f - prob_reflection) * section_pdf;
      value = (1.f - fr) * section_pdf;
    }
    value /= fabsf(dot3(out.dir, s.ns));
    if (dot3(out.dir, s.n) < 0.f) value *= eta * eta;
    out.value = f3(value, value, value);
    return out;
  }
  if (m.shader == TT_SHADER_SPECULAR_DENSE_DIELECTRIC) {
    // Reflection off the coating with probability R(w_in), else the attenuated diffuse base.
    const float cos_in = fmaxf(0.f, dot3(s.ns, wi));
    const float r_in = schlick(m.spec, cos_in);
    if (rng.uniform() < r_in) {
      const float3 r = reflected(wi, s.ns);
      out.dir = r;
      out.pdf = r_in;
      out.delta = true;
      const float v = dot3(s.n, r) >= 0.f ? r_in / (cos_in + kEps) : 0.f;
      out.value = f3(v, v, v);
      return out;
    }
    const Frame fr = frame_z(s.ns);
    float r[2];
    rng.square(r);
    const float3 v = to_cos_hemisphere(r);
    out.dir = fr.to_world(v);
    out.pdf = v.z / kPi * (1.f - r_in);
    const float r_out = schlick(m.spec, fmaxf(0.f, dot3(s.ns, out.dir)));
    out.value = dot3(s.n, out.dir) > 0.f
                    ? diffuse_kr(m, s, l) * ((1.f / kPi) * dense_attenuation(m.spec, r_in, r_out))
                    : f3(0.f, 0.f, 0.f);
    return out;
  }
  if (m.shader == TT_SHADER_GLOSSY_DIELECTRIC) {
    // TransmissiveMicrofacetDensity::Sample: half vector, then reflect or refract.
    const GlossyDielectric g = glossy_dielectric(m, wi, s, min_rough);
    float r[2];
    rng.square(r);
    const float3 wh = beckmann_sample_wh(g.alpha_b, r);
    float fr = fresnel_reflectivity_walter(fabsf(dot3(wh, g.wi)), g.eta);
    float3 wt;
    if (!refracted(g.wi, wh, g.eta, &wt)) fr = 1.f;
    const float3 wo = rng.uniform() < fr ? reflected(g.wi, wh) : wt;
    const float v = glossy_dielectric_eval(g, wo, &out.pdf);
    out.dir = g.fr.to_world(wo);
    out.value = f3(v, v, v);
    return out;
  }
  if (m.shader == TT_SHADER_DIFFUSE) {
    const Frame fr = frame_z(s.ns);
    float r[2];
    rng.square(r);
    const float3 v = to_cos_hemisphere(r);
    out.pdf = v.z / kPi;
    out.dir = fr.to_world(v);
    out.value = dot3(s.n, out.dir) > 0.f ? diffuse_kr(m, s, l) * (1.f / kPi) : f3(0.f, 0.f, 0.f);
    return out;
  }
  if (m.shader == TT_SHADER_SPECULAR_REFLECTIVE) {
    const float3 r = reflected(wi, s.ns);
    out.dir = r;
    out.pdf = 1.f;
    out.delta = true;
    out.value = dot3(s.n, r) < 0.f ? f3(0.f, 0.f, 0.f) : take(m.reflectance, l) * (1.f / dot3(s.ns, r));
    return out;
  }
  if (m.shader == TT_SHADER_SPECULAR_DIELECTRIC) {
    const float abs_i = fabsf(dot3(s.ns, wi));
    const bool entering = dot3(s.ng, wi) > 0.f;
    const float eta = entering ? 1.f / m.ior_ratio : m.ior_ratio;
    float fr = 1.f;
    float3 wt;
    const bool has_wt = refracted(wi, s.ns, eta, &wt);
    if (has_wt) fr = fresnel_reflectivity(abs_i, fabsf(dot3(wt, s.ns)), eta);
    const float prob_reflection = has_wt ? fmaxf(0.1f, fminf(0.9f, fr)) : 1.f;
    const bool do_reflect = has_wt ? rng.uniform() < prob_reflection : true;
    float value;
    out.delta = true;
    if (do_reflect) {
      out.dir = reflected(wi, s.ns);
      out.pdf = prob_reflection;
      value = fr;
    } else {
      out.dir = wt;
      out.pdf = 1.f - prob_reflection;
      value = 1.f - fr;
    }
    value /= fabsf(dot3(out.dir, s.ns));
    if (dot3(out.dir, s.n) < 0.f) value *= eta * eta;  // radiance transport
    out.value = f3(value, value, value);
    return out;
  }
  // TT_SHADER_MICROFACET
  const Frame fr = frame_z(s.ns);
  const float3 lwi = fr.to_local(wi);
  float r[2];
  rng.square(r);
  const float alpha = fmaxf(m.alpha, min_rough);
  float3 wh = beckmann_sample_wh(alpha, r);
  {
    // VisibleNdfVCavity::Sample
    const float3 whp = f3(-wh.x, -wh.y, wh.z);
    const float prob = clamp_dot(lwi, whp) / (clamp_dot(lwi, wh) + clamp_dot(lwi, whp) + kWiBelowHorizonFix);
    if (rng.uniform() < prob) wh = whp;
  }
  const float3 lwo = reflected(lwi, wh);
  const float3 ng = fr.to_local(s.n);
  const float ns_out = lwo.z, ns_in = lwi.z, ns_wh = wh.z;
  const float wh_out = dot3(lwo, wh), wh_in = dot3(lwi, wh);
  const float d = beckmann_d(alpha, fabsf(ns_wh));
  const float g = g2_vcavity(wh_in, wh_out, ns_in, ns_out, ns_wh);
  const float3 whf = wh.z < 0.f ? -wh : wh;
  out.pdf = vndf_pdf(d, whf, lwi) * 0.25f / (fabsf(dot3(whf, lwi)) + kEps);
  out.dir = fr.to_world(lwo);
  if (dot3(ng, lwo) <= 0.f) {
    out.value = f3(0.f, 0.f, 0.f);
    return out;
  }
  const float3 kr = take(m.reflectance, l);
  const float x = 1.f - fabsf(wh_in);
  const float f5 = x * x * x * x * x;
  const float mono = g * d * 0.25f / (fabsf(ns_in * ns_out) + kEps);
  out.value = f3(kr.x + (1.f - kr.x) * f5, kr.y + (1.f - kr.y) * f5, kr.z + (1.f - kr.z) * f5) * mono;
  return out;
}

// BsdfCorrectionFactor (rendering_randomwalk_impl.hxx:616-622), radiance transport.
__device__ __forceinline__ float bsdf_correction(const Surf& s, float3 exitant) {
  return fabsf(dot3(s.ns, exitant)) / (fabsf(dot3(s.n, exitant)) + kEps);
}

// ----------------------------------------------------------------------------------------
// Environmental lights (light.hxx:146-304, light.cxx:10-189).
__device__ __forceinline__ float3 env_local(const DevEnvLight& L, float3 d) {
  return f3(L.X[0] * d.x + L.X[1] * d.y + L.X[2] * d.z, L.Y[0] * d.x + L.Y[1] * d.y + L.Y[2] * d.z,
            L.Z[0] * d.x + L.Z[1] * d.y + L.Z[2] * d.z);
}
__device__ __forceinline__ float3 env_world(const DevEnvLight& L, float3 v) {
  return f3(L.X[0] * v.x + L.Y[0] * v.y + L.Z[0] * v.z, L.X[1] * v.x + L.Y[1] * v.y + L.Z[1] * v.z,
            L.X[2] * v.x + L.Y[2] * v.y + L.Z[2] * v.z);
}

// EnvMapLight::MapToImage: KartesianToSpherical (third component up, vec3f.hxx:298-321),
// SphericalToUv, UvToPixel (texture.hxx:37-55).
__device__ __forceinline__ void envmap_pixel(const DevEnvLight& L, float3 dir_out, int* px, int* py) {
  const float3 loc = env_local(L, dir_out);
  const float x = loc.x, z = loc.y, y = loc.z;
  const float ax = fabsf(x), az = fabsf(z);
  const float r = sqrtf(loc.x * loc.x + loc.y * loc.y + loc.z * loc.z);
  const float theta = acosf(y / r);
  float phi;
  if (ax > az) {
    phi = atan2f(z, ax);
    phi = (x > 0.f) ? phi : kPi - phi;
  } else {
    phi = atan2f(x, az);
    phi = (z > 0.f) ? (kPi / 2.f) - phi : (3.f / 2.f * kPi) + phi;
  }
  float u = phi / (2.f * kPi), v = theta / kPi;
  float dummy;
  u = modff(u, &dummy);
  v = modff(v, &dummy);
  if (u < 0.f) u = 1.f + u;
  if (v < 0.f) v = 1.f + v;
  if (u > 1.f - kEpsF) u -= kEpsF;
  if (v > 1.f - kEpsF) v -= kEpsF;
  int ix = (int)(u * L.w);
  int iy = (int)(v * L.h);
  iy = L.h - iy - 1;
  *px = min(max(ix, 0), L.w - 1);
  *py = min(max(iy, 0), L.h - 1);
}
__device__ __forceinline__ void envmap_pixel_angles(const DevEnvLight& L, int x, int y, float* phi0, float* z0,
                                                    float* phi1, float* z1) {
  float ul = (float)x / L.w, vl = (float)y / L.h;
  float uu = ul + 1.f / L.w, vu = vl + 1.f / L.h;
  vl = 1.f - vl;
  vu = 1.f - vu;
  *phi0 = ul * (2.f * kPi);
  *phi1 = uu * (2.f * kPi);
  *z0 = cosf(vl * kPi);
  *z1 = cosf(vu * kPi);
}
__device__ __forceinline__ float3 envmap_value(const DevEnvLight& L, int x, int y, Lambda l) {
  const float* p = L.tex + 3 * ((size_t)y * L.w + x);
  return rgb_to_selection(__ldg(p), __ldg(p + 1), __ldg(p + 2), l);
}
__device__ __forceinline__ float envmap_pdf_of_pixel(const DevEnvLight& L, int x, int y) {
  const float proby = prob_from_cmf(L.cmf_rows, y);
  const float probx = prob_from_cmf(L.cmf_cols + (size_t)y * L.w, x);
  float phi0, z0, phi1, z1;
  envmap_pixel_angles(L, x, y, &phi0, &z0, &phi1, &z1);
  return proby * probx / ((z1 - z0) * (phi1 - phi0));
}

__device__ __forceinline__ float3 env_eval_one(const DevEnvLight& L, float3 dir_out, Lambda l) {
  switch (L.kind) {
    // Dome frame Z = down direction: light reaches directions pointing down.
    case TT_ENV_DOME: return dot3(dir_out, f3(L.Z[0], L.Z[1], L.Z[2])) > 0.f ? take(L.spectrum, l) : f3(0.f, 0.f, 0.f);
    case TT_ENV_SUN: return dot3(dir_out, f3(L.Z[0], L.Z[1], L.Z[2])) > L.cos_opening ? take(L.spectrum, l) : f3(0.f, 0.f, 0.f);
    case TT_ENV_MAP: {
      int x, y;
      envmap_pixel(L, dir_out, &x, &y);
      return envmap_value(L, x, y, l);
    }
    default: return f3(0.f, 0.f, 0.f);
  }
}
__device__ __forceinline__ float env_pdf_one(const DevEnvLight& L, float3 dir_out) {
  switch (L.kind) {
    case TT_ENV_DOME: return dot3(dir_out, f3(L.Z[0], L.Z[1], L.Z[2])) > 0.f ? 1.f / (2.f * kPi) : 0.f;
    case TT_ENV_SUN: return dot3(dir_out, f3(L.Z[0], L.Z[1], L.Z[2])) > L.cos_opening ? L.pdf_val : 0.f;
    case TT_ENV_MAP: {
      int x, y;
      envmap_pixel(L, dir_out, &x, &y);
      return envmap_pdf_of_pixel(L, x, y);
    }
    default: return 0.f;
  }
}

struct DirSample {
  float3 dir;
  float3 value;
  float pdf;
  bool delta;
};

template <class R>
__device__ __forceinline__ DirSample env_sample_one(const DevEnvLight& L, R& rng, Lambda l) {
  DirSample s;
  s.delta = false;
  float r[2];
  switch (L.kind) {
    case TT_ENV_DOME:
      rng.square(r);
      s.dir = env_world(L, to_uniform_hemisphere(r));
      s.value = take(L.spectrum, l);
      s.pdf = 1.f / (2.f * kPi);
      return s;
    case TT_ENV_SUN:
      rng.square(r);
      s.dir = env_world(L, to_sphere_section(L.cos_opening, r));
      s.value = take(L.spectrum, l);
      s.pdf = L.pdf_val;
      return s;
    case TT_ENV_DIRECTIONAL:
      s.dir = f3(L.dir[0], L.dir[1], L.dir[2]);
      s.value = take(L.spectrum, l);
      s.pdf = 1.f;
      s.delta = true;
      return s;
    default: {  // TT_ENV_MAP
      rng.square(r);
      const int y = guided_bisection(L.cmf_rows, L.guide_rows, L.h, r[1]);
      const float proby = prob_from_cmf(L.cmf_rows, y);
      const float* row = L.cmf_cols + (size_t)y * L.w;
      const int x = guided_bisection(row, L.guide_cols + (size_t)y * (kEnvGuide + 1), L.w, r[0]);
      const float probx = prob_from_cmf(row, x);
      float phi0, z0, phi1, z1;
      envmap_pixel_angles(L, x, y, &phi0, &z0, &phi1, &z1);
      float r2[2];
      rng.square(r2);
      s.dir = env_world(L, to_sphere_section(r2, phi0, z0, phi1, z1));
      s.pdf = proby * probx / ((z1 - z0) * (phi1 - phi0));
      s.value = envmap_value(L, x, y, l);
      return s;
    }
  }
}

// TotalEnvironmentalRadianceField::Evaluate / EvaluatePdf (light.cxx:60-85).
__device__ __forceinline__ float3 env_eval_total(const DevScene& sc, float3 dir_out, Lambda l) {
  float3 acc = f3(0.f, 0.f, 0.f);
  for (int i = 0; i < sc.num_env; ++i) acc = acc + env_eval_one(sc.env[i], dir_out, l);
  return acc;
}
__device__ __forceinline__ float env_pdf_total(const DevScene& sc, float3 dir_out) {
  float sum = 0.f;
  for (int i = 0; i < sc.num_env; ++i) sum += env_pdf_one(sc.env[i], dir_out);
  return sum * (sc.num_env > 0 ? 1.f / sc.num_env : 1.f);
}

// ----------------------------------------------------------------------------------------
// Camera (camera.hxx:62-232).
__device__ __forceinline__ float pixel_pdf_wrt_solid_angle(const DevCamera& c, float x, float y) {
  const float area = c.xperpixel * c.yperpixel;
  const float l = sqrtf(x * x + y * y + 1.f);
  const float vz = 1.f / l;
  return 1.f / area * (l * l / fabsf(vz + kEps));
}

template <class R>
__device__ __forceinline__ DirSample camera_sample(const DevCamera& c, int unit, R& rng) {
  DirSample s;
  const int py = unit / c.xres, px = unit - py * c.xres;
  float r[2];
  rng.square(r);
  const float3 right = f3(c.right[0], c.right[1], c.right[2]), up = f3(c.up[0], c.up[1], c.up[2]),
               dir = f3(c.dir[0], c.dir[1], c.dir[2]);
  if (c.kind == TT_CAMERA_PINHOLE) {
    float3 v = f3(c.xmin + (r[0] + px) * c.xperpixel, c.ymin + (r[1] + py) * c.yperpixel, 1.f);
    v = normalize3(v);
    s.dir = right * v.x + up * v.y + dir * v.z;
    const float pdf = pixel_pdf_wrt_solid_angle(c, v.x, v.y);  // normalized components, as the reference
    s.value = f3(pdf, pdf, pdf);
    s.pdf = pdf;
    s.delta = false;
  } else {
    const float u = (r[0] + px) * c.per_pixel_delta - 1.f;
    const float v = (r[1] + py) * c.per_pixel_delta - 1.f;
    const float rho = u * u + v * v;
    float3 w = f3(2.f * u, 2.f * v, rho - 1.f) * (1.f / (1.f + rho));
    w.z = -w.z;
    if (rho <= 1.f) {
      s.dir = right * w.x + up * w.y + dir * w.z;
      s.value = f3(1.f, 1.f, 1.f);
    } else {
      s.dir = dir;
      s.value = f3(0.f, 0.f, 0.f);
    }
    s.pdf = 1.f;
    s.delta = true;
  }
  return s;
}

// PerspectiveCamera::Evaluate (camera.hxx:126-155): unit index and pdf, or unit -1.
__device__ __forceinline__ int camera_evaluate(const DevCamera& c, float3 dir_out, float* pdf) {
  *pdf = 0.f;
  if (c.kind != TT_CAMERA_PINHOLE) return -1;
  float z = dir_out.x * c.dir[0] + dir_out.y * c.dir[1] + dir_out.z * c.dir[2];
  float x = dir_out.x * c.right[0] + dir_out.y * c.right[1] + dir_out.z * c.right[2];
  float y = dir_out.x * c.up[0] + dir_out.y * c.up[1] + dir_out.z * c.up[2];
  if (z <= 0.f) return -1;
  x /= z;
  y /= z;
  const int px = (int)((x - c.xmin) / c.xperpixel);
  const int py = (int)((y - c.ymin) / c.yperpixel);
  if (px < 0 || px >= c.xres || py < 0 || py >= c.yres) return -1;
  *pdf = pixel_pdf_wrt_solid_angle(c, x, y);
  return py * c.xres + px;
}

// ----------------------------------------------------------------------------------------
// Participating media.

// Phase functions (phasefunctions.cxx:23-138).  mu is the cosine between the direction of
// travel before and after scattering.
__device__ __forceinline__ float phase_value(int kind, float g, float mu) {
  if (kind == TT_PHASE_RAYLEIGH) return (3.f / (16.f * kPi)) * (1.f + mu * mu);
  if (kind == TT_PHASE_HENYEY_GREENSTEIN) {
    const float g2 = g * g;
    const float term = 1.f + g2 - 2.f * g * mu;
    return (1.f / (4.f * kPi)) * (1.f - g2) / (sqrtf(term) * term);
  }
  return 1.f / (4.f * kPi);
}

// Evaluate at a volume vertex: wi = reverse incident direction, wo = outgoing direction.
__device__ __forceinline__ float phase_eval(int kind, float g, float3 wi, float3 wo) {
  return phase_value(kind, g, dot3(-wi, wo));
}

// Sample about the direction of travel -wi.  Rayleigh inverts its cdf in closed form;
// Henyey-Greenstein uses its textbook inversion with a series for |g| <= 1e-3.
// Directions are laid out as (sin(2 pi r1) rho, cos(2 pi r1) rho, mu) in the frame whose
// z axis is the direction of travel.
template <class R>
__device__ __forceinline__ float3 phase_sample(int kind, float g, float3 wi, R& rng, float* pdf) {
  float r[2];
  rng.square(r);
  if (kind == TT_PHASE_UNIFORM) {
    *pdf = 1.f / (4.f * kPi);
    return to_uniform_sphere(r);
  }
  float mu;
  if (kind == TT_PHASE_RAYLEIGH) {
    const float a = cbrtf(-2.f + 4.f * r[0] + sqrtf(5.f - 16.f * r[0] + 16.f * r[0] * r[0]));
    mu = a - 1.f / a;
  } else {
    const float g2 = g * g, x = 2.f * r[0] - 1.f;
    if (fabsf(g) > 1.0e-3f) {
      const float t1 = (1.f - g2) / (1.f + g * x);
      mu = (1.f + g2 - t1 * t1) / (2.f * g);
    } else {
      const float x2 = x * x;
      mu = x + 1.5f * g * (1.f - x2) - 2.f * g2 * x * (1.f - x2);
    }
  }
  mu = fminf(1.f, fmaxf(-1.f, mu));
  const float rho = sqrtf(fmaxf(0.f, 1.f - mu * mu));
  float sn, cs;
  sincosf(2.f * kPi * r[1], &sn, &cs);
  const Frame fr = frame_z(-wi);
  *pdf = phase_value(kind, g, mu);
  return normalize3(fr.to_world(f3(sn * rho, cs * rho, mu)));
}

// MediumTracker (rendering_util.hxx:18-126): up to four overlapping media in byte slots
// (0xff empty) and the current one (-1 = the vacuum of empty space, priority -1).
struct MTracker {
  uint32_t slots;
  int cur;
};
__device__ __forceinline__ MTracker load_tracker(uint2 v) { return MTracker{v.x, (int)v.y}; }
__device__ __forceinline__ uint2 store_tracker(const MTracker& t) { return make_uint2(t.slots, (unsigned)t.cur); }
__device__ __forceinline__ int medium_priority(const DevScene& sc, int m) {
  return m < 0 ? -1 : sc.media[m].priority;
}

// goingThroughSurface: crossing a surface of material `mat` along dir, with the winding
// normal ng deciding which side is entered.
__device__ __forceinline__ void going_through(const DevScene& sc, MTracker& t, float3 dir, float3 ng, int mat) {
  const DevMaterial& M = sc.materials[mat];
  int to_enter = M.med_in, to_exit = M.med_out;
  if (to_enter < 0 && to_exit < 0) return;
  if (dot3(dir, ng) > 0.f) { const int x = to_enter; to_enter = to_exit; to_exit = x; }
  if (to_exit >= 0) {
    for (int i = 0; i < 4; ++i)
      if ((int)((t.slots >> (8 * i)) & 0xffu) == to_exit) { t.slots |= 0xffu << (8 * i); break; }
    if (to_exit == t.cur) {
      int best = -1;
      for (int i = 0; i < 4; ++i) {
        const int m = (int)((t.slots >> (8 * i)) & 0xffu);
        if (m != 0xff && medium_priority(sc, best) < medium_priority(sc, m)) best = m;
      }
      t.cur = best;
    }
  }
  if (to_enter >= 0) {
    bool inserted = false;
    for (int i = 0; i < 4; ++i)
      if (((t.slots >> (8 * i)) & 0xffu) == 0xffu) {
        t.slots = (t.slots & ~(0xffu << (8 * i))) | ((uint32_t)to_enter << (8 * i));
        inserted = true;
        break;
      }
    if (inserted && medium_priority(sc, to_enter) > medium_priority(sc, t.cur)) t.cur = to_enter;
  }
}

__device__ __forceinline__ float mean3(float3 a) { return (a.x + a.y + a.z) * (1.f / 3.f); }
__device__ __forceinline__ float3 exp_neg(float3 s, float x) { return f3(expf(-s.x * x), expf(-s.y * x), expf(-s.z * x)); }

struct InteractionSample {
  float t;
  float3 weight;
  float3 sigma_s;
};

// HomogeneousMedium::SampleInteractionPoint (shader.cxx:1259-1270) with
// HomogeneousSpectralTracking (media_integrator.cxx:43-87; Kutz et al. 2017, history-aware
// collision probabilities).  `hist` is the tracking weight accumulated so far on this ray.
// At most 99 collisions are simulated; the capped sample reports an interaction with zero
// sigma_s, as the reference's emergency abort does.
__device__ __forceinline__ InteractionSample sample_interaction(const DevMedium& m, float length, float3 hist,
                                                                 Rng& rng, Lambda l) {
  InteractionSample out;
  const float3 se = take(m.sigma_ext, l);
  if (!m.scattering) {
    out.t = kLargeNumber;
    out.weight = exp_neg(se, length);
    out.sigma_s = f3(0.f, 0.f, 0.f);
    return out;
  }
  const float3 ss = take(m.sigma_s, l);
  const float maj = max3(se);
  const float3 sn = f3(maj - se.x, maj - se.y, maj - se.z);
  const float inv = 1.f / maj;
  out.t = 0.f;
  out.weight = f3(1.f, 1.f, 1.f);
  out.sigma_s = f3(0.f, 0.f, 0.f);
  for (int it = 1; it < 100; ++it) {
    out.t -= logf(rng.uniform()) * inv;
    if (out.t > length) return out;
    const float3 w = mul(out.weight, hist);
    float pt = mean3(mul(ss, w)), pn = mean3(mul(sn, w));
    const float norm = pt + pn;
    if (norm > 0.f) { pt /= norm; pn /= norm; } else { pt = pn = 0.5f; }
    if (rng.uniform() < pt) {
      out.weight = out.weight * (inv / pt);
      out.sigma_s = ss;
      return out;
    }
    out.weight = mul(out.weight, sn) * (inv / pn);
  }
  return out;
}

// VolumePdfCoefficients::transmittance of one segment (ComputeVolumePdfCoefficients,
// shader.cxx:1297-1309): the mean over the three wavelengths.
__device__ __forceinline__ float segment_tr(const DevMedium& m, float len, Lambda l) {
  return mean3(exp_neg(take(m.sigma_ext, l), len));
}

// ----------------------------------------------------------------------------------------
// Analytic spheres (Spheres, primitive.hxx:94-136).

// FillPosBoundsSphere (primitive.cxx:302-306): Gamma<float>(5).
__device__ __forceinline__ float gamma5() { return (5.f * kEpsF) / (1.f - 5.f * kEpsF); }

// Slot tag of the BVH slot arrays: triangles 0, spheres 1 (tt_bvh.h).
__device__ __forceinline__ bool is_sphere_slot(const float4* tris, int slot) {
  return __float_as_int(__ldg(&tris[3 * slot + 2]).w) != 0;
}

// Interaction on the sphere at `slot` from the outward direction (nx, ny, nz) (unit, in
// double): the position is the centre plus radius times the normal, as
// FirstIntersectionSphere and Spheres::GetLocalGeometry place it.
__device__ __forceinline__ Surf sphere_surface(const float4* tris, int slot, double nx, double ny, double nz) {
  const float4 a = __ldg(&tris[3 * slot]);
  const float4 b = __ldg(&tris[3 * slot + 1]);
  Surf s;
  s.prim = __float_as_int(a.w);
  s.material = __float_as_int(b.w);
  s.pos = f3((float)(a.x + b.x * nx), (float)(a.y + b.x * ny), (float)(a.z + b.x * nz));
  s.ng = f3((float)nx, (float)ny, (float)nz);
  s.ns_raw = s.ng;
  s.bounds = abs3(s.pos) * gamma5();
  s.n = s.ng;
  s.ns = s.ns_raw;
  s.uv = direction_uv(s.ng);
  return s;
}

// Hit at distance t along (o, d).
__device__ __forceinline__ Surf sphere_hit_surface(const float4* tris, int slot, float3 o, float3 d, float t) {
  const float4 a = __ldg(&tris[3 * slot]);
  double nx = (double)o.x + (double)t * d.x - a.x, ny = (double)o.y + (double)t * d.y - a.y,
         nz = (double)o.z + (double)t * d.z - a.z;
  const double inv = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
  return sphere_surface(tris, slot, nx * inv, ny * inv, nz * inv);
}

// ----------------------------------------------------------------------------------------
// Tabulated atmosphere (TabulatedConstituents + SphereGeometry, atmosphere.hxx:79-123,
// atmosphere.cxx:234-348).  Distances to the planet centre are taken in double: at a
// radius of thousands of km single precision would leave altitude errors of metres.
__device__ __forceinline__ float atm_altitude(const DevMedium& m, float3 p) {
  const double dx = (double)p.x - m.center[0], dy = (double)p.y - m.center[1], dz = (double)p.z - m.center[2];
  return (float)(sqrt(dx * dx + dy * dy + dz * dz) - (double)m.radius);
}

// SphereGeometry::ComputeLowestPointAlong.
__device__ __forceinline__ float3 atm_lowest_point(const DevMedium& m, float3 org, float3 dir, float len) {
  double t = -(((double)org.x - m.center[0]) * dir.x + ((double)org.y - m.center[1]) * dir.y +
               ((double)org.z - m.center[2]) * dir.z);
  if (t > len) t = len;
  else if (t < 0.0) t = 0.0;
  return f3((float)(org.x + t * dir.x), (float)(org.y + t * dir.y), (float)(org.z + t * dir.z));
}

// ComputeCollisionCoefficients with EvaluateCoeffs' sigma_t = sigma_a + sigma_s.  The row
// index truncates toward zero like the reference's (int) cast, so the first row below h0
// extrapolates.
__device__ __forceinline__ void atm_coeffs(const DevMedium& m, float alt, Lambda l, float3* ss, float3* st) {
  const float ri = (alt - m.h0) * m.inv_dh;
  if (ri >= (float)(m.rows - 1)) {
    *ss = f3(0.f, 0.f, 0.f);
    *st = f3(0.f, 0.f, 0.f);
    return;
  }
  const int i = (int)ri;
  const int bins[3] = {l.i0, l.i1, l.i2};
  float s3[3], t3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float s_, t_;
    if (i >= 0) {
      const float f = ri - (float)i;
      const float4 A = __ldg(&m.table[(size_t)i * NBINS + bins[k]]);
      const float4 B = __ldg(&m.table[(size_t)(i + 1) * NBINS + bins[k]]);
      s_ = ((1.f - f) * A.z + f * B.z) + ((1.f - f) * A.y + f * B.y);
      t_ = (1.f - f) * A.x + f * B.x;
    } else {
      const float4 A = __ldg(&m.table[bins[k]]);
      s_ = A.z + A.y;
      t_ = A.x;
    }
    s3[k] = s_;
    t3[k] = (t_ - s_) + s_;
  }
  *ss = f3(s3[0], s3[1], s3[2]);
  *st = f3(t3[0], t3[1], t3[2]);
}

// ComputeSigmaS: molecular and aerosol scattering separately.
__device__ __forceinline__ void atm_sigma_s(const DevMedium& m, float alt, Lambda l, float3* mol, float3* aer) {
  const float ri = (alt - m.h0) * m.inv_dh;
  const int i = (int)ri;
  const int bins[3] = {l.i0, l.i1, l.i2};
  float m3[3], a3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (i >= 0 && i < m.rows - 1) {
      const float f = ri - (float)i;
      const float4 A = __ldg(&m.table[(size_t)i * NBINS + bins[k]]);
      const float4 B = __ldg(&m.table[(size_t)(i + 1) * NBINS + bins[k]]);
      m3[k] = (1.f - f) * A.y + f * B.y;
      a3[k] = (1.f - f) * A.z + f * B.z;
    } else if (i < 0) {
      const float4 A = __ldg(&m.table[bins[k]]);
      m3[k] = A.y;
      a3[k] = A.z;
    } else {
      m3[k] = a3[k] = 0.f;
    }
  }
  *mol = f3(m3[0], m3[1], m3[2]);
  *aer = f3(a3[0], a3[1], a3[2]);
}

// ComputeSigmaTMajorante.
__device__ __forceinline__ float atm_majorant(const DevMedium& m, float alt) {
  const float ri = (alt - m.h0) * m.inv_dh;
  const int i = (int)ri;
  if (i >= 0 && i < m.rows - 1) {
    const float f = ri - (float)i;
    return (1.f - f) * __ldg(&m.maj[i]) + f * __ldg(&m.maj[i + 1]);
  }
  return i < 0 ? __ldg(&m.maj[0]) : 0.f;
}

// AtmosphereTemplate::ComputeMajorante: at the segment's lowest point, clamped to h0.
__device__ __forceinline__ float atm_segment_majorant(const DevMedium& m, float3 org, float3 dir, float len) {
  return atm_majorant(m, fmaxf(m.h0, atm_altitude(m, atm_lowest_point(m, org, dir, len))));
}

__device__ __forceinline__ void history_probabilities(float3 w, float3 a, float3 b, float* pa, float* pb) {
  *pa = mean3(mul(a, w));
  *pb = mean3(mul(b, w));
  const float norm = *pa + *pb;
  if (norm > 0.f) { *pa /= norm; *pb /= norm; } else { *pa = *pb = 0.5f; }
}

// SpectralTracking (media_integrator.cxx:90-147) against the segment majorant; the weight
// starts at `initial`, as in the reference.  At most 999 collisions.
__device__ __forceinline__ InteractionSample atm_tracking(const DevMedium& m, float3 org, float3 dir, float len,
                                                          float3 initial, Rng& rng, Lambda l) {
  InteractionSample out;
  out.t = 0.f;
  out.weight = initial;
  out.sigma_s = f3(0.f, 0.f, 0.f);
  const float maj = atm_segment_majorant(m, org, dir, len);
  if (!(maj > 0.f)) {
    out.t = kLargeNumber;
    return out;
  }
  const float mfp = 1.f / maj;
  for (int it = 1; it < 1000; ++it) {
    out.t -= logf(rng.uniform()) * mfp;
    if (out.t > len) return out;
    float3 ss, st;
    atm_coeffs(m, atm_altitude(m, org + dir * out.t), l, &ss, &st);
    const float3 sn = f3(fmaxf(0.f, maj - st.x), fmaxf(0.f, maj - st.y), fmaxf(0.f, maj - st.z));
    float pt, pn;
    history_probabilities(out.weight, ss, sn, &pt, &pn);
    if (rng.uniform() < pt) {
      out.weight = out.weight * (mfp / pt);
      out.sigma_s = ss;
      return out;
    }
    out.weight = mul(out.weight, sn) * (mfp / pn);
  }
  return out;
}

// EstimateTransmission (media_integrator.cxx:150-187): ratio tracking with Russian roulette
// after five steps.  Capped at 2^16 steps (error bit ERR_CROSSINGS).
__device__ __forceinline__ float3 atm_transmission(const DevMedium& m, float3 org, float3 dir, float len, Rng& rng,
                                                   Lambda l, unsigned int* err) {
  float3 est = f3(1.f, 1.f, 1.f);
  const float maj = atm_segment_majorant(m, org, dir, len);
  if (!(maj > 0.f)) return est;
  const float inv = 1.f / maj;
  float t = 0.f;
  for (int it = 0;; ++it) {
    if (it >= (1 << 16)) {
      atomicOr(err, ERR_CROSSINGS);
      return f3(0.f, 0.f, 0.f);
    }
    t -= logf(rng.uniform()) * inv;
    if (t > len) break;
    float3 ss, st;
    atm_coeffs(m, atm_altitude(m, org + dir * t), l, &ss, &st);
    est = mul(est, f3(maj - st.x, maj - st.y, maj - st.z)) * inv;
    const float w = max3(est);
    if (!(w > 0.f)) break;
    if (it < 5) continue;
    const float p = fminf(w, 1.f);
    if (rng.uniform() < p) est = est * (1.f / p);
    else return f3(0.f, 0.f, 0.f);
  }
  return est;
}

// Medium-generic operations on a segment (org, dir, len) and at a volume vertex.
__device__ __forceinline__ InteractionSample medium_interaction(const DevMedium& m, float3 org, float3 dir, float len,
                                                                float3 hist, Rng& rng, Lambda l) {
  if (m.kind == TT_MEDIUM_ATMOSPHERE) return atm_tracking(m, org, dir, len, hist, rng, l);
  return sample_interaction(m, len, hist, rng, l);
}
__device__ __forceinline__ float medium_segment_tr(const DevMedium& m, float3 org, float3 dir, float len, Lambda l) {
  if (m.kind == TT_MEDIUM_ATMOSPHERE) {
    // AtmosphereTemplate::ComputeVolumePdfCoefficients (atmosphere.cxx:66-80): the
    // majorant at the lowest point, unclamped, as a homogeneous extinction.
    return expf(-atm_majorant(m, atm_altitude(m, atm_lowest_point(m, org, dir, len))) * len);
  }
  return segment_tr(m, len, l);
}
__device__ __forceinline__ float3 medium_transmission(const DevMedium& m, float3 org, float3 dir, float len, Rng& rng,
                                                      Lambda l, unsigned int* err) {
  if (m.kind == TT_MEDIUM_ATMOSPHERE) return atm_transmission(m, org, dir, len, rng, l, err);
  return exp_neg(take(m.sigma_ext, l), len);
}

// SimpleCombined (phasefunctions.cxx:206-273) of Rayleigh (molecules) and
// Henyey-Greenstein (aerosols) in proportion to their sigma_s at the vertex.
struct CombinedPhase {
  float sel0, sel1;
  float3 w0, w1;
};
__device__ __forceinline__ CombinedPhase atm_phase(const DevMedium& m, float3 pos, Lambda l) {
  CombinedPhase c;
  atm_sigma_s(m, atm_altitude(m, pos), l, &c.w0, &c.w1);
  const float s0 = c.w0.x + c.w0.y + c.w0.z, s1 = c.w1.x + c.w1.y + c.w1.z;
  if (s0 + s1 > 0.f) {
    c.sel0 = s0 / (s0 + s1);
    c.sel1 = s1 / (s0 + s1);
    const float3 tot = c.w0 + c.w1;
    const float3 inv = f3(1.f / tot.x, 1.f / tot.y, 1.f / tot.z);
    c.w0 = mul(c.w0, inv);
    c.w1 = mul(c.w1, inv);
  } else {
    c.sel0 = c.sel1 = 0.5f;
  }
  return c;
}

// Phase function value per wavelength and pdf at a volume vertex at pos.
__device__ __forceinline__ float3 medium_phase_eval(const DevMedium& m, float3 pos, float3 wi, float3 wo, Lambda l,
                                                    float* pdf) {
  if (m.kind != TT_MEDIUM_ATMOSPHERE) {
    const float v = phase_eval(m.phase, m.g, wi, wo);
    *pdf = v;
    return f3(v, v, v);
  }
  const CombinedPhase c = atm_phase(m, pos, l);
  const float p0 = phase_eval(TT_PHASE_RAYLEIGH, 0.f, wi, wo), p1 = phase_eval(TT_PHASE_HENYEY_GREENSTEIN, m.g, wi, wo);
  *pdf = c.sel0 * p0 + c.sel1 * p1;
  return c.w0 * p0 + c.w1 * p1;
}

template <class R>
__device__ __forceinline__ float3 medium_phase_sample(const DevMedium& m, float3 pos, float3 wi, R& rng, Lambda l,
                                                      float3* value, float* pdf) {
  if (m.kind != TT_MEDIUM_ATMOSPHERE) {
    const float3 d = phase_sample(m.phase, m.g, wi, rng, pdf);
    *value = f3(*pdf, *pdf, *pdf);
    return d;
  }
  const CombinedPhase c = atm_phase(m, pos, l);
  const bool aer = !(rng.uniform() >= c.sel1);  // TowerSampling over (molecules, aerosols)
  float pk;
  const float3 d = aer ? phase_sample(TT_PHASE_HENYEY_GREENSTEIN, m.g, wi, rng, &pk)
                       : phase_sample(TT_PHASE_RAYLEIGH, 0.f, wi, rng, &pk);
  const float po = aer ? phase_eval(TT_PHASE_RAYLEIGH, 0.f, wi, d) : phase_eval(TT_PHASE_HENYEY_GREENSTEIN, m.g, wi, d);
  const float p0 = aer ? po : pk, p1 = aer ? pk : po;
  *value = c.w0 * p0 + c.w1 * p1;
  *pdf = c.sel0 * p0 + c.sel1 * p1;
  return d;
}

}  // namespace tt
