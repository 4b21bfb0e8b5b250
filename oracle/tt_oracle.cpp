// ORACLE -- test infrastructure only (see tt_oracle.h).
//
// A CPU, double-precision restatement of ToyTrace's forward path tracer with next-event
// estimation (`--algo pt`).  Each function names the reference code it restates; paths
// are relative to the reference project root.  Geometry is single precision as in the
// reference (Mesh stores float vertices, primitive.hxx:62-72); everything else is double.
//
// Random numbers: the reference draws from two default-seeded PCG32 generators per
// worker (Sampler's sequence and its RandGen, sampler.hxx:93-121), so its streams are not
// reproducible per pixel.  Here every path owns one PCG32 stream, seeded with
// (seed, sample_index * num_pixels + pixel), and draws happen in the reference's call
// order.  The CUDA tracer uses the same streams, which makes per-path comparison possible.
#include "tt_oracle.h"
#include "../naivetrace_b200/csrc/tt_tables.h"
#include "../naivetrace_b200/csrc/tt_sobol_data.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace orc {

constexpr double Pi = 3.14159265358979323846264338327950288;
constexpr double Eps = std::numeric_limits<double>::epsilon();        // vec3f.hxx:15
constexpr float EpsF = std::numeric_limits<float>::epsilon();         // vec3f.hxx:16
constexpr double LargeNumber = std::numeric_limits<double>::max() / 16;  // vec3f.hxx:22
constexpr double Infinity = std::numeric_limits<double>::infinity();
constexpr int NBINS = 36;

static thread_local std::string g_err;

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, double s) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double Dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 Cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double Length(V3 a) { return std::sqrt(Dot(a, a)); }
inline V3 Normalized(V3 a) { return a / Length(a); }
inline V3 Abs(V3 a) { return {std::abs(a.x), std::abs(a.y), std::abs(a.z)}; }
inline double Sqr(double a) { return a * a; }
inline double Sign(double x) { return std::copysign(1.0, x); }  // util.hxx:116-119

struct F3 { float x, y, z; };
inline F3 Ff(V3 a) { return {(float)a.x, (float)a.y, (float)a.z}; }

struct S3 {
  double v[3] = {0, 0, 0};
  S3() = default;
  explicit S3(double a) { v[0] = v[1] = v[2] = a; }
  S3(double a, double b, double c) { v[0] = a; v[1] = b; v[2] = c; }
  double& operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
  bool IsZero() const { return v[0] == 0 && v[1] == 0 && v[2] == 0; }
  double Max() const { return std::max(v[0], std::max(v[1], v[2])); }
  double Sum() const { return v[0] + v[1] + v[2]; }
};
inline S3 operator*(S3 a, S3 b) { return {a[0] * b[0], a[1] * b[1], a[2] * b[2]}; }
inline S3 operator*(double s, S3 a) { return {s * a[0], s * a[1], s * a[2]}; }
inline S3 operator*(S3 a, double s) { return {s * a[0], s * a[1], s * a[2]}; }
inline S3 operator/(S3 a, double s) { return {a[0] / s, a[1] / s, a[2] / s}; }
inline S3 operator+(S3 a, S3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }

// Listing 3 of Duff et al. (2017), as used by OrthogonalSystemZAligned (vec3f.hxx:240-258).
// Columns X, Y, Z.
struct Frame {
  V3 X, Y, Z;
  V3 ToWorld(V3 v) const { return X * v.x + Y * v.y + Z * v.z; }
  V3 ToLocal(V3 w) const { return {Dot(X, w), Dot(Y, w), Dot(Z, w)}; }
};
inline Frame OrthogonalSystemZAligned(V3 z) {
  Frame f;
  f.Z = z;
  const double sign = std::copysign(1.0, z.z);
  const double a = -1.0 / (sign + z.z);
  const double b = z.x * z.y * a;
  f.X = {1.0 + sign * z.x * z.x * a, sign * b, -sign * z.x};
  f.Y = {b, sign + z.y * z.y * a, -z.y};
  return f;
}

// ---------------------------------------------------------------------------------------
// PCG32 (O'Neill 2014), with the interface of the pcg32 submodule the reference uses
// (RandGen, sampler.cxx:366-393): seed(initstate, initseq), nextUInt, nextDouble
// (32 random bits in the mantissa), nextUInt(bound) with rejection of the biased range.
struct Pcg32 {
  uint64_t state = 0x853c49e6748fea9bULL, inc = 0xda3e39cb94b95bdbULL;
  void Seed(uint64_t initstate, uint64_t initseq) {
    state = 0u;
    inc = (initseq << 1u) | 1u;
    NextUInt();
    state += initstate;
    NextUInt();
  }
  uint32_t NextUInt() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
  }
  double NextDouble() { return (double)NextUInt() * (1.0 / 4294967296.0); }
  uint32_t NextBounded(uint32_t bound) {
    uint32_t threshold = (~bound + 1u) % bound;
    for (;;) {
      uint32_t r = NextUInt();
      if (r >= threshold) return r % bound;
    }
  }
};

// Per-path stream: PCG32 streams whose increments differ by small amounts are strongly
// correlated, so the (seed, path index) pair is first scrambled with the SplitMix64
// finalizer (Steele, Lea and Flood 2014) into the initial state and the stream selector.
inline uint64_t SplitMix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
inline void SeedPath(Pcg32& g, uint64_t seed, uint64_t path) {
  const uint64_t s1 = SplitMix64(seed ^ SplitMix64(path));
  const uint64_t s2 = SplitMix64(s1 ^ 0xd1b54a32d192ed03ULL);
  g.Seed(s1, s2);
}

// SobolMatrixMult (sampler.cxx:224-234): the point index's bits select generator columns.
inline double SobolMult(uint32_t point, const uint32_t* m) {
  uint32_t c = 0;
  for (int i = 0; i < 32; ++i, point >>= 1) c ^= (point & 1u) ? m[i] : 0u;
  return (double)c / 4294967296.0;
}

// One stream per path; Uniform01 / UniformUnitSquare / UniformInt as Sampler and RandGen.
// With `qmc` set it is QuasiRandomSequence (sampler.cxx:254-331): point index, per-pixel
// rotation, subsequence (SetSubsequenceId: dimension offset id << 6, draw counter); the
// k-th 1D draw is dimension offset + 2 + k for k < 62, then PCG32; 2D draws are dimensions
// offset and offset + 1; every draw is rotated modulo 1.  UniformInt is always PCG32.
struct Sampler {
  Pcg32 g;
  const uint32_t* qmc = nullptr;  // generator matrices, 32 columns per dimension
  uint32_t point = 0, offset = 0, sub = 0;
  double rot[2] = {0., 0.};
  void SetSubsequenceId(uint32_t id) { offset = id << 6; sub = 0; }
  static double Wrap(double x) { return x >= 1. ? x - 1. : x; }
  double Uniform01() {
    if (!qmc) return g.NextDouble();
    const double x = sub < 62 ? SobolMult(point, qmc + 32 * (size_t)(offset + 2 + sub)) : g.NextDouble();
    ++sub;
    return Wrap(x + rot[0]);
  }
  void UniformUnitSquare(double r[2]) {
    if (!qmc) {
      r[0] = g.NextDouble();
      r[1] = g.NextDouble();
      return;
    }
    r[0] = Wrap(SobolMult(point, qmc + 32 * (size_t)offset) + rot[0]);
    r[1] = Wrap(SobolMult(point, qmc + 32 * (size_t)(offset + 1)) + rot[1]);
  }
  int UniformInt(int a, int b_inclusive) {  // RandGen::UniformInt, sampler.cxx:384-391
    return a + (int)g.NextBounded((uint32_t)(b_inclusive + 1 - a));
  }
};

// ---------------------------------------------------------------------------------------
// Warps, sampler.cxx:6-124.
inline V3 ToUniformSphere(const double r[2]) {
  double z = 1. - 2. * r[1];
  double s = std::sqrt(r[1] * (1. - r[1]));
  double omega = 2. * Pi * r[0];
  return {2. * std::cos(omega) * s, 2. * std::sin(omega) * s, z};
}
inline V3 ToUniformHemisphere(const double r[2]) {
  V3 v = ToUniformSphere(r);
  v.z = v.z >= 0. ? v.z : -v.z;
  return v;
}
inline V3 ToUniformSphereSection(double cos_opening, const double r[2]) {
  double z = 1. - r[1] * (1. - cos_opening);
  double s = std::sqrt(1. - z * z);
  double omega = 2. * Pi * r[0];
  return {std::cos(omega) * s, std::sin(omega) * s, z};
}
inline V3 ToUniformSphereSection(const double r[2], double phi0, double z0, double phi1, double z1) {
  const double z = z0 + r[1] * (z1 - z0);
  double s = std::sqrt(1. - z * z);
  s = std::isnan(s) ? 0. : s;
  double omega = phi0 + (phi1 - phi0) * r[0];
  return {std::cos(omega) * s, std::sin(omega) * s, z};
}
inline V3 ToCosHemisphere(const double r[2]) {
  double rho = std::sqrt(1. - r[0]);
  double z = std::sqrt(r[0]);
  double omega = 2. * Pi * r[1];
  return {std::cos(omega) * rho, std::sin(omega) * rho, z};
}
inline V3 ToTriangleBarycentricCoords(const double r[2]) {
  double s = std::sqrt(r[0]);
  return {1. - s, (1. - r[1]) * s, r[1] * s};
}
inline V3 ToUniformDisc(const double r[2]) {
  double s = std::sqrt(r[1]);
  double omega = 2. * Pi * r[0];
  return {s * std::cos(omega), s * std::sin(omega), 0};
}
// sampler.hxx:133-144
inline double PowerHeuristic(double p, double other) {
  double pp = p * p;
  return pp / (pp + other * other + Eps);
}
// sampler.hxx:147-166
inline int TowerSampling4(const double* probs, double r) {
  int n = 3;
  while (r >= probs[n] && n > 0) { r -= probs[n]; --n; }
  return n;
}
// sampler.hxx:169-205 (float CMFs of the env map)
inline int TowerSamplingBisection(const float* cmf, int size, float r) {
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
inline float ProbFromCmf(const float* cmf, int idx) { return cmf[idx] - (idx > 0 ? cmf[idx - 1] : 0.f); }

// ---------------------------------------------------------------------------------------
// Spectral, spectral.cxx:81-140.
inline void LinComb3(double* dst, double a, const double* sa, double b, const double* sb, double c,
                     const double* sc, const int32_t* idx) {
  for (int i = 0; i < 3; ++i) dst[i] = a * sa[idx[i]] + b * sb[idx[i]] + c * sc[idx[i]];
}
inline void LinCombN(double* dst, double a, const double* sa, double b, const double* sb, double c,
                     const double* sc) {
  for (int i = 0; i < NBINS; ++i) dst[i] = a * sa[i] + b * sb[i] + c * sc[i];
}
// Smits' case split (spectral.cxx:81-115) over either all bins or a selection.
template <class F>
inline void SmitsCases(double red, double green, double blue, F lincomb) {
  if (red <= green && red <= blue) {
    if (green <= blue) lincomb(red, TT_SMITS_WHITE, green - red, TT_SMITS_CYAN, blue - green, TT_SMITS_BLUE);
    else lincomb(red, TT_SMITS_WHITE, blue - red, TT_SMITS_CYAN, green - blue, TT_SMITS_GREEN);
  } else if (green <= red && green <= blue) {
    if (red <= blue) lincomb(green, TT_SMITS_WHITE, red - green, TT_SMITS_MAGENTA, blue - red, TT_SMITS_BLUE);
    else lincomb(green, TT_SMITS_WHITE, blue - green, TT_SMITS_MAGENTA, red - blue, TT_SMITS_RED);
  } else {
    if (red <= green) lincomb(blue, TT_SMITS_WHITE, red - blue, TT_SMITS_YELLOW, green - red, TT_SMITS_GREEN);
    else lincomb(blue, TT_SMITS_WHITE, green - blue, TT_SMITS_YELLOW, red - green, TT_SMITS_RED);
  }
}
inline S3 RGBToSpectralSelection(const double rgb[3], const int32_t idx[3]) {
  S3 ret;
  SmitsCases(rgb[0], rgb[1], rgb[2], [&](double a, int ia, double b, int ib, double c, int ic) {
    LinComb3(ret.v, a, kSmitsBasis[ia], b, kSmitsBasis[ib], c, kSmitsBasis[ic], idx);
  });
  return ret;
}
inline void SpectralSelectionToRGB(const S3& val, const int32_t idx[3], double rgb[3]) {
  for (int i = 0; i < 3; ++i) {
    rgb[i] = 0;
    for (int j = 0; j < 3; ++j) rgb[i] += val[j] * kSpectrumToRgb[i][idx[j]];
  }
}
inline S3 Take(const float* spec, const int32_t idx[3]) { return {spec[idx[0]], spec[idx[1]], spec[idx[2]]}; }
inline S3 TakeD(const double* spec, const int32_t idx[3]) { return {spec[idx[0]], spec[idx[1]], spec[idx[2]]}; }

// ---------------------------------------------------------------------------------------
// Reflection/refraction, shader_physics.hxx:10-148.
inline V3 Reflected(V3 wi, V3 n) { return 2. * Dot(wi, n) * n - wi; }
inline bool Refracted(V3 wi, V3 m, double eta, V3* out) {
  const double c = Dot(m, wi);
  const double t1 = 1. - c * c;
  const double t2 = 1.0 - eta * eta * t1;
  if (t2 < 0.) return false;
  const double s = Dot(wi, m) >= 0. ? 1.0 : -1.0;
  const double t3 = std::sqrt(t2);
  *out = (eta * c - s * t3) * m - eta * wi;
  return true;
}
inline V3 HalfVector(V3 wi, V3 wo) {
  V3 ret = wo + wi;
  double norm = Length(ret);
  if (norm > 0) return ret / norm;
  return OrthogonalSystemZAligned(wi).X;
}
inline bool HalfVectorRefracted(V3 wi, V3 wo, double eta, V3* out) {
  V3 ret = -(eta * wi + wo);
  double norm = Length(ret);
  if (norm > 0) ret = ret / norm; else ret = wi;
  if (Dot(ret, wi) * Dot(ret, wo) < 0.) { *out = ret; return true; }
  return false;
}
inline double HalfVectorPdfToReflectedPdf(double pdf_wh, double wh_dot_in) {
  return pdf_wh * 0.25 / (std::abs(wh_dot_in) + Eps);
}
inline double FresnelReflectivity(double cs_i, double cs_t, double eta) {
  double rs_nom = eta * cs_i - cs_t, rs_den = eta * cs_i + cs_t;
  double rp_nom = eta * cs_t - cs_i, rp_den = eta * cs_t + cs_i;
  return 0.5 * (Sqr(rs_nom / rs_den) + Sqr(rp_nom / rp_den));
}
inline double FresnelReflectivityWalter(double cos_n_wi, double eta) {
  double c = std::abs(cos_n_wi);
  double tmp = Sqr(1.0 / eta) - 1.0 + c * c;
  if (tmp < 0.) return 1.;
  double g = std::sqrt(tmp);
  if ((g == 0.) & (c == 0.)) return 1.;
  double nom = c * (g + c) - 1.;
  double denom = c * (g - c) + 1.;
  return 0.5 * Sqr((g - c) / (g + c)) * (1. + Sqr(nom / denom));
}

// Beckmann NDF, G terms and VNDF selection, normaldistributionfunction.hxx:8-127.
struct Beckman {
  double alpha;
  double EvalByHalfVector(double cs) const {
    if (cs <= 0.) return 0.;
    const double t1 = (cs * cs - 1.) / (cs * cs * alpha * alpha);
    const double t2 = alpha * alpha * cs * cs * cs * cs * Pi;
    return std::exp(t1) / t2;
  }
  V3 SampleHalfVector(const double r[2]) const {
    const double t1 = -alpha * alpha * std::log(r[0]);
    const double t = 1 / (t1 + 1);
    const double z = std::sqrt(t);
    const double rho = std::sqrt(1 - t);
    const double omega = 2 * Pi * r[1];
    return {std::cos(omega) * rho, std::sin(omega) * rho, z};
  }
};
inline double G1VCavity(double cos_v_m, double cos_v_n, double cos_n_m) {
  if (cos_v_m * cos_v_n < 0.) return 0.;
  return std::min(1., 2. * std::abs(cos_n_m * cos_v_n) / (std::abs(cos_v_m) + Eps));
}
inline double G2VCavity(double wh_dot_in, double wh_dot_out, double ns_dot_in, double ns_dot_out, double ns_dot_wh) {
  return std::min(G1VCavity(wh_dot_in, ns_dot_in, ns_dot_wh), G1VCavity(wh_dot_out, ns_dot_out, ns_dot_wh));
}
// G2VCavityTransmissive, normaldistributionfunction.hxx:87-94.
inline double G2VCavityTransmissive(double wh_dot_in, double wh_dot_out, double ns_dot_in, double ns_dot_out,
                                    double ns_dot_wh) {
  return std::max(G1VCavity(wh_dot_in, ns_dot_in, ns_dot_wh) + G1VCavity(wh_dot_out, ns_dot_out, ns_dot_wh) - 1., 0.);
}
// HalfVectorPdfToTransmittedPdf, shader_physics.hxx:80-88.
inline double HalfVectorPdfToTransmittedPdf(double pdf_wh, double eta, double dot_wi_wh, double dot_wo_wh) {
  double denom = eta * dot_wi_wh + dot_wo_wh;
  if (denom == 0.) return pdf_wh;
  denom *= denom;
  return pdf_wh * std::abs(dot_wo_wh) / denom;
}
inline double ClampDot(V3 a, V3 b) { return std::max(0., Dot(a, b)); }
constexpr double WI_BELOW_HORIZON_FIX_FACTOR = 1.e-6;
inline void VndfSample(V3& wh, V3 wi, double r) {
  V3 whp{-wh.x, -wh.y, wh.z};
  double prob = ClampDot(wi, whp) / (ClampDot(wi, wh) + ClampDot(wi, whp) + WI_BELOW_HORIZON_FIX_FACTOR);
  if (r < prob) wh = whp;
}
inline double VndfPdf(double ndf_val, V3 wh, V3 wi) {
  V3 whp{-wh.x, -wh.y, wh.z};
  const double a = ClampDot(wi, whp);
  const double b = ClampDot(wh, wi);
  const double prob = (2. * b + WI_BELOW_HORIZON_FIX_FACTOR) / (b + a + WI_BELOW_HORIZON_FIX_FACTOR);
  return ndf_val * std::abs(wh.z) * prob;
}

// ---------------------------------------------------------------------------------------
// Surface interaction, scene.hxx:77-95, scene.cxx:229-261.
struct Surf {
  int prim = -1;
  V3 barry;            // HitId::barry
  V3 pos;
  V3 geometry_normal;  // raw winding normal
  V3 smooth_normal;
  V3 normal;           // oriented toward where the incident ray came from
  V3 shading_normal;
  V3 pos_bounds;
  float tex_u = 0.f, tex_v = 0.f;        // SurfaceInteraction::tex_coord
  const struct Texture* tex = nullptr;   // the material's diffuse texture, if any
};

// Texture (texture.hxx:15-117): linear RGB, row 0 at the top; UvToPixel wraps the
// coordinates to [0, 1) with v up, GetPixel returns the texel.
struct Texture {
  int w = 0, h = 0;
  std::vector<float> rgb;
  void Lookup(float u, float v, double out[3]) const {
    float dummy;
    u = std::modf(u, &dummy);
    v = std::modf(v, &dummy);
    if (u < 0.f) u = 1.f + u;
    if (v < 0.f) v = 1.f + v;
    if (u > 1.f - EpsF) u -= EpsF;
    if (v > 1.f - EpsF) v -= EpsF;
    const int x = std::min(std::max((int)(u * w), 0), w - 1);
    const int y = std::min(std::max(h - (int)(v * h) - 1, 0), h - 1);
    const float* p = &rgb[3 * ((size_t)y * w + x)];
    out[0] = p[0];
    out[1] = p[1];
    out[2] = p[2];
  }
};

// KartesianToSpherical (third component up, vec3f.hxx:298-321) and SphericalToUv
// (vec3f.hxx:286-295) in float, as FirstIntersectionSphere maps a sphere hit's normal
// (embreeaccelerator.cxx:258).
inline void DirectionToUv(V3 d, float* u, float* v) {
  const float x = (float)d.x, z = (float)d.y, y = (float)d.z;
  const float ax = std::abs(x), az = std::abs(z);
  const float r = std::sqrt(x * x + y * y + z * z);
  const float theta = std::acos(std::min(1.f, std::max(-1.f, y / r)));
  float phi;
  const float pi = (float)Pi;
  if (ax > az) {
    phi = std::atan2(z, ax);
    phi = (x > 0.f) ? phi : pi - phi;
  } else {
    phi = std::atan2(x, az);
    phi = (z > 0.f) ? (pi / 2.f) - phi : (3.f / 2.f * pi) + phi;
  }
  *u = phi / (2.f * pi);
  *v = theta / pi;
}

inline V3 AntiSelfIntersectionOffset(const Surf& s, V3 exitant_dir) {
  const V3 n = s.geometry_normal;
  const double delta = Dot(s.pos_bounds, Abs(n));
  return delta * (Dot(exitant_dir, n) > 0. ? 1. : -1.) * n;
}

// util::Gamma<float>(7), util.hxx:124-127 (note: uses the full float epsilon).
inline double Gamma7() { return (7 * (double)EpsF) / (1 - 7 * (double)EpsF); }

struct EnvLight {
  int kind;
  double spectrum[NBINS];
  V3 dir;
  double scalar, scalar2;
  // Sun
  Frame frame;
  double cos_opening, pdf_val;
  double sun_emission[NBINS];
  // Dome
  V3 down_dir;
  // Env map (float data as in EnvMapLight, light.cxx:88-189)
  int w = 0, h = 0;
  std::vector<float> tex;
  std::vector<float> cmf_rows, cmf_cols;
  float fX[3], fY[3], fZ[3];  // float frame columns
};

struct Material {
  tt_material m;
};

struct Camera {
  int kind;
  V3 pos, up, dir, right;
  int xres, yres;
  double xmin, ymin, xperpixel, yperpixel;
  double per_pixel_delta;
};

// ---------------------------------------------------------------------------------------
// BVH over triangles for the oracle's own closest-hit / occlusion queries.  Binned SAH,
// double-precision slab and watertight triangle tests (Woop, Benthin, Wald 2013).
struct BNode {
  double lo[3], hi[3];
  int left = -1, right = -1, start = 0, count = 0;
};

struct MediumDesc {
  int kind = TT_MEDIUM_HOMOGENEOUS;
  int priority;
  double sigma_s[NBINS], sigma_a[NBINS], sigma_ext[NBINS];
  bool is_scattering;
  int phase;
  double g;
  // Atmosphere (TabulatedConstituents + SphereGeometry, atmosphere.hxx:79-123), km units.
  V3 center;
  double radius = 0;
  int n = 0;                                  // altitude rows
  double h0 = 0, dh = 1, inv_dh = 1;
  std::vector<double> sig_t, sig_mol, sig_aer;  // n x NBINS
  std::vector<double> maj;                    // per-row majorant, non-increasing with altitude
};

struct Scene {
  std::vector<uint32_t> sobol;     // quasi-random generator matrices (pt2 with qmc), else empty
  // Primitives: triangles 0 .. ntri-1, then spheres (global id ntri + i).
  uint32_t ntri = 0;
  std::vector<V3> sph_c;           // sphere centres (from float)
  std::vector<double> sph_r;       // sphere radii (from float)
  std::vector<V3> tv0, tv1, tv2;   // triangle vertices as double (from float)
  std::vector<F3> vert, nrm;
  std::vector<uint32_t> idx, mat_of_tri;  // mat_of_tri: per primitive (triangles, then spheres)
  bool has_normals = false;
  std::vector<float> uv;           // 2 per vertex (Mesh::uvs), empty when none were given
  std::vector<Texture> textures;
  std::vector<Material> materials;
  std::vector<EnvLight> env;
  std::vector<tt_point_light> points;
  std::vector<int> area_lights;    // global primitive id per area light number
  Camera cam;
  double bb_lo[3], bb_hi[3];
  double diag = 0, long_distance = 0;
  V3 box_center;
  double type_probs[4];            // ENV, AREA, POINT, VOLUME (light.hxx:322-326)
  double in_class[4];
  tt_params params;
  // Surfaces and medium boundaries are separate triangle sets with their own BVH, as in
  // Scene::BuildAccelStructure (scene.cxx:116-141).  Entries are global triangle indices.
  struct TriSet {
    std::vector<int> tris;
    std::vector<BNode> nodes;
    std::vector<int> order;
  } surf, vol;
  std::vector<MediumDesc> media;
};

inline bool IsSphere(const Scene& s, int prim) { return (uint32_t)prim >= s.ntri; }

inline void TriBounds(const Scene& s, int t, double lo[3], double hi[3]) {
  if (IsSphere(s, t)) {
    const V3 c = s.sph_c[t - s.ntri];
    const double r = s.sph_r[t - s.ntri];
    for (int k = 0; k < 3; ++k) { lo[k] = c[k] - r; hi[k] = c[k] + r; }
    return;
  }
  for (int k = 0; k < 3; ++k) {
    lo[k] = std::min(s.tv0[t][k], std::min(s.tv1[t][k], s.tv2[t][k]));
    hi[k] = std::max(s.tv0[t][k], std::max(s.tv1[t][k], s.tv2[t][k]));
  }
}

static double HalfArea(const double lo[3], const double hi[3]) {
  double d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
  if (d0 < 0 || d1 < 0 || d2 < 0) return 0;
  return d0 * d1 + d1 * d2 + d2 * d0;
}

static void BuildBvh(const Scene& sc, Scene::TriSet& s) {
  const int n = (int)s.tris.size();
  s.order.resize(n);
  const size_t np = sc.mat_of_tri.size();
  std::vector<double> cen(3 * np), blo(3 * np), bhi(3 * np);
  for (int i = 0; i < n; ++i) {
    const int g = s.tris[i];
    s.order[i] = g;
    TriBounds(sc, g, &blo[3 * (size_t)g], &bhi[3 * (size_t)g]);
    for (int k = 0; k < 3; ++k) cen[3 * (size_t)g + k] = 0.5 * (blo[3 * (size_t)g + k] + bhi[3 * (size_t)g + k]);
  }
  s.nodes.clear();
  s.nodes.reserve(2 * (size_t)std::max(n, 1));
  struct Task { int node, start, count; };
  std::vector<Task> stack;
  s.nodes.push_back(BNode{});
  stack.push_back({0, 0, n});
  constexpr int NB = 16;
  while (!stack.empty()) {
    Task t = stack.back();
    stack.pop_back();
    BNode& nd = s.nodes[t.node];
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 3; ++k) { nd.lo[k] = 1e300; nd.hi[k] = -1e300; }
    for (int i = t.start; i < t.start + t.count; ++i) {
      int tri = s.order[i];
      for (int k = 0; k < 3; ++k) {
        nd.lo[k] = std::min(nd.lo[k], blo[3 * tri + k]);
        nd.hi[k] = std::max(nd.hi[k], bhi[3 * tri + k]);
        clo[k] = std::min(clo[k], cen[3 * tri + k]);
        chi[k] = std::max(chi[k], cen[3 * tri + k]);
      }
    }
    if (t.count <= 4) { nd.start = t.start; nd.count = t.count; continue; }
    int best_axis = -1, best_split = -1;
    double best_cost = 1e300;
    for (int axis = 0; axis < 3; ++axis) {
      double ext = chi[axis] - clo[axis];
      if (ext <= 0) continue;
      int cnt[NB] = {0};
      double bl[NB][3], bh[NB][3];
      for (int b = 0; b < NB; ++b)
        for (int k = 0; k < 3; ++k) { bl[b][k] = 1e300; bh[b][k] = -1e300; }
      for (int i = t.start; i < t.start + t.count; ++i) {
        int tri = s.order[i];
        int b = std::min(NB - 1, (int)(NB * (cen[3 * tri + axis] - clo[axis]) / ext));
        cnt[b]++;
        for (int k = 0; k < 3; ++k) {
          bl[b][k] = std::min(bl[b][k], blo[3 * tri + k]);
          bh[b][k] = std::max(bh[b][k], bhi[3 * tri + k]);
        }
      }
      double rl[NB][3], rh[NB][3];
      int rc[NB];
      double al[3] = {1e300, 1e300, 1e300}, ah[3] = {-1e300, -1e300, -1e300};
      int ac = 0;
      for (int b = NB - 1; b >= 1; --b) {
        for (int k = 0; k < 3; ++k) { al[k] = std::min(al[k], bl[b][k]); ah[k] = std::max(ah[k], bh[b][k]); }
        ac += cnt[b];
        for (int k = 0; k < 3; ++k) { rl[b][k] = al[k]; rh[b][k] = ah[k]; }
        rc[b] = ac;
      }
      for (int k = 0; k < 3; ++k) { al[k] = 1e300; ah[k] = -1e300; }
      ac = 0;
      for (int b = 0; b < NB - 1; ++b) {
        for (int k = 0; k < 3; ++k) { al[k] = std::min(al[k], bl[b][k]); ah[k] = std::max(ah[k], bh[b][k]); }
        ac += cnt[b];
        if (ac == 0 || rc[b + 1] == 0) continue;
        double cost = ac * HalfArea(al, ah) + rc[b + 1] * HalfArea(rl[b + 1], rh[b + 1]);
        if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = b; }
      }
    }
    int mid;
    if (best_axis < 0) {
      mid = t.start + t.count / 2;  // all centroids coincide: split by count
    } else {
      double ext = chi[best_axis] - clo[best_axis];
      auto it = std::partition(s.order.begin() + t.start, s.order.begin() + t.start + t.count, [&](int tri) {
        int b = std::min(NB - 1, (int)(NB * (cen[3 * tri + best_axis] - clo[best_axis]) / ext));
        return b <= best_split;
      });
      mid = (int)(it - s.order.begin());
      if (mid == t.start || mid == t.start + t.count) mid = t.start + t.count / 2;
    }
    int l = (int)s.nodes.size();
    s.nodes.push_back(BNode{});
    s.nodes.push_back(BNode{});
    s.nodes[t.node].left = l;
    s.nodes[t.node].right = l + 1;
    stack.push_back({l, t.start, mid - t.start});
    stack.push_back({l + 1, mid, t.start + t.count - mid});
  }
}

// Ray/triangle test in double precision: inside/outside from the watertight sheared edge
// functions of Woop, Benthin and Wald (2013); distance from the plane equation
// t = Ng.(v0 - o) / Ng.d, exactly 0 for an origin on an axis-aligned triangle, so a ray
// leaving such a surface with tnear = 0 does not re-hit it.  Returns true with t in
// (tnear, tfar] and barycentrics (b1, b2) = Embree's (u, v).
inline bool IntersectTri(V3 org, V3 dir, V3 v0, V3 v1, V3 v2, double tnear, double tfar, double* tout,
                         double* uout, double* vout) {
  int kz = 0;
  double ad[3] = {std::abs(dir.x), std::abs(dir.y), std::abs(dir.z)};
  if (ad[1] > ad[kz]) kz = 1;
  if (ad[2] > ad[kz]) kz = 2;
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  if (dir[kz] < 0) std::swap(kx, ky);
  const double Sx = dir[kx] / dir[kz], Sy = dir[ky] / dir[kz];
  const V3 A = v0 - org, B = v1 - org, C = v2 - org;
  const double Ax = A[kx] - Sx * A[kz], Ay = A[ky] - Sy * A[kz];
  const double Bx = B[kx] - Sx * B[kz], By = B[ky] - Sy * B[kz];
  const double Cx = C[kx] - Sx * C[kz], Cy = C[ky] - Sy * C[kz];
  const double U = Cx * By - Cy * Bx;
  const double V = Ax * Cy - Ay * Cx;
  const double W = Bx * Ay - By * Ax;
  if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
  const double det = U + V + W;
  if (det == 0) return false;
  const V3 ng = Cross(v1 - v0, v2 - v0);
  const double den = Dot(ng, dir);
  if (den == 0) return false;
  // Axis-aligned planes: the distance along that axis alone (coplanar faces tie exactly).
  double t;
  if (ng.y == 0 && ng.z == 0) t = A.x / dir.x;
  else if (ng.x == 0 && ng.z == 0) t = A.y / dir.y;
  else if (ng.x == 0 && ng.y == 0) t = A.z / dir.z;
  else t = Dot(ng, A) / den;
  if (!(t > tnear && t <= tfar)) return false;
  *tout = t;
  *uout = V / det;
  *vout = W / det;
  return true;
}

// Ray/sphere roots in double precision: t^2 |d|^2 + 2 t (v.d) + |v|^2 - r^2 = 0 with
// v = org - centre, solved with the cancellation-free pairing q = -(b + sign(b) sqrt(D)),
// t = q / a and c / q (PBRT's Quadratic, util.hxx:131-144).  The reference tests spheres in
// single precision with PBRT error bounds (embreeaccelerator.cxx:307-427); double
// precision keeps planet-sized spheres usable a few metres above the ground.
inline bool SphereRoots(V3 org, V3 dir, V3 c, double r, double* t0, double* t1) {
  const V3 v = org - c;
  const double a = Dot(dir, dir), b = Dot(v, dir), cc = Dot(v, v) - r * r;
  const double D = b * b - a * cc;
  if (D < 0) return false;
  const double q = -(b + std::copysign(std::sqrt(D), b));
  if (q == 0) { *t0 = *t1 = 0; return true; }
  *t0 = q / a;
  *t1 = cc / q;
  if (*t0 > *t1) std::swap(*t0, *t1);
  return true;
}

inline bool IntersectPrim(const Scene& sc, int prim, V3 org, V3 dir, double tnear, double tfar, double* t,
                          double* u, double* v) {
  if (!IsSphere(sc, prim)) return IntersectTri(org, dir, sc.tv0[prim], sc.tv1[prim], sc.tv2[prim], tnear, tfar, t, u, v);
  double t0, t1;
  if (!SphereRoots(org, dir, sc.sph_c[prim - sc.ntri], sc.sph_r[prim - sc.ntri], &t0, &t1)) return false;
  *u = *v = 0;
  if (t0 > tnear && t0 <= tfar) { *t = t0; return true; }
  if (t1 > tnear && t1 <= tfar) { *t = t1; return true; }
  return false;
}

inline bool SlabHit(const BNode& nd, V3 org, V3 inv, double tnear, double tfar, double* tentry) {
  double t0 = tnear, t1 = tfar;
  for (int k = 0; k < 3; ++k) {
    double a = (nd.lo[k] - org[k]) * inv[k];
    double b = (nd.hi[k] - org[k]) * inv[k];
    if (a > b) std::swap(a, b);
    // NaN-safe: 0 * inf
    if (!(a <= b)) { a = -1e300; b = 1e300; }
    t0 = std::max(t0, a);
    t1 = std::min(t1, b * (1 + 4 * Eps));
    if (t0 > t1) return false;
  }
  *tentry = t0;
  return true;
}

// Closest hit in (tnear, tfar].  any_hit: stop at the first hit (occlusion).  Hits at the
// same distance resolve to the lower primitive id, so coplanar overlapping faces give the
// same answer whatever the traversal order (Embree leaves such ties to its traversal).
static int Trace(const Scene& sc, const Scene::TriSet& s, V3 org, V3 dir, double tnear, double tfar, bool any_hit,
                 double* t_out, double* u_out, double* v_out) {
  if (s.nodes.empty() || s.tris.empty()) return -1;
  V3 inv{1.0 / dir.x, 1.0 / dir.y, 1.0 / dir.z};
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  int best = -1;
  double best_t = tfar, bu = 0, bv = 0;
  while (sp > 0) {
    const BNode& nd = s.nodes[stack[--sp]];
    double te;
    if (!SlabHit(nd, org, inv, tnear, best_t, &te)) continue;
    if (nd.count > 0) {
      for (int i = nd.start; i < nd.start + nd.count; ++i) {
        int tri = s.order[i];
        double t, u, v;
        if (IntersectPrim(sc, tri, org, dir, tnear, best_t, &t, &u, &v) && (any_hit || t < best_t || best < 0 || tri < best)) {
          best = tri; best_t = t; bu = u; bv = v;
          if (any_hit) { *t_out = t; return tri; }
        }
      }
    } else {
      if (sp + 2 > 128) return -2;
      stack[sp++] = nd.right;
      stack[sp++] = nd.left;
    }
  }
  if (best >= 0) { *t_out = best_t; *u_out = bu; *v_out = bv; }
  return best;
}

static int TraceBrute(const Scene& sc, const Scene::TriSet& s, V3 org, V3 dir, double tnear, double tfar,
                      double* t_out, double* u_out, double* v_out) {
  int best = -1;
  double best_t = tfar, bu = 0, bv = 0;
  for (int tri : s.tris) {
    double t, u, v;
    if (IntersectPrim(sc, tri, org, dir, tnear, best_t, &t, &u, &v) && (t < best_t || best < 0 || tri < best)) {
      best = tri; best_t = t; bu = u; bv = v;
    }
  }
  if (best >= 0) { *t_out = best_t; *u_out = bu; *v_out = bv; }
  return best;
}

// A medium-boundary (or surface) crossing: BoundaryIntersection (embreeaccelerator.hxx:27-35).
struct Crossing {
  int prim;
  uint32_t material;
  double t;
  F3 n;  // unnormalised winding normal, float like Embree's Ng
};

// All intersections with t in (tnear, tfar], sorted by t, duplicates (same material, same
// t) removed: EmbreeAccelerator::IntersectionsInOrder with its filter callback
// (embreeaccelerator.cxx:134-213).
static void AllHits(const Scene& sc, const Scene::TriSet& s, V3 org, V3 dir, double tnear, double tfar,
                    std::vector<Crossing>& out) {
  out.clear();
  if (s.nodes.empty() || s.tris.empty()) return;
  V3 inv{1.0 / dir.x, 1.0 / dir.y, 1.0 / dir.z};
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const BNode& nd = s.nodes[stack[--sp]];
    double te;
    if (!SlabHit(nd, org, inv, tnear, tfar, &te)) continue;
    if (nd.count > 0) {
      for (int i = nd.start; i < nd.start + nd.count; ++i) {
        const int tri = s.order[i];
        double ts[2];
        int nt = 0;
        if (IsSphere(sc, tri)) {
          // Both roots of a sphere are crossings (the intersect callback reports t0, then t1).
          double t0, t1;
          if (SphereRoots(org, dir, sc.sph_c[tri - sc.ntri], sc.sph_r[tri - sc.ntri], &t0, &t1)) {
            if (t0 > tnear && t0 <= tfar) ts[nt++] = t0;
            if (t1 > tnear && t1 <= tfar && t1 != t0) ts[nt++] = t1;
          }
        } else {
          double t, u, v;
          if (IntersectTri(org, dir, sc.tv0[tri], sc.tv1[tri], sc.tv2[tri], tnear, tfar, &t, &u, &v)) ts[nt++] = t;
        }
        for (int j = 0; j < nt; ++j) {
          Crossing c;
          c.prim = tri;
          c.material = sc.mat_of_tri[tri];
          c.t = ts[j];
          const V3 ng = IsSphere(sc, tri) ? org + dir * ts[j] - sc.sph_c[tri - sc.ntri]
                                          : Cross(sc.tv1[tri] - sc.tv0[tri], sc.tv2[tri] - sc.tv0[tri]);
          c.n = Ff(ng);
          bool dup = false;
          for (const auto& o : out) dup |= (o.material == c.material) & (o.t == c.t);
          if (!dup) out.push_back(c);
        }
      }
    } else {
      if (sp + 2 > 128) return;
      stack[sp++] = nd.right;
      stack[sp++] = nd.left;
    }
  }
  std::sort(out.begin(), out.end(), [](const Crossing& a, const Crossing& b) { return a.t < b.t; });
}

// ---------------------------------------------------------------------------------------
// Geometry queries.
inline V3 VertD(const Scene& s, uint32_t i) { return {s.vert[i].x, s.vert[i].y, s.vert[i].z}; }

// FillPosBoundsTriangle, primitive.cxx:291-299 (barry weights p0, p1, p2 in that order).
inline V3 PosBounds(V3 p0, V3 p1, V3 p2, V3 b) {
  V3 r = Abs(p0 * b.x) + Abs(p1 * b.y) + Abs(p2 * b.z);
  return r * Gamma7();
}

inline V3 SmoothNormal(const Scene& s, int prim, double w0, double w1, double w2, V3 ng) {
  if (!s.has_normals || IsSphere(s, prim)) return ng;
  uint32_t a = s.idx[3 * prim], b = s.idx[3 * prim + 1], c = s.idx[3 * prim + 2];
  V3 na{s.nrm[a].x, s.nrm[a].y, s.nrm[a].z}, nb{s.nrm[b].x, s.nrm[b].y, s.nrm[b].z},
      nc{s.nrm[c].x, s.nrm[c].y, s.nrm[c].z};
  return Normalized(na * w0 + nb * w1 + nc * w2);
}

inline V3 GeometryNormal(const Scene& s, int prim) {
  return Normalized(Cross(s.tv1[prim] - s.tv0[prim], s.tv2[prim] - s.tv0[prim]));
}

// FillPosBoundsSphere, primitive.cxx:302-306: |pos| (as float) x Gamma<float>(5).
inline double Gamma5() { return (5 * (double)EpsF) / (1 - 5 * (double)EpsF); }
inline V3 SphereBounds(V3 pos) {
  const F3 p = Ff(pos);
  return V3{std::abs((double)p.x), std::abs((double)p.y), std::abs((double)p.z)} * Gamma5();
}

// Sphere surface point with outward normal n (Spheres::GetLocalGeometry,
// primitive.cxx:214-223, and FirstIntersectionSphere, embreeaccelerator.cxx:247-260: the
// position is projected onto the sphere along the normal).
inline const Texture* MaterialTexture(const Scene& s, int prim) {
  const int t = s.materials[s.mat_of_tri[prim]].m.diffuse_texture - 1;
  return t >= 0 ? &s.textures[t] : nullptr;
}

inline Surf SphereSurface(const Scene& s, int prim, V3 n) {
  Surf si;
  si.prim = prim;
  si.barry = n;
  si.pos = s.sph_c[prim - s.ntri] + n * s.sph_r[prim - s.ntri];
  si.geometry_normal = n;
  si.smooth_normal = n;
  si.pos_bounds = SphereBounds(si.pos);
  si.tex = MaterialTexture(s, prim);
  if (si.tex) DirectionToUv(n, &si.tex_u, &si.tex_v);
  return si;
}

// EmbreeAccelerator::FirstIntersectionTriangle (embreeaccelerator.cxx:216-244) followed by
// SurfaceInteraction::SetOrientedNormals (scene.cxx:240-245).  Spheres take the hit
// distance t along (org, ray_dir).
inline Surf SurfaceFromHit(const Scene& s, int prim, double u, double v, V3 org, V3 ray_dir, double t) {
  if (IsSphere(s, prim)) {
    Surf si = SphereSurface(s, prim, Normalized(org + ray_dir * t - s.sph_c[prim - s.ntri]));
    const double sign = -Sign(Dot(ray_dir, si.geometry_normal));
    si.normal = sign * si.geometry_normal;
    si.shading_normal = sign * si.smooth_normal;
    return si;
  }
  Surf si;
  si.prim = prim;
  si.barry = {u, v, 1. - u - v};
  const V3 p0 = s.tv0[prim], p1 = s.tv1[prim], p2 = s.tv2[prim];
  si.pos = p0 * (1. - u - v) + p1 * u + p2 * v;
  si.geometry_normal = GeometryNormal(s, prim);
  si.smooth_normal = SmoothNormal(s, prim, 1. - u - v, u, v, si.geometry_normal);
  si.pos_bounds = PosBounds(p0, p1, p2, si.barry);
  si.tex = MaterialTexture(s, prim);
  if (si.tex && !s.uv.empty()) {
    // rtcInterpolate1 of the uv attribute (embreeaccelerator.cxx:226-228), in float.
    const uint32_t a = s.idx[3 * prim], b = s.idx[3 * prim + 1], c = s.idx[3 * prim + 2];
    const float fu = (float)u, fv = (float)v, fw = 1.f - fu - fv;
    si.tex_u = s.uv[2 * a] * fw + s.uv[2 * b] * fu + s.uv[2 * c] * fv;
    si.tex_v = s.uv[2 * a + 1] * fw + s.uv[2 * b + 1] * fu + s.uv[2 * c + 1] * fv;
  }
  const double sign = -Sign(Dot(ray_dir, si.geometry_normal));
  si.normal = sign * si.geometry_normal;
  si.shading_normal = sign * si.smooth_normal;
  return si;
}

// SurfaceInteraction(HitId) + Mesh::GetLocalGeometry (primitive.cxx:91-116).  For a
// sphere `barry` is the offset from the centre (Spheres::SampleUniformPosition).
inline Surf SurfaceFromBarycentric(const Scene& s, int prim, V3 barry) {
  if (IsSphere(s, prim)) {
    Surf si = SphereSurface(s, prim, Normalized(barry));
    si.pos = s.sph_c[prim - s.ntri] + barry;
    si.pos_bounds = SphereBounds(si.pos);
    si.normal = si.geometry_normal;
    si.shading_normal = si.smooth_normal;
    return si;
  }
  Surf si;
  si.prim = prim;
  si.barry = barry;
  const V3 p0 = s.tv0[prim], p1 = s.tv1[prim], p2 = s.tv2[prim];
  si.pos = p0 * barry.x + p1 * barry.y + p2 * barry.z;
  si.geometry_normal = GeometryNormal(s, prim);
  si.smooth_normal = SmoothNormal(s, prim, barry.x, barry.y, barry.z, si.geometry_normal);
  si.pos_bounds = PosBounds(p0, p1, p2, barry);
  si.normal = si.geometry_normal;
  si.shading_normal = si.smooth_normal;
  return si;
}

inline double TriArea(const Scene& s, int prim) {  // Mesh::Area, primitive.cxx:129-137; Spheres::Area :206-211
  if (IsSphere(s, prim)) {
    const double r = s.sph_r[prim - s.ntri];
    return r * r * 4. * Pi;
  }
  return 0.5 * Length(Cross(s.tv1[prim] - s.tv0[prim], s.tv2[prim] - s.tv0[prim]));
}

// ---------------------------------------------------------------------------------------
// Shaders (shader.cxx).
struct ScatterSample {
  V3 dir;
  S3 value;
  double pdf = 0;
  bool delta = false;
};

// DiffuseShader::EvaluateBSDF / SampleBSDF, shader.cxx:280-318.
// SpecularReflectiveShader, shader.cxx:338-366.
// SpecularTransmissiveDielectricShader::SampleBsdfRegular, shader.cxx:401-473.
// MicrofacetShader + MicrofacetShaderWrapper, shader.cxx:74-130, 676-707.
// Shader::MyRoughness (shader.cxx:244-247, 666-670): the microfacet's alpha, 0 otherwise.
inline double MyRoughness(const tt_material& m) {
  return (m.shader == TT_SHADER_MICROFACET || m.shader == TT_SHADER_GLOSSY_DIELECTRIC) ? (double)m.alpha : 0.;
}

// GlossyTransmissiveDielectricShader, shader.cxx:710-787: the wrapper
// GlossyTransmissiveDielectricWrapper (shader.cxx:126-190) over the local frame of the
// shading normal, sampled by TransmissiveMicrofacetDensity
// (normaldistributionfunction.hxx:149-197) with the broadened roughness
// AlphaBroadeningFormula (shader.cxx:59-62).
struct GlossyDielectric {
  Frame frame;
  V3 wi, ng;  // local
  double eta;  // eta_i / eta_t, i = the incident side
  Beckman ndf, broadened;

  GlossyDielectric(const tt_material& m, V3 wi_world, const Surf& si, double min_roughness)
      : frame(OrthogonalSystemZAligned(si.shading_normal)), ndf{0.}, broadened{0.} {
    wi = frame.ToLocal(wi_world);
    ng = frame.ToLocal(si.normal);
    eta = Dot(si.geometry_normal, wi_world) < 0. ? (double)m.ior_ratio : 1. / m.ior_ratio;
    const double alpha = std::max(min_roughness, (double)m.alpha);
    ndf = Beckman{alpha};
    broadened = Beckman{alpha * (1.2 - 0.2 * std::abs(wi.z))};
  }
  double Pdf(V3 wo) const {  // TransmissiveMicrofacetDensity::Pdf
    double pdf_wot = 0.;
    V3 wht;
    if (HalfVectorRefracted(wi, wo, eta, &wht)) {
      const double fr_wht = FresnelReflectivityWalter(std::abs(Dot(wht, wi)), eta);
      const double ndf_transm = broadened.EvalByHalfVector(std::abs(wht.z)) * std::abs(wht.z);
      pdf_wot = HalfVectorPdfToTransmittedPdf(ndf_transm, eta, Dot(wht, wi), Dot(wht, wo)) * (1.0 - fr_wht);
    }
    const V3 whr = HalfVector(wi, wo);
    const double fr_whr = FresnelReflectivityWalter(std::abs(Dot(whr, wi)), eta);
    const double ndf_reflect = broadened.EvalByHalfVector(std::abs(whr.z)) * std::abs(whr.z);
    return HalfVectorPdfToReflectedPdf(ndf_reflect, Dot(whr, wi)) * fr_whr + pdf_wot;
  }
  double Evaluate(V3 wo, double* pdf) const {
    if (pdf) *pdf = Pdf(wo);
    const double ns_dot_out = wo.z, ns_dot_in = wi.z;
    if (Dot(ng, wo) >= 0) {
      const V3 whr = HalfVector(wi, wo);
      const double wh_dot_out = Dot(wo, whr), wh_dot_in = Dot(wi, whr);
      const double fr_whr = FresnelReflectivityWalter(std::abs(wh_dot_in), eta);
      const double D = ndf.EvalByHalfVector(std::abs(whr.z));
      const double G = G2VCavity(wh_dot_in, wh_dot_out, ns_dot_in, ns_dot_out, whr.z);
      return fr_whr * G * D * 0.25 / (std::abs(ns_dot_in * ns_dot_out) + Eps);
    }
    V3 wht;
    if (!HalfVectorRefracted(wi, wo, eta, &wht)) return 0.;
    if (wht.z < 0.) wht = -wht;
    const double wh_dot_out = Dot(wo, wht), wh_dot_in = Dot(wi, wht);
    const double fr_wht = FresnelReflectivityWalter(std::abs(wh_dot_in), eta);
    const double D = ndf.EvalByHalfVector(std::abs(wht.z));
    const double J = HalfVectorPdfToTransmittedPdf(1.0, eta, wh_dot_in, wh_dot_out);
    const double G = G2VCavityTransmissive(wh_dot_in, wh_dot_out, ns_dot_in, ns_dot_out, wht.z);
    return (1.0 - fr_wht) * std::abs(wh_dot_in) * G * D * J / (std::abs(ns_dot_in * ns_dot_out) + Eps);
  }
  V3 Sample(const double r1[2], double r2) const {  // TransmissiveMicrofacetDensity::Sample
    const V3 wh = broadened.SampleHalfVector(r1);
    double fr = FresnelReflectivityWalter(std::abs(Dot(wh, wi)), eta);
    V3 wt;
    if (!Refracted(wi, wh, eta, &wt)) fr = 1.0;
    return r2 < fr ? Reflected(wi, wh) : wt;
  }
};

// SpecularTransmissiveDielectricShader::Sample/EvaluateBsdfMollified (shader.cxx:482-605):
// with a path roughness r > 0 (pt2's path regularisation) the specular lobes become
// uniform cones of cos opening 1 - r around the reflected and refracted directions.
static S3 EvaluateDielectricMollified(const tt_material& m, V3 wi, const Surf& si, V3 wo, double roughness,
                                      double* pdf) {
  const double opening_cos = 1. - roughness;
  const bool entering = Dot(si.geometry_normal, wi) > 0.;
  const double eta = entering ? 1. / m.ior_ratio : (double)m.ior_ratio;
  const double radiance_weight = Sqr(eta);
  const double abs_shn_dot_i = std::abs(Dot(si.shading_normal, wi));
  double fr = 1.;
  V3 wt;
  const bool has_wt = Refracted(wi, si.shading_normal, eta, &wt);
  if (has_wt) fr = FresnelReflectivity(abs_shn_dot_i, std::abs(Dot(wt, si.shading_normal)), eta);
  const double prob_reflection = has_wt ? std::max(0.1, std::min(0.9, fr)) : 1.;
  const double section_pdf = 1. / (2. * Pi * (1. - opening_cos));
  const V3 refl = Reflected(wi, si.shading_normal);
  const bool maybe_reflected = Dot(refl, wo) > opening_cos;
  double total_pdf = maybe_reflected ? section_pdf * prob_reflection : 0.;
  double total_val = maybe_reflected ? prob_reflection * fr : 0.;
  if (has_wt) {
    const bool maybe_refracted = Dot(wt, wo) > opening_cos;
    total_val += maybe_refracted ? (1. - fr) * section_pdf : 0.;
    total_pdf += maybe_refracted ? (1. - prob_reflection) * section_pdf : 0.;
  }
  if (Dot(wo, si.normal) < 0) total_val *= radiance_weight;
  total_val /= std::abs(Dot(wo, si.shading_normal));
  if (pdf) *pdf = total_pdf;
  return S3(total_val);
}

// DiffuseShader's reflectance times MaybeMultiplyTextureLookup (shader.cxx:17-27): the
// texel's RGB as the selected wavelengths' values.
inline S3 DiffuseReflectance(const tt_material& m, const Surf& si, const int32_t idx[3]) {
  S3 kr = Take(m.reflectance, idx);
  if (si.tex) {
    double rgb[3];
    si.tex->Lookup(si.tex_u, si.tex_v, rgb);
    kr = kr * RGBToSpectralSelection(rgb, idx);
  }
  return kr;
}

// SpecularDenseDielectricShader (shader.cxx:977-1081): SchlicksApproximation
// (shader_physics.hxx:95-101) and DiffuseAttenuationFactor with the average albedo of
// AverageOfProjectedSchlicksApproximationOverHemisphere.
inline double Schlick(double k, double cos_n) { return k + (1. - k) * std::pow(1. - cos_n, 5.); }
inline double DenseAttenuation(double k, double r_in, double r_out) {
  const double avg = k + (1. - k) * 2. / 42.;
  return (1. - r_in) * (1. - r_out) / (1. - avg);
}

static S3 EvaluateBSDF(const tt_material& m, V3 wi, const Surf& si, V3 wo, const int32_t idx[3], double* pdf,
                       double min_roughness = 0.) {
  if (m.shader == TT_SHADER_SPECULAR_DIELECTRIC && min_roughness > 0.)
    return EvaluateDielectricMollified(m, wi, si, wo, min_roughness, pdf);
  switch (m.shader) {
    case TT_SHADER_DIFFUSE: {
      S3 ret(0.);
      double n_dot_out = Dot(si.normal, wo);
      double nsh_dot_out = Dot(si.shading_normal, wo);
      if (n_dot_out > 0.) ret = DiffuseReflectance(m, si, idx) * (1. / Pi);
      if (pdf) *pdf = std::max(0., nsh_dot_out) / Pi;
      return ret;
    }
    case TT_SHADER_SPECULAR_REFLECTIVE:
    case TT_SHADER_SPECULAR_DIELECTRIC:
      if (pdf) *pdf = 0.;
      return S3(0.);
    case TT_SHADER_GLOSSY_DIELECTRIC: {
      const GlossyDielectric g(m, wi, si, min_roughness);
      return S3(g.Evaluate(g.frame.ToLocal(wo), pdf));
    }
    case TT_SHADER_SPECULAR_DENSE_DIELECTRIC: {
      if (!(Dot(si.normal, wo) > 0.)) {
        if (pdf) *pdf = 0.;
        return S3(0.);
      }
      const double k = m.specular_reflectivity;
      const double r_in = Schlick(k, std::max(0., Dot(si.shading_normal, wi)));
      const double r_out = Schlick(k, std::max(0., Dot(si.shading_normal, wo)));
      if (pdf) *pdf = std::max(0., Dot(si.shading_normal, wo)) / Pi * (1. - r_in);
      return DiffuseReflectance(m, si, idx) * (DenseAttenuation(k, r_in, r_out) / Pi);
    }
    case TT_SHADER_MICROFACET: {
      const Frame fr = OrthogonalSystemZAligned(si.shading_normal);
      const V3 ng = fr.ToLocal(si.normal);
      const Beckman ndf{std::max((double)m.alpha, min_roughness)};
      const V3 lwi = fr.ToLocal(wi), lwo = fr.ToLocal(wo);
      const V3 wh = Normalized(lwi + lwo);
      const double n_dot_out = Dot(ng, lwo);
      const double ns_dot_out = lwo.z, ns_dot_in = lwi.z, ns_dot_wh = wh.z;
      const double wh_dot_out = Dot(lwo, wh), wh_dot_in = Dot(lwi, wh);
      double D = ndf.EvalByHalfVector(std::abs(ns_dot_wh));
      const double G = G2VCavity(wh_dot_in, wh_dot_out, ns_dot_in, ns_dot_out, ns_dot_wh);
      if (pdf) {
        V3 wh_flip = wh.z < 0 ? -wh : wh;
        double sp = VndfPdf(D, wh_flip, lwi);
        *pdf = HalfVectorPdfToReflectedPdf(sp, Dot(wh_flip, lwi));
      }
      if (n_dot_out <= 0.) return S3(0.);
      const S3 kr = Take(m.reflectance, idx);
      const double f5 = std::pow(1 - std::abs(wh_dot_in), 5.);
      S3 fresnel{kr[0] + (1. - kr[0]) * f5, kr[1] + (1. - kr[1]) * f5, kr[2] + (1. - kr[2]) * f5};
      double mono = G * D * 0.25 / (std::abs(ns_dot_in * ns_dot_out) + Eps);
      return fresnel * mono;
    }
  }
  if (pdf) *pdf = 0;
  return S3(0.);
}

static ScatterSample SampleBSDF(const tt_material& m, V3 wi, const Surf& si, Sampler& smp, const int32_t idx[3],
                                double min_roughness = 0.) {
  ScatterSample out;
  if (m.shader == TT_SHADER_SPECULAR_DIELECTRIC && min_roughness > 0.) {
    // SampleBsdfMollified (shader.cxx:482-549).
    const double opening_cos = 1. - min_roughness;
    const double abs_shn_dot_i = std::abs(Dot(si.shading_normal, wi));
    const bool entering = Dot(si.geometry_normal, wi) > 0.;
    const double eta = entering ? 1. / m.ior_ratio : (double)m.ior_ratio;
    const double radiance_weight = Sqr(eta);
    double fr = 1.;
    V3 wt;
    const bool has_wt = Refracted(wi, si.shading_normal, eta, &wt);
    if (has_wt) fr = FresnelReflectivity(abs_shn_dot_i, std::abs(Dot(wt, si.shading_normal)), eta);
    const double prob_reflection = has_wt ? std::max(0.1, std::min(0.9, fr)) : 1.;
    const bool do_reflect = has_wt ? smp.Uniform01() < prob_reflection : true;
    const double section_pdf = 1. / (2. * Pi * (1. - opening_cos));
    double r[2];
    double value;
    const V3 axis = do_reflect ? Reflected(wi, si.shading_normal) : wt;
    smp.UniformUnitSquare(r);
    out.dir = OrthogonalSystemZAligned(axis).ToWorld(ToUniformSphereSection(opening_cos, r));
    if (do_reflect) {
      out.pdf = prob_reflection * section_pdf;
      value = fr * section_pdf;
    } else {
      out.pdf = (1. - prob_reflection) * section_pdf;
      value = (1. - fr) * section_pdf;
    }
    value /= std::abs(Dot(out.dir, si.shading_normal));
    if (Dot(out.dir, si.normal) < 0) value *= radiance_weight;
    out.value = S3(value);
    return out;
  }
  switch (m.shader) {
    case TT_SHADER_SPECULAR_DENSE_DIELECTRIC: {
      const double k = m.specular_reflectivity;
      const double cos_in = std::max(0., Dot(si.shading_normal, wi));
      const double r_in = Schlick(k, cos_in);
      if (smp.Uniform01() < r_in) {
        const V3 r = Reflected(wi, si.shading_normal);
        out.dir = r;
        out.pdf = r_in;
        out.delta = true;
        out.value = Dot(si.normal, r) >= 0. ? S3(r_in / (cos_in + Eps)) : S3(0.);
        return out;
      }
      const Frame fr = OrthogonalSystemZAligned(si.shading_normal);
      double r[2];
      smp.UniformUnitSquare(r);
      const V3 v = ToCosHemisphere(r);
      out.dir = fr.ToWorld(v);
      out.pdf = v.z / Pi * (1. - r_in);
      const double r_out = Schlick(k, std::max(0., Dot(si.shading_normal, out.dir)));
      out.value = Dot(si.normal, out.dir) > 0
                      ? DiffuseReflectance(m, si, idx) * (DenseAttenuation(k, r_in, r_out) / Pi)
                      : S3(0.);
      return out;
    }
    case TT_SHADER_GLOSSY_DIELECTRIC: {
      const GlossyDielectric g(m, wi, si, min_roughness);
      double r[2];
      smp.UniformUnitSquare(r);
      const V3 wo = g.Sample(r, smp.Uniform01());
      out.value = S3(g.Evaluate(wo, &out.pdf));
      out.dir = g.frame.ToWorld(wo);
      return out;
    }
    case TT_SHADER_DIFFUSE: {
      const Frame fr = OrthogonalSystemZAligned(si.shading_normal);
      double r[2];
      smp.UniformUnitSquare(r);
      V3 v = ToCosHemisphere(r);
      out.pdf = v.z / Pi;
      out.dir = fr.ToWorld(v);
      out.value = Dot(si.normal, out.dir) > 0 ? DiffuseReflectance(m, si, idx) * (1. / Pi) : S3(0.);
      return out;
    }
    case TT_SHADER_SPECULAR_REFLECTIVE: {
      V3 r = Reflected(wi, si.shading_normal);
      double cos_rn = Dot(si.normal, r);
      out.dir = r;
      out.pdf = 1.;
      out.delta = true;
      if (cos_rn < 0.) out.value = S3(0.);
      else out.value = Take(m.reflectance, idx) / Dot(si.shading_normal, r);
      return out;
    }
    case TT_SHADER_SPECULAR_DIELECTRIC: {
      const double abs_shn_dot_i = std::abs(Dot(si.shading_normal, wi));
      const bool entering = Dot(si.geometry_normal, wi) > 0.;
      const double eta = entering ? 1. / m.ior_ratio : (double)m.ior_ratio;
      const double radiance_weight = Sqr(eta);  // RADIANCE transport
      double fr = 1.;
      V3 wt;
      const bool has_wt = Refracted(wi, si.shading_normal, eta, &wt);
      if (has_wt) fr = FresnelReflectivity(abs_shn_dot_i, std::abs(Dot(wt, si.shading_normal)), eta);
      const double prob_reflection = has_wt ? std::max(0.1, std::min(0.9, fr)) : 1.;
      const bool do_reflect = has_wt ? smp.Uniform01() < prob_reflection : true;
      double value;
      out.delta = true;
      if (do_reflect) {
        out.dir = Reflected(wi, si.shading_normal);
        out.pdf = prob_reflection;
        value = fr;
      } else {
        out.dir = wt;
        out.pdf = 1. - prob_reflection;
        value = 1. - fr;
      }
      value /= std::abs(Dot(out.dir, si.shading_normal));
      if (Dot(out.dir, si.normal) < 0) value *= radiance_weight;
      out.value = S3(value);
      return out;
    }
    case TT_SHADER_MICROFACET: {
      const Frame fr = OrthogonalSystemZAligned(si.shading_normal);
      const Beckman ndf{std::max((double)m.alpha, min_roughness)};
      const V3 lwi = fr.ToLocal(wi);
      double r[2];
      smp.UniformUnitSquare(r);
      V3 wh = ndf.SampleHalfVector(r);
      VndfSample(wh, lwi, smp.Uniform01());
      const V3 lwo = Reflected(lwi, wh);
      // MicrofacetShaderWrapper::Evaluate with the sampled half vector.
      const V3 ng = fr.ToLocal(si.normal);
      const double n_dot_out = Dot(ng, lwo);
      const double ns_dot_out = lwo.z, ns_dot_in = lwi.z, ns_dot_wh = wh.z;
      const double wh_dot_out = Dot(lwo, wh), wh_dot_in = Dot(lwi, wh);
      const double D = ndf.EvalByHalfVector(std::abs(ns_dot_wh));
      const double G = G2VCavity(wh_dot_in, wh_dot_out, ns_dot_in, ns_dot_out, ns_dot_wh);
      V3 wh_flip = wh.z < 0 ? -wh : wh;
      double sp = VndfPdf(D, wh_flip, lwi);
      out.pdf = HalfVectorPdfToReflectedPdf(sp, Dot(wh_flip, lwi));
      out.dir = fr.ToWorld(lwo);
      if (n_dot_out <= 0.) { out.value = S3(0.); return out; }
      const S3 kr = Take(m.reflectance, idx);
      const double f5 = std::pow(1 - std::abs(wh_dot_in), 5.);
      S3 fresnel{kr[0] + (1. - kr[0]) * f5, kr[1] + (1. - kr[1]) * f5, kr[2] + (1. - kr[2]) * f5};
      double mono = G * D * 0.25 / (std::abs(ns_dot_in * ns_dot_out) + Eps);
      out.value = fresnel * mono;
      return out;
    }
  }
  out.value = S3(0.);
  return out;
}

// RadianceEstimatorBase::BsdfCorrectionFactor (rendering_randomwalk_impl.hxx:616-622),
// RADIANCE transport: the light-incident direction is the exitant direction.
inline double BsdfCorrectionFactor(const Surf& si, V3 exitant_dir) {
  return std::abs(Dot(si.shading_normal, exitant_dir)) / (std::abs(Dot(si.normal, exitant_dir)) + Eps);
}

// ---------------------------------------------------------------------------------------
// Environmental lights (light.hxx:146-304, light.cxx:10-189).
// KartesianToSpherical (vec3f.hxx:298-321): the THIRD component is "up".
inline void KartesianToSphericalF(const float xyz[3], float* phi, float* theta) {
  const float x = xyz[0], z = xyz[1], y = xyz[2];
  const float ax = std::abs(x), az = std::abs(z);
  const float r = std::sqrt(xyz[0] * xyz[0] + xyz[1] * xyz[1] + xyz[2] * xyz[2]);
  *theta = std::acos(y / r);
  float p;
  if (ax > az) {
    p = std::atan2(z, ax);
    p = (x > 0.f) ? p : (float)Pi - p;
  } else {
    p = std::atan2(x, az);
    p = (z > 0.f) ? (float)(Pi / 2.) - p : (float)(3. / 2. * Pi) + p;
  }
  *phi = p;
}
// UvToPixel, texture.hxx:37-55.
inline void UvToPixel(int w, int h, float u, float v, int* px, int* py) {
  float dummy;
  u = std::modf(u, &dummy);
  v = std::modf(v, &dummy);
  if (u < 0.f) u = 1.f + u;
  if (v < 0.f) v = 1.f + v;
  if (u > 1.f - EpsF) u -= EpsF;
  if (v > 1.f - EpsF) v -= EpsF;
  int x = (int)(u * w);
  int y = (int)(v * h);
  y = h - y - 1;
  *px = x;
  *py = y;
}

inline void EnvMapPixelOf(const EnvLight& L, V3 dir_out, int* px, int* py) {
  // EnvMapLight::MapToImage, light.cxx:117-121 (float frame, transposed).
  float d[3] = {(float)dir_out.x, (float)dir_out.y, (float)dir_out.z};
  float loc[3] = {L.fX[0] * d[0] + L.fX[1] * d[1] + L.fX[2] * d[2],
                  L.fY[0] * d[0] + L.fY[1] * d[1] + L.fY[2] * d[2],
                  L.fZ[0] * d[0] + L.fZ[1] * d[1] + L.fZ[2] * d[2]};
  float phi, theta;
  KartesianToSphericalF(loc, &phi, &theta);
  const float u = phi / (float)(2. * Pi), v = theta / (float)Pi;
  UvToPixel(L.w, L.h, u, v, px, py);
}

inline void EnvMapPixelAngles(const EnvLight& L, int x, int y, float* phi0, float* z0, float* phi1, float* z1) {
  // PixelToUvBounds (texture.hxx:71-86) + UvToSpherical.
  float ul = (float)x / L.w, vl = (float)y / L.h;
  float uu = ul + 1.f / L.w, vu = vl + 1.f / L.h;
  vl = 1.f - vl;
  vu = 1.f - vu;
  float th_l = vl * (float)Pi, th_u = vu * (float)Pi;
  *phi0 = ul * (float)(2. * Pi);
  *phi1 = uu * (float)(2. * Pi);
  *z0 = std::cos(th_l);
  *z1 = std::cos(th_u);
}

inline S3 EnvMapValue(const EnvLight& L, int x, int y, const int32_t idx[3]) {
  const float* p = &L.tex[3 * ((size_t)y * L.w + x)];
  double rgb[3] = {p[0], p[1], p[2]};
  return RGBToSpectralSelection(rgb, idx);
}

static double EnvEvaluatePdfOne(const EnvLight& L, V3 dir_out) {
  switch (L.kind) {
    case TT_ENV_DOME: return Dot(dir_out, L.down_dir) > 0. ? 1. / (2. * Pi) : 0.;
    case TT_ENV_SUN: return Dot(dir_out, L.frame.Z) > L.cos_opening ? L.pdf_val : 0.;
    case TT_ENV_DIRECTIONAL: return 0.;
    case TT_ENV_MAP: {
      int x, y;
      EnvMapPixelOf(L, dir_out, &x, &y);
      const float proby = ProbFromCmf(L.cmf_rows.data(), y);
      const float probx = ProbFromCmf(&L.cmf_cols[(size_t)y * L.w], x);
      float phi0, z0, phi1, z1;
      EnvMapPixelAngles(L, x, y, &phi0, &z0, &phi1, &z1);
      double pdf = (double)proby * probx;
      pdf /= ((double)z1 - z0) * ((double)phi1 - phi0);
      return pdf;
    }
  }
  return 0;
}

static S3 EnvEvaluateOne(const EnvLight& L, V3 dir_out, const int32_t idx[3]) {
  switch (L.kind) {
    case TT_ENV_DOME: return Dot(dir_out, L.down_dir) > 0. ? TakeD(L.spectrum, idx) : S3(0.);
    case TT_ENV_SUN: return Dot(dir_out, L.frame.Z) > L.cos_opening ? TakeD(L.sun_emission, idx) : S3(0.);
    case TT_ENV_DIRECTIONAL: return S3(0.);
    case TT_ENV_MAP: {
      int x, y;
      EnvMapPixelOf(L, dir_out, &x, &y);
      return EnvMapValue(L, x, y, idx);
    }
  }
  return S3(0.);
}

struct DirSample { V3 dir; S3 value; double pdf; bool delta; };

static DirSample EnvTakeDirectionSampleOne(const EnvLight& L, Sampler& smp, const int32_t idx[3]) {
  DirSample s{};
  double r[2];
  switch (L.kind) {
    case TT_ENV_DOME:
      smp.UniformUnitSquare(r);
      s.dir = L.frame.ToWorld(ToUniformHemisphere(r));
      s.value = TakeD(L.spectrum, idx);
      s.pdf = 1. / (2. * Pi);
      return s;
    case TT_ENV_SUN:
      smp.UniformUnitSquare(r);
      s.dir = L.frame.ToWorld(ToUniformSphereSection(L.cos_opening, r));
      s.value = TakeD(L.sun_emission, idx);
      s.pdf = L.pdf_val;
      return s;
    case TT_ENV_DIRECTIONAL:
      s.dir = L.dir;
      s.value = TakeD(L.spectrum, idx);
      s.pdf = 1.;
      s.delta = true;
      return s;
    case TT_ENV_MAP: {
      smp.UniformUnitSquare(r);
      const int y = TowerSamplingBisection(L.cmf_rows.data(), L.h, (float)r[1]);
      const float proby = ProbFromCmf(L.cmf_rows.data(), y);
      const float* row = &L.cmf_cols[(size_t)y * L.w];
      const int x = TowerSamplingBisection(row, L.w, (float)r[0]);
      const float probx = ProbFromCmf(row, x);
      float phi0, z0, phi1, z1;
      EnvMapPixelAngles(L, x, y, &phi0, &z0, &phi1, &z1);
      double r2[2];
      smp.UniformUnitSquare(r2);
      V3 loc = ToUniformSphereSection(r2, phi0, z0, phi1, z1);
      float lf[3] = {(float)loc.x, (float)loc.y, (float)loc.z};
      float d[3];
      for (int k = 0; k < 3; ++k) d[k] = L.fX[k] * lf[0] + L.fY[k] * lf[1] + L.fZ[k] * lf[2];
      s.dir = {d[0], d[1], d[2]};
      double pdf = (double)proby * probx;
      pdf /= ((double)z1 - z0) * ((double)phi1 - phi0);
      s.pdf = pdf;
      s.value = EnvMapValue(L, x, y, idx);
      return s;
    }
  }
  return s;
}

// TotalEnvironmentalRadianceField (light.cxx:28-85).
static S3 EnvEvaluateTotal(const Scene& sc, V3 dir_out, const int32_t idx[3]) {
  S3 acc(0.);
  for (const auto& L : sc.env) acc = acc + EnvEvaluateOne(L, dir_out, idx);
  return acc;
}
static double EnvEvaluatePdfTotal(const Scene& sc, V3 dir_out) {
  const double sel = sc.env.size() > 0 ? 1. / sc.env.size() : 1.;
  double sum = 0;
  for (const auto& L : sc.env) sum += EnvEvaluatePdfOne(L, dir_out);
  return sum * sel;
}
static DirSample EnvTakeDirectionSampleTotal(const Scene& sc, Sampler& smp, const int32_t idx[3]) {
  const int n = (int)sc.env.size();
  int i = smp.UniformInt(0, n - 1);
  DirSample s = EnvTakeDirectionSampleOne(sc.env[i], smp, idx);
  s.pdf *= 1. / n;
  return s;
}

// ---------------------------------------------------------------------------------------
// Path nodes (rendering_randomwalk_impl.hxx:32-188).
enum NodeType { SURFACE_SCATTER, VOLUME_SCATTER, SURFACE_EMITTER, VOLUME_EMITTER, ENV, POINT_LIGHT, CAMERA, ZERO };

struct Node {
  NodeType type = ZERO;
  V3 incident_dir;
  Surf surf;
  V3 coords;       // ENV: direction; POINT/CAMERA/VOLUME: position; surfaces use surf.pos
  S3 radiance;     // ENV radiance
  int unit = -1;   // CAMERA unit index
  int point = -1;  // point light index
  int medium = -1; // VOLUME_SCATTER: medium index
  S3 sigma_s;      // VOLUME_SCATTER: scattering coefficient at the interaction
  bool IsSurface() const { return type == SURFACE_EMITTER || type == SURFACE_SCATTER; }
  bool IsVolume() const { return type == VOLUME_SCATTER || type == VOLUME_EMITTER; }
  bool IsScatter() const { return type == SURFACE_SCATTER || type == VOLUME_SCATTER; }
  V3 Coordinates() const { return IsSurface() ? surf.pos : coords; }
};

// ---------------------------------------------------------------------------------------
// Phase functions (phasefunctions.cxx:23-138).  Directions sampled about the incident
// travel direction with mu_to_direction's (sin, cos, mu) layout.
inline V3 MuToDirection(double mu, double r2) {
  const double sn = std::sin(Pi * 2. * r2), cs = std::cos(Pi * 2. * r2);
  const double rho = std::sqrt(1. - mu * mu);
  return {sn * rho, cs * rho, mu};
}
inline double RayleighValue(double mu) { return (3. / (16. * Pi)) * (1. + mu * mu); }
inline double RayleighSampleMu(double r) {
  double a = std::pow(-2. + 4. * r + std::sqrt(5. - 16. * r + 16. * r * r), 1. / 3.);
  return a - 1. / a;
}
inline double HgValue(double mu, double g) {
  const double g2 = g * g;
  const double term = 1.0 + g2 - 2.0 * g * mu;
  return 1.0 / (4. * Pi) * (1.0 - g2) / (std::sqrt(term) * term);
}
inline double HgSampleMu(double r, double g) {
  const double s = 2.0 * r - 1.0, g2 = g * g;
  if (std::abs(g) > 1.0e-3) {
    const double t1 = (1.0 - g2) / (1.0 + g * s);
    return (1.0 + g2 - t1 * t1) / (2.0 * g);
  }
  const double s2 = s * s;
  return s + 1.5 * g * (1.0 - s2) - 2.0 * g2 * s * (1.0 - s2);
}

static double PhaseEvaluate(const MediumDesc& m, V3 reverse_incident, V3 out) {
  switch (m.phase) {
    case TT_PHASE_RAYLEIGH: return RayleighValue(Dot(-reverse_incident, out));
    case TT_PHASE_HENYEY_GREENSTEIN: return HgValue(Dot(-reverse_incident, out), m.g);
    default: return 1. / (4. * Pi);
  }
}

static ScatterSample PhaseSample(const MediumDesc& m, V3 reverse_incident, Sampler& smp) {
  ScatterSample out;
  double r[2];
  smp.UniformUnitSquare(r);
  if (m.phase == TT_PHASE_UNIFORM) {
    out.dir = ToUniformSphere(r);
    out.pdf = 1. / (4. * Pi);
  } else {
    const Frame f = OrthogonalSystemZAligned(-reverse_incident);
    const double mu = m.phase == TT_PHASE_RAYLEIGH ? RayleighSampleMu(r[0]) : HgSampleMu(r[0], m.g);
    out.dir = f.ToWorld(MuToDirection(mu, r[1]));
    out.pdf = m.phase == TT_PHASE_RAYLEIGH ? RayleighValue(mu) : HgValue(mu, m.g);
  }
  out.value = S3(out.pdf);
  return out;
}

// SimpleCombined (phasefunctions.cxx:206-273) of the atmosphere's constituents at `pos`:
// Rayleigh for molecules, Henyey-Greenstein(g) for aerosols, mixed in proportion to their
// sigma_s (AtmosphereTemplate::SamplePhaseFunction / EvaluatePhaseFunction,
// atmosphere.cxx:101-123).
struct CombinedPhase {
  MediumDesc pf[2];
  double sel[2];
  S3 w[2];
};
static void MakeCombinedPhase(const MediumDesc& m, V3 pos, const int32_t idx[3], CombinedPhase* c);
static void AtmSigmaS(const MediumDesc& m, double alt, const int32_t idx[3], S3 out[2]);
inline double Altitude(const MediumDesc& m, V3 p);
static void MakeCombinedPhase(const MediumDesc& m, V3 pos, const int32_t idx[3], CombinedPhase* c) {
  c->pf[0].phase = TT_PHASE_RAYLEIGH;
  c->pf[1].phase = TT_PHASE_HENYEY_GREENSTEIN;
  c->pf[1].g = m.g;
  AtmSigmaS(m, Altitude(m, pos), idx, c->w);
  const double s0 = c->w[0].Sum(), s1 = c->w[1].Sum();
  if (s0 + s1 > 0.) {
    c->sel[0] = s0 / (s0 + s1);
    c->sel[1] = s1 / (s0 + s1);
    const S3 tot = c->w[0] + c->w[1];
    for (int i = 0; i < 2; ++i)
      for (int k = 0; k < 3; ++k) c->w[i][k] = c->w[i][k] * (1. / tot[k]);
  } else {
    c->sel[0] = c->sel[1] = 0.5;
  }
}

// Phase function of medium m at a volume vertex at pos (value per wavelength, pdf).
static S3 MediumPhaseEvaluate(const MediumDesc& m, V3 pos, V3 wi, V3 out, const int32_t idx[3], double* pdf) {
  if (m.kind != TT_MEDIUM_ATMOSPHERE) {
    const double v = PhaseEvaluate(m, wi, out);
    if (pdf) *pdf = v;
    return S3(v);
  }
  CombinedPhase c;
  MakeCombinedPhase(m, pos, idx, &c);
  const double p0 = PhaseEvaluate(c.pf[0], wi, out), p1 = PhaseEvaluate(c.pf[1], wi, out);
  if (pdf) *pdf = c.sel[0] * p0 + c.sel[1] * p1;
  return c.w[0] * p0 + c.w[1] * p1;
}
static ScatterSample MediumPhaseSample(const MediumDesc& m, V3 pos, V3 wi, Sampler& smp, const int32_t idx[3]) {
  if (m.kind != TT_MEDIUM_ATMOSPHERE) return PhaseSample(m, wi, smp);
  CombinedPhase c;
  MakeCombinedPhase(m, pos, idx, &c);
  const double r = smp.Uniform01();
  const int k = r >= c.sel[1] ? 0 : 1;  // TowerSampling over two bins
  ScatterSample s = PhaseSample(c.pf[k], wi, smp);
  double pdfs[2];
  pdfs[k] = s.pdf;
  pdfs[1 - k] = PhaseEvaluate(c.pf[1 - k], wi, s.dir);
  s.value = c.w[k] * s.pdf + c.w[1 - k] * pdfs[1 - k];
  s.pdf = c.sel[0] * pdfs[0] + c.sel[1] * pdfs[1];
  return s;
}

// ---------------------------------------------------------------------------------------
// MediumTracker (rendering_util.hxx:18-126, rendering_util.cxx:13-38).  Medium -1 is the
// empty-space vacuum with priority -1; slots hold up to 4 overlapping media.
struct MediumTracker {
  int current = -1;
  int media[4] = {-2, -2, -2, -2};  // -2 = empty slot
};

inline int MediumPriority(const Scene& sc, int m) { return m < 0 ? -1 : sc.media[m].priority; }

static void GoingThroughSurface(const Scene& sc, MediumTracker& mt, V3 dir, F3 n, uint32_t material) {
  const tt_material& mat = sc.materials[material].m;
  int to_enter = mat.medium_inside - 1, to_exit = mat.medium_outside - 1;
  if (to_enter < 0 && to_exit < 0) return;
  const float d = (float)dir.x * n.x + (float)dir.y * n.y + (float)dir.z * n.z;
  if (d > 0.f) std::swap(to_enter, to_exit);
  if (to_exit >= 0) {
    bool found = false;
    for (int i = 0; i < 4 && !found; ++i) {
      found = mt.media[i] == to_exit;
      if (found) mt.media[i] = -2;
    }
    if (to_exit == mt.current) {
      int best = -1;
      for (int i = 0; i < 4; ++i)
        if (mt.media[i] != -2 && MediumPriority(sc, best) < MediumPriority(sc, mt.media[i])) best = mt.media[i];
      mt.current = best;
    }
  }
  if (to_enter >= 0) {
    bool inserted = false;
    for (int i = 0; i < 4 && !inserted; ++i) {
      inserted = mt.media[i] == -2;
      if (inserted) mt.media[i] = to_enter;
    }
    if (inserted && MediumPriority(sc, to_enter) > MediumPriority(sc, mt.current)) mt.current = to_enter;
  }
}

// MediumTracker::initializePosition: count the boundaries between a point outside the
// bounding box (+x side) and pos.
static void InitializeMediumTracker(const Scene& sc, MediumTracker& mt, V3 pos) {
  mt = MediumTracker{};
  const bool inside = pos.x >= sc.bb_lo[0] && pos.x <= sc.bb_hi[0] && pos.y >= sc.bb_lo[1] && pos.y <= sc.bb_hi[1] &&
                      pos.z >= sc.bb_lo[2] && pos.z <= sc.bb_hi[2];
  if (!inside) return;
  const double go = 2. * std::max(sc.bb_hi[0] - sc.bb_lo[0], std::max(sc.bb_hi[1] - sc.bb_lo[1], sc.bb_hi[2] - sc.bb_lo[2]));
  V3 org = pos;
  org.x += go;
  const V3 dir{-1., 0., 0.};
  std::vector<Crossing> hits;
  AllHits(sc, sc.vol, org, dir, 0., go, hits);
  for (const auto& h : hits) GoingThroughSurface(sc, mt, dir, h.n, h.material);
  AllHits(sc, sc.surf, org, dir, 0., go, hits);
  for (const auto& h : hits) GoingThroughSurface(sc, mt, dir, h.n, h.material);
}

// VolumePdfCoefficients and Accumulate (shader.hxx:133-157).
struct VolCoeffs {
  double fwd = 1., bwd = 1., tr = 1.;
};
inline void Accumulate(VolCoeffs& acc, const VolCoeffs& seg, bool is_first, bool is_last) {
  acc.fwd *= is_last ? seg.fwd : seg.tr;
  acc.bwd *= is_first ? seg.bwd : seg.tr;
  acc.tr *= seg.tr;
}

inline S3 TakeD3(const double* a, const int32_t idx[3]) { return {a[idx[0]], a[idx[1]], a[idx[2]]}; }
inline S3 ExpNeg(S3 s, double x) { return {std::exp(-s[0] * x), std::exp(-s[1] * x), std::exp(-s[2] * x)}; }
inline double Mean(S3 s) { return (s[0] + s[1] + s[2]) / 3.; }

// ---------------------------------------------------------------------------------------
// Atmosphere::Tabulated (atmosphere.cxx:18-126, 234-348; atmosphere.hxx:95-123), km units.
inline double Altitude(const MediumDesc& m, V3 p) { return Length(p - m.center) - m.radius; }
inline V3 LowestPoint(const MediumDesc& m, V3 org, V3 dir, double length) {
  double t = -Dot(org - m.center, dir);
  if (t > length) t = length;
  else if (t < 0.) t = 0.;
  return org + dir * t;
}
inline double TabLerp(const std::vector<double>& tab, int row, double f, int bin) {
  return (1. - f) * tab[(size_t)row * NBINS + bin] + f * tab[(size_t)(row + 1) * NBINS + bin];
}
// ComputeCollisionCoefficients followed by EvaluateCoeffs' sigma_t = sigma_a + sigma_s.
// The row index truncates toward zero, so altitudes less than one row below h0 are
// extrapolated from rows 0 and 1, as the reference's (int) cast does.
static void AtmCoeffs(const MediumDesc& m, double alt, const int32_t idx[3], S3* sigma_s, S3* sigma_t) {
  const double ri = (alt - m.h0) * m.inv_dh;
  if (ri >= (double)(m.n - 1)) { *sigma_s = S3(0.); *sigma_t = S3(0.); return; }
  const int i = (int)ri;
  for (int k = 0; k < 3; ++k) {
    double ss, st;
    if (i >= 0) {
      const double f = ri - i;
      ss = TabLerp(m.sig_aer, i, f, idx[k]) + TabLerp(m.sig_mol, i, f, idx[k]);
      st = TabLerp(m.sig_t, i, f, idx[k]);
    } else {
      ss = m.sig_aer[idx[k]] + m.sig_mol[idx[k]];
      st = m.sig_t[idx[k]];
    }
    const double sa = st - ss;
    (*sigma_s)[k] = ss;
    (*sigma_t)[k] = sa + ss;
  }
}
// ComputeSigmaS: per constituent (0 molecules, 1 aerosols).
static void AtmSigmaS(const MediumDesc& m, double alt, const int32_t idx[3], S3 out[2]) {
  const double ri = (alt - m.h0) * m.inv_dh;
  const int i = (int)ri;
  const std::vector<double>* tabs[2] = {&m.sig_mol, &m.sig_aer};
  for (int c = 0; c < 2; ++c)
    for (int k = 0; k < 3; ++k) {
      if (i >= 0 && i < m.n - 1) out[c][k] = TabLerp(*tabs[c], i, ri - i, idx[k]);
      else if (i < 0) out[c][k] = (*tabs[c])[idx[k]];
      else out[c][k] = 0.;
    }
}
// ComputeSigmaTMajorante: the per-row maximum over all bins, made non-increasing upwards.
static double AtmMajorant(const MediumDesc& m, double alt) {
  const double ri = (alt - m.h0) * m.inv_dh;
  const int i = (int)ri;
  if (i >= 0 && i < m.n - 1) {
    const double f = ri - i;
    return (1. - f) * m.maj[i] + f * m.maj[i + 1];
  }
  return i < 0 ? m.maj[0] : 0.;
}
// AtmosphereTemplate::ComputeMajorante: at the lowest point of the segment, clamped to the
// table's lower altitude.
inline double AtmSegmentMajorant(const MediumDesc& m, V3 org, V3 dir, double length) {
  return AtmMajorant(m, std::max(m.h0, Altitude(m, LowestPoint(m, org, dir, length))));
}

// ComputeProbabilitiesHistoryScheme (media_integrator.cxx:11-40) for two collision types.
inline void HistoryProbabilities(S3 w, S3 a, S3 b, double* pa, double* pb) {
  *pa = Mean(a * w);
  *pb = Mean(b * w);
  const double norm = *pa + *pb;
  if (norm > 0.) { *pa /= norm; *pb /= norm; } else { *pa = *pb = 0.5; }
}

// VacuumMedium / HomogeneousMedium / AtmosphereTemplate::ComputeVolumePdfCoefficients
// (shader.cxx:1204-1211, 1297-1309; atmosphere.cxx:66-80).
static VolCoeffs VolumeCoeffs(const Scene& sc, int medium, V3 org, V3 dir, double length, const int32_t idx[3]) {
  if (medium < 0) return {0., 0., 1.};
  const MediumDesc& m = sc.media[medium];
  if (m.kind == TT_MEDIUM_ATMOSPHERE) {
    const double maj = AtmMajorant(m, Altitude(m, LowestPoint(m, org, dir, length)));
    const double tr = std::exp(-maj * length);
    return {maj * tr, maj * tr, tr};
  }
  const S3 se = TakeD3(m.sigma_ext, idx);
  const double tr = Mean(ExpNeg(se, length)), e = Mean(se);
  return {e * tr, e * tr, tr};
}

struct InteractionSample {
  double t;
  S3 weight;
  S3 sigma_s;
};

// SpectralTracking (media_integrator.cxx:90-147), the atmosphere's SampleInteractionPoint:
// null-collision tracking against the segment majorant with spectral MIS.  The weight
// starts at initial_weights, as in the reference.
static InteractionSample AtmTracking(const MediumDesc& m, V3 org, V3 dir, double length, S3 initial_weights,
                                     Sampler& smp, const int32_t idx[3]) {
  InteractionSample smpl{0., initial_weights, S3(0.)};
  const double maj = AtmSegmentMajorant(m, org, dir, length);
  if (maj <= 0.) { smpl.t = LargeNumber; return smpl; }
  const double mfp = 1. / maj;
  int iteration = 0;
  while (++iteration < 1000) {
    smpl.t -= std::log(smp.Uniform01()) * mfp;
    if (smpl.t > length) return smpl;
    S3 ss, st;
    AtmCoeffs(m, Altitude(m, org + dir * smpl.t), idx, &ss, &st);
    S3 sn;
    for (int k = 0; k < 3; ++k) sn[k] = std::max(0., maj - st[k]);
    double pt, pn;
    HistoryProbabilities(smpl.weight, ss, sn, &pt, &pn);
    if (smp.Uniform01() < pt) {
      smpl.weight = smpl.weight * (mfp / pt);
      smpl.sigma_s = ss;
      return smpl;
    }
    smpl.weight = smpl.weight * sn * (mfp / pn);
  }
  return smpl;
}

// EstimateTransmission (media_integrator.cxx:150-187): ratio tracking with Russian
// roulette after five steps (RussianRouletteSurvival, media_integrator.hxx:15-33).
static S3 AtmTransmission(const MediumDesc& m, V3 org, V3 dir, double length, Sampler& smp, const int32_t idx[3]) {
  S3 est(1.);
  const double maj = AtmSegmentMajorant(m, org, dir, length);
  if (maj <= 0.) return est;
  const double inv = 1. / maj;
  double t = 0.;
  int iteration = 0;
  for (;;) {
    t -= std::log(smp.Uniform01()) * inv;
    if (t > length) break;
    S3 ss, st;
    AtmCoeffs(m, Altitude(m, org + dir * t), idx, &ss, &st);
    S3 sn;
    for (int k = 0; k < 3; ++k) sn[k] = maj - st[k];
    est = est * sn * inv;
    const double w = est.Max();
    const int it = iteration++;
    if (w <= 0.) break;
    if (it < 5) continue;
    const double p = std::min(w, 1.);
    if (smp.Uniform01() < p) est = est * (1. / p);
    else { est = est * 0.; break; }
  }
  return est;
}

// Medium::EvaluateTransmission of one segment: closed form for homogeneous media, ratio
// tracking for the atmosphere.
static S3 SegmentTransmission(const Scene& sc, int medium, V3 org, V3 dir, double length, Sampler& smp,
                              const int32_t idx[3]) {
  if (medium < 0) return S3(1.);
  const MediumDesc& m = sc.media[medium];
  if (m.kind == TT_MEDIUM_ATMOSPHERE) return AtmTransmission(m, org, dir, length, smp, idx);
  return ExpNeg(TakeD3(m.sigma_ext, idx), length);
}

// Medium::SampleInteractionPoint of one segment: HomogeneousMedium (shader.cxx:1259-1270)
// with HomogeneousSpectralTracking (media_integrator.cxx:43-87, Kutz et al. 2017), or the
// atmosphere's SpectralTracking.
static InteractionSample SampleInteraction(const Scene& sc, int medium, V3 org, V3 dir, double length,
                                           S3 initial_weights, Sampler& smp, const int32_t idx[3]) {
  if (medium < 0) return {LargeNumber, S3(1.), S3(0.)};
  const MediumDesc& m = sc.media[medium];
  if (m.kind == TT_MEDIUM_ATMOSPHERE) return AtmTracking(m, org, dir, length, initial_weights, smp, idx);
  const S3 sigma_ext = TakeD3(m.sigma_ext, idx), sigma_s = TakeD3(m.sigma_s, idx);
  if (!m.is_scattering) return {LargeNumber, ExpNeg(sigma_ext, length), S3(0.)};
  InteractionSample smpl{0., S3(1.), S3(0.)};
  const double majorant = sigma_ext.Max();
  const S3 sigma_n{majorant - sigma_ext[0], majorant - sigma_ext[1], majorant - sigma_ext[2]};
  const double inv_majorant = 1. / majorant;
  int iteration = 0;
  while (++iteration < 100) {
    smpl.t -= std::log(smp.Uniform01()) * inv_majorant;
    if (smpl.t > length) return smpl;
    // ComputeProbabilitiesHistoryScheme (media_integrator.cxx:11-40).
    const S3 w = smpl.weight * initial_weights;
    double pt = Mean(sigma_s * w), pn = Mean(sigma_n * w);
    const double norm = pt + pn;
    if (norm > 0.) { pt /= norm; pn /= norm; } else { pt = pn = 0.5; }
    if (smp.Uniform01() < pt) {
      smpl.weight = smpl.weight * (inv_majorant / pt);
      smpl.sigma_s = sigma_s;
      return smpl;
    }
    smpl.weight = smpl.weight * sigma_n * (inv_majorant / pn);
  }
  return smpl;
}

struct PathCtx {
  int32_t idx[3];
};

// Camera (camera.hxx).
inline double PixelPdfWrtSolidAngle(const Camera& c, double x, double y) {
  double area = c.xperpixel * c.yperpixel;
  V3 v{x, y, 1.};
  double l = Length(v);
  v = v * (1. / l);
  // PdfConversion::AreaToSolidAngle(l, v, (0,0,1)) = l^2 / (|v.z| + Eps)
  return 1. / area * (Sqr(l) / std::abs(v.z + Eps));
}

struct CameraResponse { int unit; double pdf; };

static CameraResponse CameraEvaluate(const Camera& c, V3 dir_out) {
  CameraResponse r{-1, 0.};
  if (c.kind != TT_CAMERA_PINHOLE) return r;  // FisheyeHemisphereCamera::Evaluate returns nothing
  double z = Dot(dir_out, c.dir), x = Dot(dir_out, c.right), y = Dot(dir_out, c.up);
  if (z <= 0.) return r;
  x /= z;
  y /= z;
  int px = (int)((x - c.xmin) / c.xperpixel);
  int py = (int)((y - c.ymin) / c.yperpixel);
  if (px < 0 || px >= c.xres || py < 0 || py >= c.yres) return r;
  r.pdf = PixelPdfWrtSolidAngle(c, x, y);
  r.unit = py * c.xres + px;
  return r;
}

static DirSample CameraTakeDirectionSample(const Camera& c, int unit, Sampler& smp) {
  DirSample s{};
  int py = unit / c.xres, px = unit - py * c.xres;
  double r[2];
  smp.UniformUnitSquare(r);
  if (c.kind == TT_CAMERA_PINHOLE) {
    V3 v{c.xmin + (r[0] + px) * c.xperpixel, c.ymin + (r[1] + py) * c.yperpixel, 1.0};
    v = Normalized(v);
    s.dir = c.right * v.x + c.up * v.y + c.dir * v.z;
    double pdf = PixelPdfWrtSolidAngle(c, v.x, v.y);  // sic: normalized components
    s.value = S3(pdf);
    s.pdf = pdf;
  } else {
    double u = (r[0] + px) * c.per_pixel_delta - 1.0;
    double v = (r[1] + py) * c.per_pixel_delta - 1.0;
    double rho = u * u + v * v;
    V3 w{2. * u, 2. * v, rho - 1.};
    w = w * (1. / (1. + rho));
    w.z = -w.z;
    if (rho <= 1.) {
      s.dir = c.right * w.x + c.up * w.y + c.dir * w.z;
      s.value = S3(1.);
    } else {
      s.dir = c.dir;
      s.value = S3(0.);
    }
    s.pdf = 1.;
    s.delta = true;
  }
  return s;
}

// ---------------------------------------------------------------------------------------
// The estimator.
struct Worker {
  const Scene& sc;
  Sampler smp;
  PathCtx ctx;
  int sensor_connection_unit = -1;
  bool do_sample_brdf = true, do_sample_lights = true;
  int max_path_node_count;
  Worker(const Scene& s) : sc(s) {
    max_path_node_count = s.params.max_ray_depth + 1;
    if (s.params.pt_sample_mode == TT_SAMPLE_BSDF) do_sample_lights = false;
    if (s.params.pt_sample_mode == TT_SAMPLE_LIGHTS) do_sample_brdf = false;
    // A scene without lights has nothing to connect to (and no light to pick).
    if (s.env.empty() && s.area_lights.empty() && s.points.empty()) do_sample_lights = false;
  }

  double DFactorOf(const Node& n, V3 dir) const {
    if (n.IsSurface()) return std::abs(Dot(n.surf.geometry_normal, dir));
    return 1.;
  }
  void AddAntiSelfIntersectionOffsetAt(V3& p, const Node& n, V3 dir) const {
    if (n.IsSurface()) p = p + AntiSelfIntersectionOffset(n.surf, dir);
  }

  // EmitterSampleVisitor + TrivialLightPicker::PickLight (rendering_randomwalk_impl.hxx:192-250,
  // lightpicker_trivial.hxx:66-114).
  Node SampleEmissiveEnd(double* pdf, bool* delta) {
    Node node;
    int which = TowerSampling4(sc.type_probs, smp.Uniform01());
    *delta = false;
    switch (which) {
      case 0: {
        double prob = sc.type_probs[0];
        DirSample s = EnvTakeDirectionSampleTotal(sc, smp, ctx.idx);
        node.type = ENV;
        node.coords = s.dir;
        node.radiance = s.value;
        *pdf = prob * s.pdf;
        *delta = s.delta;
        break;
      }
      case 2: {
        int n = (int)sc.points.size();
        int i = smp.UniformInt(0, n - 1);
        double prob = sc.type_probs[2] / n;
        node.type = POINT_LIGHT;
        node.point = i;
        node.coords = {sc.points[i].pos[0], sc.points[i].pos[1], sc.points[i].pos[2]};
        *pdf = prob;
        *delta = true;
        break;
      }
      case 1: {
        int n = (int)sc.area_lights.size();
        int i = smp.UniformInt(0, n - 1);
        int prim = sc.area_lights[i];
        double prob = sc.type_probs[1] / n;
        double r[2];
        smp.UniformUnitSquare(r);
        V3 b = IsSphere(sc, prim) ? ToUniformSphere(r) * sc.sph_r[prim - sc.ntri] : ToTriangleBarycentricCoords(r);
        node.type = SURFACE_EMITTER;
        node.surf = SurfaceFromBarycentric(sc, prim, b);
        *pdf = prob * (1. / TriArea(sc, prim));
        break;
      }
      default:
        *pdf = 0;
        break;
    }
    return node;
  }

  // Emitter Evaluate for the non-scatter node kinds (rendering_randomwalk_impl.hxx:420-461).
  S3 EvaluateEmitter(const Node& n, V3 out_dir, double* pdf) {
    if (n.type == CAMERA) {
      CameraResponse r = CameraEvaluate(sc.cam, out_dir);
      sensor_connection_unit = r.unit;
      if (pdf) *pdf = r.pdf;
      return r.unit >= 0 ? S3(r.pdf) : S3(0.);
    } else if (n.type == ENV) {
      if (pdf) *pdf = 1. / (Pi * 0.25 * Sqr(sc.diag));
      return n.radiance;
    } else if (n.type == SURFACE_EMITTER) {
      const tt_material& m = sc.materials[sc.mat_of_tri[n.surf.prim]].m;
      // UniformAreaLightDirectionalPart::Evaluate, light.hxx:96-104 (uses the raw winding normal).
      double vis = Dot(n.surf.geometry_normal, out_dir) > 0. ? 1. : 0.;
      if (pdf) *pdf = vis / (2. * Pi);
      return Take(m.emission, ctx.idx) * (vis / (2. * Pi));
    } else if (n.type == POINT_LIGHT) {
      if (pdf) *pdf = 1. / (4. * Pi);
      return Take(sc.points[n.point].spectrum, ctx.idx) * (1. / (4. * Pi));
    }
    return S3(0.);
  }

  S3 EvaluateScatterer(const Node& n, V3 out_dir, double* pdf) {
    const V3 wi = -n.incident_dir;
    if (n.IsVolume()) {  // EvaluateScatterCoordinateOfScatterer, volume branch
      return MediumPhaseEvaluate(sc.media[n.medium], n.coords, wi, out_dir, ctx.idx, pdf) * n.sigma_s;
    }
    const tt_material& m = sc.materials[sc.mat_of_tri[n.surf.prim]].m;
    S3 fs = EvaluateBSDF(m, wi, n.surf, out_dir, ctx.idx, pdf);
    return fs * BsdfCorrectionFactor(n.surf, out_dir);
  }

  S3 Evaluate(const Node& n, V3 out_dir, double* pdf) {
    return n.IsScatter() ? EvaluateScatterer(n, out_dir, pdf) : EvaluateEmitter(n, out_dir, pdf);
  }

  // CalculateSegmentToTarget, rendering_randomwalk_impl.hxx:663-725.
  void SegmentToTarget(const Node& src, const Node& tgt, V3* org, V3* dir, double* len) {
    V3 cs = src.Coordinates(), ct = tgt.Coordinates();
    auto figure = [&](V3* d, double* l) {
      if (tgt.type != ENV) {
        V3 dd = ct - cs;
        double ll = Length(dd);
        *d = dd / ll;
        *l = ll;
      } else {
        *d = -ct;
        *l = sc.long_distance;
      }
    };
    V3 d;
    double l;
    figure(&d, &l);
    AddAntiSelfIntersectionOffsetAt(cs, src, d);
    AddAntiSelfIntersectionOffsetAt(ct, tgt, -d);
    figure(&d, &l);
    *org = cs;
    *dir = d;
    *len = l;
  }

  // MaybeHandlePassageThroughSurface (rendering_randomwalk_impl.hxx:516-527).
  void MaybeHandlePassage(const Node& n, V3 dir, MediumTracker& mt) const {
    if (n.IsSurface() && Dot(dir, n.surf.normal) < 0.)
      GoingThroughSurface(sc, mt, dir, Ff(n.surf.geometry_normal), sc.mat_of_tri[n.surf.prim]);
  }

  // TransmittanceEstimate (rendering_util.cxx:40-67): occlusion by surfaces, then the
  // product of the media's transmittances over the boundary-delimited segments.
  // Ratio tracking through heterogeneous media draws from `shadow`, a stream seeded from
  // the path's stream at the connection, so that the path's own stream advances as it
  // would without media.
  S3 TransmittanceEstimate(V3 org, V3 dir, double length, MediumTracker& mt, VolCoeffs* coeff, Sampler& shadow) {
    length *= 0.9999;
    double t, u, v;
    if (Trace(sc, sc.surf, org, dir, 0., length, true, &t, &u, &v) >= 0) return S3(0.);
    std::vector<Crossing> hits;
    AllHits(sc, sc.vol, org, dir, 0., length, hits);
    S3 result(1.);
    double snear = 0.;
    size_t k = 0;
    while (snear != length) {
      const double sfar = k < hits.size() ? hits[k].t : length;
      const int medium = mt.current;
      const V3 sorg = org + dir * snear;
      if (coeff) Accumulate(*coeff, VolumeCoeffs(sc, medium, sorg, dir, sfar - snear, ctx.idx), snear == 0., sfar == length);
      result = result * SegmentTransmission(sc, medium, sorg, dir, sfar - snear, shadow, ctx.idx);
      if (k >= hits.size()) break;
      GoingThroughSurface(sc, mt, dir, hits[k].n, hits[k].material);
      snear = hits[k].t;
      ++k;
    }
    return result;
  }

  // CalculateConnection, rendering_randomwalk_impl.hxx:373-409.
  S3 CalculateConnection(const Node& eye, const MediumTracker& eye_mt, const Node& light, double* pdf_source,
                         V3* seg_dir, double* seg_len, VolCoeffs* coeff) {
    V3 org, dir;
    double len;
    SegmentToTarget(eye, light, &org, &dir, &len);
    *seg_dir = dir;
    *seg_len = len;
    S3 sf = Evaluate(eye, dir, pdf_source);
    S3 tf = Evaluate(light, -dir, nullptr);
    if (sf.IsZero() || tf.IsZero()) return S3(0.);
    sf = sf * DFactorOf(eye, dir);
    tf = tf * DFactorOf(light, -dir);
    MediumTracker mt = eye_mt;
    MaybeHandlePassage(eye, dir, mt);
    Sampler shadow;
    SeedPath(shadow.g, smp.g.state, smp.g.inc);
    const S3 T = TransmittanceEstimate(org, dir, len, mt, coeff, shadow);
    bool wrt_solid_angle = eye.type == ENV || light.type == ENV;
    double r2 = wrt_solid_angle ? 1. : 1. / Sqr(len);
    return T * sf * tf * r2;
  }

  // PdfConversionFactor, rendering_randomwalk_impl.hxx:493-513.
  double PdfConversionFactor(const Node& src, const Node& tgt, V3 dir, double len, const VolCoeffs& coeff,
                             bool parallel) const {
    double factor = DFactorOf(tgt, dir);
    if (src.type != ENV && tgt.type != ENV && !parallel) factor /= (Sqr(len) + Eps);
    factor *= tgt.IsVolume() ? coeff.fwd : coeff.tr;
    return factor;
  }

  double MisWeight(double pdf_taken, bool taken_delta, double pdf_other) const {
    if (!taken_delta && do_sample_brdf && do_sample_lights) return PowerHeuristic(pdf_taken, pdf_other);
    return 1.;
  }

  struct Step {
    Node node;
    V3 ray_dir;
    double seg_len = 0;
    double scatter_pdf = 0;
    bool scatter_delta = false;
    S3 beta_factor;
    VolCoeffs coeff;
  };

  // TakeRandomWalkStep, rendering_randomwalk_impl.hxx:285-363, with TrackToNextInteraction
  // (rendering_util.hxx:215-269).
  Step TakeRandomWalkStep(const Node& src, MediumTracker& mt) {
    Step st;
    V3 org = src.Coordinates();
    V3 dir;
    S3 value;
    double pdf;
    bool delta;
    if (src.IsVolume()) {  // SamplePhaseFunction x sigma_s
      ScatterSample s = MediumPhaseSample(sc.media[src.medium], src.coords, -src.incident_dir, smp, ctx.idx);
      dir = s.dir; value = s.value * src.sigma_s; pdf = s.pdf; delta = false;
    } else if (src.IsScatter()) {
      const tt_material& m = sc.materials[sc.mat_of_tri[src.surf.prim]].m;
      ScatterSample s = SampleBSDF(m, -src.incident_dir, src.surf, smp, ctx.idx);
      s.value = s.value * BsdfCorrectionFactor(src.surf, s.dir);
      dir = s.dir; value = s.value; pdf = s.pdf; delta = s.delta;
    } else {  // camera
      DirSample s = CameraTakeDirectionSample(sc.cam, src.unit, smp);
      dir = s.dir; value = s.value; pdf = s.pdf; delta = s.delta;
    }
    value = value * DFactorOf(src, dir);
    AddAntiSelfIntersectionOffsetAt(org, src, dir);
    st.beta_factor = value / std::abs(pdf);
    if (st.beta_factor.IsZero()) { st.node.type = ZERO; return st; }
    MaybeHandlePassage(src, dir, mt);
    Step tr = TrackFrom(org, dir, mt);
    tr.beta_factor = st.beta_factor * tr.beta_factor;
    tr.scatter_pdf = std::abs(pdf);
    tr.scatter_delta = delta;
    return tr;
  }

  // TrackToNextInteraction (rendering_util.hxx:215-269): closest surface hit, then spectral
  // tracking through the media between the boundary crossings in front of it.  Returns the
  // node (volume, surface or environment), segment length, tracking weight and the
  // accumulated volume pdf coefficients.
  Step TrackFrom(V3 org, V3 dir, MediumTracker& mt) {
    Step st;
    st.beta_factor = S3(1.);
    double t = 0, u = 0, v = 0;
    double tfar = LargeNumber;
    int prim = Trace(sc, sc.surf, org, dir, 0., LargeNumber, false, &t, &u, &v);
    if (prim >= 0) tfar = t;
    // Volume segments up to 0.9999 of the surface distance.
    const double vend = tfar * 0.9999;
    std::vector<Crossing> hits;
    AllHits(sc, sc.vol, org, dir, 0., vend, hits);
    S3 weight(1.);
    double snear = 0.;
    size_t k = 0;
    while (snear != vend) {
      const double sfar = k < hits.size() ? hits[k].t : vend;
      const int medium = mt.current;
      const V3 sorg = org + dir * snear;
      const InteractionSample ms = SampleInteraction(sc, medium, sorg, dir, sfar - snear, weight, smp, ctx.idx);
      weight = weight * ms.weight;
      const bool interacted = ms.t < sfar - snear;
      const double seglen = interacted ? ms.t : sfar - snear;
      Accumulate(st.coeff, VolumeCoeffs(sc, medium, sorg, dir, seglen, ctx.idx), snear == 0., interacted);
      if (interacted) {
        const double dist = snear + ms.t;
        st.node.type = VOLUME_SCATTER;
        st.node.coords = org + dir * dist;
        st.node.medium = medium;
        st.node.sigma_s = ms.sigma_s;
        st.seg_len = dist;
        st.beta_factor = weight;
        st.node.incident_dir = dir;
        st.ray_dir = dir;
        return st;
      }
      if (k >= hits.size()) break;
      GoingThroughSurface(sc, mt, dir, hits[k].n, hits[k].material);
      snear = hits[k].t;
      ++k;
    }
    st.beta_factor = weight;
    if (prim >= 0) {
      st.node.type = SURFACE_SCATTER;
      st.node.surf = SurfaceFromHit(sc, prim, u, v, org, dir, t);
      st.seg_len = t;
    } else {
      st.node.type = ENV;
      st.node.coords = -dir;
      st.node.radiance = EnvEvaluateTotal(sc, -dir, ctx.idx);
      st.seg_len = LargeNumber;
    }
    st.node.incident_dir = dir;
    st.ray_dir = dir;
    return st;
  }

  // GetPdfOfGeneratingSampleOnEmitter, rendering_randomwalk_impl.hxx:624-651.
  double PdfOfGeneratingSampleOnEmitter(const Node& n) const {
    if (n.type == SURFACE_EMITTER) return (1. / TriArea(sc, n.surf.prim)) * sc.type_probs[1] * sc.in_class[1];
    if (n.type == ENV) return EnvEvaluatePdfTotal(sc, n.coords) * sc.type_probs[0];
    return 0.;
  }

  // PathTracingWorker::RenderPixel, renderingalgorithms_pathtracing.hxx:731-817.
  template <class SplatVec>
  void RenderPixel(int pixel, double rgb_out[3], SplatVec* splats) {
    sensor_connection_unit = -1;
    // LambdaSelectionStrategy::WithWeights, shader_util.hxx:83-91.
    int main_idx = smp.UniformInt(0, 11);
    int32_t idx[3] = {main_idx, main_idx + 12, main_idx + 24};
    int rotation = smp.UniformInt(0, 2);
    std::swap(idx[0], idx[rotation]);
    for (int i = 0; i < 3; ++i) smp.Uniform01();  // SampleWavelengthStrata
    std::memcpy(ctx.idx, idx, sizeof(idx));
    S3 path_sample_values(0.);
    Step step;
    step.node.type = CAMERA;
    step.node.coords = {sc.cam.pos.x, sc.cam.pos.y, sc.cam.pos.z};
    step.node.unit = pixel;
    S3 beta(12.);  // lambda weights (strata size) / delta pdf 1
    int count = 1;
    const int npix = sc.cam.xres * sc.cam.yres;
    MediumTracker mt;
    InitializeMediumTracker(sc, mt, step.node.coords);
    while (true) {
      if (do_sample_lights) {
        double pdf_light;
        bool light_delta;
        Node light = SampleEmissiveEnd(&pdf_light, &light_delta);
        double pdf_scatter = 0;
        V3 sdir;
        double slen;
        VolCoeffs coeff;
        S3 w = CalculateConnection(step.node, mt, light, &pdf_scatter, &sdir, &slen, &coeff);
        double pdf_due = pdf_scatter * PdfConversionFactor(step.node, light, sdir, slen, coeff, false);
        double mis = MisWeight(pdf_light, light_delta, pdf_due);
        S3 pw = w * (mis / pdf_light) * beta;
        if (step.node.type == CAMERA) {
          if (sensor_connection_unit >= 0) {
            pw = pw / (double)npix;
            typename SplatVec::value_type rec;
            rec.unit = sensor_connection_unit;
            SpectralSelectionToRGB(pw, ctx.idx, rec.rgb);
            splats->push_back(rec);
          }
        } else {
          path_sample_values = path_sample_values + pw;
        }
      }
      Node prev = step.node;
      step = TakeRandomWalkStep(prev, mt);
      beta = beta * step.beta_factor;
      ++count;
      if (do_sample_brdf) {
        bool emitter = false;
        if (step.node.type == SURFACE_SCATTER && sc.materials[sc.mat_of_tri[step.node.surf.prim]].m.emissive) {
          step.node.type = SURFACE_EMITTER;
          emitter = true;
        } else if (step.node.type == ENV) {
          emitter = true;
        }
        if (emitter) {
          S3 end_weight = Evaluate(step.node, -step.ray_dir, nullptr);
          double pdf_direct = PdfOfGeneratingSampleOnEmitter(step.node);
          double pdf_due =
              PdfConversionFactor(prev, step.node, step.ray_dir, step.seg_len, step.coeff, step.scatter_delta) *
              step.scatter_pdf;
          double mis = MisWeight(pdf_due, step.scatter_delta, pdf_direct);
          path_sample_values = path_sample_values + end_weight * beta * mis;
          if (step.node.type == SURFACE_EMITTER) step.node.type = SURFACE_SCATTER;
        }
      }
      if (step.node.type == ZERO || step.node.type == ENV) break;
      // SurvivalAtNthScatterNode, rendering_randomwalk_impl.hxx:736-755.
      if (count < max_path_node_count) {
        if (count > 5) {
          double p = std::min(0.9, beta.Max());
          if (smp.Uniform01() > p) break;
          beta = beta * (1. / p);
        }
      } else {
        break;
      }
    }
    SpectralSelectionToRGB(path_sample_values, ctx.idx, rgb_out);
  }
};

// ---------------------------------------------------------------------------------------
// pt2: PathTracingAlgo2 (renderingalgorithms_pathtracing2.cxx:126-700) with the null-path
// estimators of media_integrator.cxx:216-420.  Per wavelength i and sampling wavelength j a
// 3x3 matrix accumulates p_j / f_i over the tracked events (AccumulateContributions); the
// contribution of a path is divided by the row mean, a balance heuristic over the hero
// wavelengths, and NEE against BSDF sampling is weighted with those matrices (MisWeight,
// :452-476).  No Russian roulette (RayTermination::SurvivalAtNthScatterNode with its
// roulette commented out, rendering_util.hxx:383-412), no NEE from the camera, path
// regularisation by the largest microfacet roughness met so far (ShaderQuery::minimum_roughness).
struct M33 {
  double a[3][3];
  static M33 Ones() { M33 m; for (auto& r : m.a) for (double& x : r) x = 1.; return m; }
  static M33 Inf() { M33 m; for (auto& r : m.a) for (double& x : r) x = Infinity; return m; }
};
inline void FixNan(M33& m) { for (auto& r : m.a) for (double& x : r) if (std::isnan(x)) x = Infinity; }
inline void Acc(M33& w, const M33& x) {  // AccumulateContributions(w, x), media_integrator.cxx:223-229
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) w.a[i][j] *= x.a[i][j];
  FixNan(w);
}
inline void Acc(M33& w, S3 f, S3 p) {  // AccumulateContributions(w, f, p), :231-238
  M33 t;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      t.a[i][j] = (1. / f[i]) * p[j];
      if (std::isnan(t.a[i][j])) t.a[i][j] = Infinity;
    }
  Acc(w, t);
}
inline S3 RowMean(const M33& m) {
  return {(m.a[0][0] + m.a[0][1] + m.a[0][2]) / 3., (m.a[1][0] + m.a[1][1] + m.a[1][2]) / 3.,
          (m.a[2][0] + m.a[2][1] + m.a[2][2]) / 3.};
}
inline S3 RowMeanScaledFixNan(const M33& m, double s) {
  M33 t = m;
  for (auto& r : t.a) for (double& x : r) x *= s;
  FixNan(t);
  return RowMean(t);
}

struct Factors { M33 track = M33::Ones(), nulls = M33::Ones(); };

struct Worker2 {
  const Scene& sc;
  Sampler smp;
  PathCtx ctx;
  bool use_nee = true, use_emission = true;
  int max_node_count;
  explicit Worker2(const Scene& s) : sc(s) {
    max_node_count = s.params.max_ray_depth;
    if (s.params.pt_sample_mode == TT_SAMPLE_BSDF) use_nee = false;
    if (s.params.pt_sample_mode == TT_SAMPLE_LIGHTS) use_emission = false;
    if (s.env.empty() && s.area_lights.empty() && s.points.empty()) use_nee = false;
  }

  // Medium::ComputeMajorante and EvaluateCoeffs; medium -1 is the vacuum.
  S3 Majorant(int medium, V3 org, V3 dir, double len) const {
    if (medium < 0) return S3(0.);
    const MediumDesc& m = sc.media[medium];
    if (m.kind == TT_MEDIUM_ATMOSPHERE) return S3(AtmSegmentMajorant(m, org, dir, len));
    return TakeD3(m.sigma_ext, ctx.idx);
  }
  void Coeffs(int medium, V3 pos, S3* ss, S3* st) const {
    if (medium < 0) { *ss = S3(0.); *st = S3(0.); return; }
    const MediumDesc& m = sc.media[medium];
    if (m.kind == TT_MEDIUM_ATMOSPHERE) { AtmCoeffs(m, Altitude(m, pos), ctx.idx, ss, st); return; }
    *ss = TakeD3(m.sigma_s, ctx.idx);
    *st = TakeD3(m.sigma_ext, ctx.idx);
  }
  static S3 Exp(S3 maj, double x) { return {std::exp(-x * maj[0]), std::exp(-x * maj[1]), std::exp(-x * maj[2])}; }
  static S3 Sub(S3 a, S3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }

  // nullpath::Tracking on one segment (media_integrator.cxx:240-286): hero-wavelength delta
  // tracking.  Returns true at a real collision (distance *t, scattering coefficient *ss).
  bool TrackSegment(int medium, V3 org, V3 dir, double len, Factors& f, double* t_out, S3* ss_out) {
    const S3 maj = Majorant(medium, org, dir, len);
    const double mfp = 1. / maj[0];
    double t = 0.;
    for (int it = 1; it < 10000; ++it) {
      const double tlocal = std::min(LargeNumber, -std::log(1.0 - smp.Uniform01()) * mfp);
      const S3 tr = Exp(maj, std::min(tlocal, len - t));
      t += tlocal;
      S3 ss, st;
      Coeffs(medium, org + dir * t, &ss, &st);
      if (t >= len) {
        Acc(f.track, tr, tr);
        Acc(f.nulls, tr, tr);
        return false;
      }
      const S3 sn = Sub(maj, st);
      const double prob_n = sn[0] * mfp;
      if (smp.Uniform01() < prob_n) {
        Acc(f.track, tr * sn, tr * sn);
        Acc(f.nulls, tr * sn, tr * maj);
      } else {
        Acc(f.track, tr * st, tr * st);
        Acc(f.nulls, tr * st, tr);
        *t_out = t;
        *ss_out = ss;
        return true;
      }
    }
    return false;  // iteration cap: no collision
  }

  // nullpath::Transmission on one segment (:288-325).
  void TransmitSegment(int medium, V3 org, V3 dir, double len, Factors& f, Sampler& s) {
    const S3 maj = Majorant(medium, org, dir, len);
    const double mfp = 1. / maj[0];
    double t = 0.;
    for (int it = 1; it < 10000; ++it) {
      const double tlocal = std::min(LargeNumber, -std::log(1.0 - s.Uniform01()) * mfp);
      const S3 tr = Exp(maj, std::min(tlocal, len - t));
      t += tlocal;
      if (t >= len) {
        Acc(f.track, tr, tr);
        Acc(f.nulls, tr, tr);
        return;
      }
      S3 ss, st;
      Coeffs(medium, org + dir * t, &ss, &st);
      const S3 sn = Sub(maj, st);
      Acc(f.track, tr * sn, tr * sn);
      Acc(f.nulls, tr * sn, tr * maj);
      if (f.nulls.a[0][0] > LargeNumber && f.nulls.a[1][1] > LargeNumber && f.nulls.a[2][2] > LargeNumber) {
        f.nulls = M33::Inf();
        return;
      }
    }
  }

  // MisWeight (renderingalgorithms_pathtracing2.cxx:452-476).
  std::pair<double, S3> MisWeight(bool has_pdf, double pdf, bool delta, double pdf_other, const M33& d,
                                  const M33& d_other) const {
    if (!has_pdf || delta || !(use_nee && use_emission)) return {1., RowMean(d)};
    const S3 a = RowMeanScaledFixNan(d, pdf), b = RowMeanScaledFixNan(d_other, pdf_other);
    return {pdf, a + b};
  }

  static S3 Div(S3 a, S3 b) { return {a[0] / b[0], a[1] / b[1], a[2] / b[2]}; }

  struct State {
    V3 org, dir;
    MediumTracker mt;
    M33 wt, wtn;
    S3 path_weights;
    bool has_last = false, last_delta = false;
    double last_pdf = 0.;
    double roughness = 0.;
    int count = 0;
  };

  // AddDirectLighting (:479-560).  `vol_medium` >= 0 for a volume interaction at `pos`.
  S3 DirectLighting(const State& ps, const Surf* si, V3 pos, int vol_medium) {
    const int which = TowerSampling4(sc.type_probs, smp.Uniform01());
    const int nlights = which == 0 ? 1 : (which == 1 ? (int)sc.area_lights.size() : (int)sc.points.size());
    // TowerSamplingBisection over a uniform CMF: the first index whose (k + 1) / n exceeds r.
    const double rr = smp.Uniform01();
    int li = std::min(nlights - 1, std::max(0, (int)(rr * nlights)));
    while (li > 0 && rr < (double)li / nlights) --li;
    while (li < nlights - 1 && rr >= (double)(li + 1) / nlights) ++li;
    const double prob = sc.type_probs[which] * (1. / nlights);
    V3 org = si ? si->pos : pos, dir;
    double len;
    double pdf;
    bool delta = false;
    S3 light_weight;
    if (which == 0) {
      const DirSample e = EnvTakeDirectionSampleTotal(sc, smp, ctx.idx);
      dir = -e.dir;
      len = sc.long_distance;
      if (si) org = org + AntiSelfIntersectionOffset(*si, dir);
      pdf = e.pdf;
      delta = e.delta;
      light_weight = e.value / (e.pdf * prob);
    } else {
      V3 lpos, lng, lns;
      S3 val;
      double area_pdf;
      if (which == 1) {
        const int prim = sc.area_lights[li];
        double r[2];
        smp.UniformUnitSquare(r);
        const V3 b = IsSphere(sc, prim) ? ToUniformSphere(r) * sc.sph_r[prim - sc.ntri] : ToTriangleBarycentricCoords(r);
        const Surf ls = SurfaceFromBarycentric(sc, prim, b);
        lpos = ls.pos;
        lng = ls.geometry_normal;
        lns = ls.shading_normal;
        area_pdf = 1. / TriArea(sc, prim);
      } else {
        lpos = {sc.points[li].pos[0], sc.points[li].pos[1], sc.points[li].pos[2]};
        area_pdf = 1.;
        delta = true;
      }
      // Detail::SegmentToPoint (light.cxx:239-266): offset at the eye end only.
      const V3 dd = lpos - org;
      len = Length(dd);
      if (len > 0.) dir = dd / len;
      else { len = Eps; dir = si ? si->normal : V3{1., 0., 0.}; }
      if (si) org = org + AntiSelfIntersectionOffset(*si, dir);
      if (which == 1) {
        const tt_material& lm = sc.materials[sc.mat_of_tri[sc.area_lights[li]]].m;
        const double vis = Dot(lng, -dir) > 0. ? 1. : 0.;
        val = Take(lm.emission, ctx.idx) * (vis / (2. * Pi)) * std::abs(Dot(lns, dir));
        pdf = Sqr(len) / std::abs(Dot(dir, lng) + Eps) * area_pdf;
      } else {
        val = Take(sc.points[li].spectrum, ctx.idx) * (1. / (4. * Pi));
        pdf = Sqr(len) / std::abs(0. + Eps) * area_pdf;
      }
      light_weight = val / (area_pdf * prob) / Sqr(len);
    }
    S3 pw = ps.path_weights;
    MediumTracker mt = ps.mt;
    double bsdf_pdf = 0.;
    if (si) {
      pw = pw * std::abs(Dot(si->shading_normal, dir));
      const tt_material& m = sc.materials[sc.mat_of_tri[si->prim]].m;
      pw = pw * EvaluateBSDF(m, -ps.dir, *si, dir, ctx.idx, &bsdf_pdf, ps.roughness);
      if (Dot(dir, si->normal) < 0.) GoingThroughSurface(sc, mt, dir, Ff(si->geometry_normal), sc.mat_of_tri[si->prim]);
    } else {
      S3 ss, st;
      pw = pw * MediumPhaseEvaluate(sc.media[vol_medium], pos, -ps.dir, dir, ctx.idx, &bsdf_pdf);
      Coeffs(vol_medium, pos, &ss, &st);
      pw = pw * Div(ss, st + S3(Eps));
    }
    // nullpath::Transmission (:384-420) on a stream seeded from the path's state here; a
    // quasi-random sampler continues the subsequence of the light sample.
    Sampler shadow = smp;
    SeedPath(shadow.g, smp.g.state, smp.g.inc);
    Factors f;
    const double slen = len * 0.9999;
    double t, u, v;
    if (Trace(sc, sc.surf, org, dir, 0., slen, true, &t, &u, &v) >= 0) {
      f.track = M33::Inf();
      f.nulls = M33::Inf();
    } else {
      std::vector<Crossing> hits;
      AllHits(sc, sc.vol, org, dir, 0., slen, hits);
      double snear = 0.;
      size_t k = 0;
      while (true) {
        const double sfar = k < hits.size() ? hits[k].t : slen;
        Factors seg;
        TransmitSegment(mt.current, org + dir * snear, dir, sfar - snear, seg, shadow);
        Acc(f.nulls, seg.nulls);
        Acc(f.track, seg.track);
        if (k >= hits.size()) break;
        GoingThroughSurface(sc, mt, dir, hits[k].n, hits[k].material);
        snear = sfar;
        ++k;
      }
    }
    Acc(f.track, ps.wt);
    Acc(f.nulls, ps.wt);
    const auto mw = MisWeight(true, pdf, delta, bsdf_pdf, f.nulls, f.track);
    return Div(pw * light_weight * mw.first, mw.second);
  }

  void RenderPixel(int pixel, double rgb_out[3]) {
    int main_idx = smp.UniformInt(0, 11);
    int32_t idx[3] = {main_idx, main_idx + 12, main_idx + 24};
    int rotation = smp.UniformInt(0, 2);
    std::swap(idx[0], idx[rotation]);
    for (int i = 0; i < 3; ++i) smp.Uniform01();
    std::memcpy(ctx.idx, idx, sizeof(idx));
    smp.SetSubsequenceId(2);  // PrepSamplerDimension at node count 1 (the camera direction)
    State ps;
    ps.wt = M33::Ones();
    ps.wtn = M33::Ones();
    ps.path_weights = S3(12.);
    ps.org = {sc.cam.pos.x, sc.cam.pos.y, sc.cam.pos.z};
    const DirSample cs = CameraTakeDirectionSample(sc.cam, pixel, smp);
    ps.path_weights = ps.path_weights * (cs.value / cs.pdf);
    ps.dir = cs.dir;
    InitializeMediumTracker(sc, ps.mt, ps.org);
    ps.count = 2;
    S3 total(0.);
    if (ps.path_weights.IsZero()) { SpectralSelectionToRGB(total, ctx.idx, rgb_out); return; }
    while (true) {
      // nullpath::Tracking (:330-378): closest hit, then the segments in front of it.
      double t = 0, u = 0, v = 0;
      const int prim = Trace(sc, sc.surf, ps.org, ps.dir, 0., LargeNumber, false, &t, &u, &v);
      const double tfar = prim >= 0 ? t : LargeNumber;
      const double vend = tfar * 0.9999;
      std::vector<Crossing> hits;
      AllHits(sc, sc.vol, ps.org, ps.dir, 0., vend, hits);
      Factors f;
      bool volume = false;
      int vmed = -1;
      V3 vpos;
      S3 vss;
      double snear = 0.;
      size_t k = 0;
      while (true) {
        const double sfar = k < hits.size() ? hits[k].t : vend;
        const int medium = ps.mt.current;
        Factors seg;
        double tc;
        S3 ss;
        const bool hit_medium = TrackSegment(medium, ps.org + ps.dir * snear, ps.dir, sfar - snear, seg, &tc, &ss);
        Acc(f.nulls, seg.nulls);
        Acc(f.track, seg.track);
        if (hit_medium) {
          volume = true;
          vmed = medium;
          vpos = ps.org + ps.dir * (snear + tc);
          vss = ss;
          break;
        }
        if (k >= hits.size()) break;
        GoingThroughSurface(sc, ps.mt, ps.dir, hits[k].n, hits[k].material);
        snear = sfar;
        ++k;
      }
      ps.wtn = ps.wt;
      Acc(ps.wtn, f.nulls);
      Acc(ps.wt, f.track);
      if (!volume && prim < 0) {
        // AddEnvEmission (:625-648).
        if (use_emission && !sc.env.empty()) {
          const S3 rad = EnvEvaluateTotal(sc, -ps.dir, ctx.idx);
          const double pdf_env = EnvEvaluatePdfTotal(sc, -ps.dir) * sc.type_probs[0];
          const auto mw = ps.has_last ? MisWeight(true, ps.last_pdf, ps.last_delta, pdf_env, ps.wt, ps.wtn)
                                      : MisWeight(false, 0., false, 1., ps.wt, ps.wtn);
          total = total + Div(rad * ps.path_weights * mw.first, mw.second);
        }
        break;
      }
      ScatterSample s;
      Surf si;
      if (!volume) {
        si = SurfaceFromHit(sc, prim, u, v, ps.org, ps.dir, t);
        const tt_material& m = sc.materials[sc.mat_of_tri[prim]].m;
        smp.SetSubsequenceId(((uint32_t)ps.count << 1) | 1u);  // PrepSamplerDimension(NEE_LIGHT)
        // MaybeAddEmission (:592-622).
        if (use_emission && m.emissive) {
          const double vis = Dot(si.geometry_normal, -ps.dir) > 0. ? 1. : 0.;
          const S3 rad = Take(m.emission, ctx.idx) * (vis / (2. * Pi));
          std::pair<double, S3> mw;
          if (ps.has_last) {
            const double prob_select = sc.type_probs[1] * sc.in_class[1];
            const double area_pdf = 1. / TriArea(sc, prim);
            const double cvt = Sqr(Length(ps.org - si.pos)) / std::abs(Dot(ps.dir, si.normal) + Eps);
            mw = MisWeight(true, ps.last_pdf, ps.last_delta, prob_select * area_pdf * cvt, ps.wt, ps.wtn);
          } else {
            mw = MisWeight(false, 0., false, 1., ps.wt, ps.wtn);
          }
          total = total + Div(rad * ps.path_weights * mw.first, mw.second);
        }
        if (use_nee) total = total + DirectLighting(ps, &si, si.pos, -1);
        smp.SetSubsequenceId((uint32_t)ps.count << 1);  // PrepSamplerDimension(BSDF)
        // SampleScatterer (:571-583): the query sees the roughness before this vertex.
        s = SampleBSDF(m, -ps.dir, si, smp, ctx.idx, ps.roughness);
        ps.roughness = std::max(MyRoughness(m), ps.roughness);
      } else {
        smp.SetSubsequenceId(((uint32_t)ps.count << 1) | 1u);
        if (use_nee) total = total + DirectLighting(ps, nullptr, vpos, vmed);
        smp.SetSubsequenceId((uint32_t)ps.count << 1);
        s = MediumPhaseSample(sc.media[vmed], vpos, -ps.dir, smp, ctx.idx);
        S3 ss, st;
        Coeffs(vmed, vpos, &ss, &st);
        s.value = s.value * Div(ss, st + S3(Eps));
      }
      ps.count++;
      if (ps.count > max_node_count) break;
      // PrepareStateForAfterScattering (:585-604).
      if (!volume) {
        ps.path_weights = ps.path_weights * s.value * (std::abs(Dot(si.shading_normal, s.dir)) / s.pdf);
        ps.org = si.pos + AntiSelfIntersectionOffset(si, s.dir);
        if (Dot(s.dir, si.normal) < 0.) GoingThroughSurface(sc, ps.mt, s.dir, Ff(si.geometry_normal), sc.mat_of_tri[prim]);
      } else {
        ps.path_weights = ps.path_weights * s.value / s.pdf;
        ps.org = vpos;
      }
      ps.dir = s.dir;
      ps.has_last = true;
      ps.last_pdf = s.pdf;
      ps.last_delta = s.delta;
      // A path whose weights vanished adds nothing more (stopped here; the reference would
      // continue it to the depth limit).
      if (ps.path_weights.IsZero() || !(s.pdf > 0.)) break;
    }
    SpectralSelectionToRGB(total, ctx.idx, rgb_out);
  }
};

// ---------------------------------------------------------------------------------------
// Generator matrix of one Sobol dimension as the reference's generator notebook builds it
// (misc/SobolSequenceGeneratorMatrices.ipynb, MakeTheMatrix): the s initial direction
// numbers, then for k >= s m_k = m_{k-s} ^ 2^s m_{k-s} ^ the terms 2^(s-1-i) m_{k-s+i+1}
// for which bit (s - 2 - i) of a is set; finally column k is m_k shifted left by 31 - k.
static void SobolMatrix(int s, int a, const uint16_t* m_init, uint32_t* C) {
  uint64_t m[32];
  for (int k = 0; k < 32; ++k) {
    if (k < s) { m[k] = m_init[k]; continue; }
    uint64_t pow2 = 1ull << s;
    m[k] = m[k - s] ^ (pow2 * m[k - s]);
    for (int i = 0; i < s - 1; ++i) {
      pow2 >>= 1;
      if (a & (1 << (s - 2 - i))) m[k] ^= pow2 * m[k - s + i + 1];
    }
  }
  for (int k = 0; k < 32; ++k) C[k] = (uint32_t)(m[k] << (31 - k));
}

// All dimensions: 0 is MakeIdentityGenerator, d >= 1 the Joe-Kuo line d + 1.
static void SobolMatrices(std::vector<uint32_t>& C) {
  C.assign((size_t)TT_SOBOL_DIMS * 32, 0u);
  for (int k = 0; k < 32; ++k) C[k] = 1u << (31 - k);
  const uint16_t* q = tt_sobol_sam;
  for (int d = 1; d < TT_SOBOL_DIMS; ++d) {
    const int s = q[0], a = q[1];
    SobolMatrix(s, a, q + 2, &C[32 * (size_t)d]);
    q += 2 + s;
  }
}

static bool BuildScene(Scene& s, const tt_scene_desc* d, const tt_params* p) {
  if (!d || !p) { g_err = "null argument"; return false; }
  s.params = *p;
  if (s.params.max_ray_depth <= 0) s.params.max_ray_depth = 25;
  if (s.params.algo == TT_ALGO_PT2 && s.params.qmc) {
    if (s.params.max_ray_depth > 31) { g_err = "qmc needs max_ray_depth <= 31"; return false; }
    SobolMatrices(s.sobol);
  }
  s.vert.resize(d->num_vertices);
  for (uint32_t i = 0; i < d->num_vertices; ++i)
    s.vert[i] = {d->vertices[3 * i], d->vertices[3 * i + 1], d->vertices[3 * i + 2]};
  s.has_normals = d->normals != nullptr;
  if (s.has_normals) {
    s.nrm.resize(d->num_vertices);
    for (uint32_t i = 0; i < d->num_vertices; ++i)
      s.nrm[i] = {d->normals[3 * i], d->normals[3 * i + 1], d->normals[3 * i + 2]};
  }
  s.idx.assign(d->indices, d->indices + 3 * (size_t)d->num_triangles);
  s.mat_of_tri.assign(d->material_ids, d->material_ids + d->num_triangles);
  if (d->uvs) s.uv.assign(d->uvs, d->uvs + 2 * (size_t)d->num_vertices);
  for (uint32_t i = 0; i < d->num_textures; ++i) {
    const tt_texture& t = d->textures[i];
    if (!t.rgb || t.width <= 0 || t.height <= 0) { g_err = "bad texture"; return false; }
    Texture tx;
    tx.w = t.width;
    tx.h = t.height;
    tx.rgb.assign(t.rgb, t.rgb + 3 * (size_t)t.width * t.height);
    s.textures.push_back(std::move(tx));
  }
  for (uint32_t i = 0; i < d->num_media; ++i) {
    const tt_medium& m = d->media[i];
    MediumDesc md;
    md.priority = m.priority;
    md.is_scattering = false;
    for (int b = 0; b < NBINS; ++b) {
      md.sigma_s[b] = m.sigma_s[b];
      md.sigma_a[b] = m.sigma_a[b];
      md.sigma_ext[b] = md.sigma_s[b] + md.sigma_a[b];
      md.is_scattering |= md.sigma_s[b] > 0.;
    }
    md.phase = m.phase;
    md.g = m.phase_g;
    md.kind = m.kind;
    if (m.kind == TT_MEDIUM_ATMOSPHERE) {
      // TabulatedConstituents::TabulatedConstituents, atmosphere.cxx:234-276.
      if (m.table_size < 2 || !m.sigma_t || !m.sigma_s_molecules || !m.sigma_s_aerosols || !(m.table_dh > 0.f)) {
        g_err = "bad atmosphere table";
        return false;
      }
      md.is_scattering = true;
      md.center = {m.planet_center[0], m.planet_center[1], m.planet_center[2]};
      md.radius = m.planet_radius;
      md.n = m.table_size;
      md.h0 = m.table_h0;
      md.dh = m.table_dh;
      md.inv_dh = 1. / md.dh;
      md.sig_t.assign(m.sigma_t, m.sigma_t + (size_t)md.n * NBINS);
      md.sig_mol.assign(m.sigma_s_molecules, m.sigma_s_molecules + (size_t)md.n * NBINS);
      md.sig_aer.assign(m.sigma_s_aerosols, m.sigma_s_aerosols + (size_t)md.n * NBINS);
      md.maj.resize(md.n);
      for (int r = 0; r < md.n; ++r) {
        double mx = 0.;
        for (int b = 0; b < NBINS; ++b) mx = std::max(mx, md.sig_t[(size_t)r * NBINS + b]);
        md.maj[r] = mx;
      }
      for (int r = md.n - 2; r >= 0; --r) md.maj[r] = std::max(md.maj[r], md.maj[r + 1]);
    } else if (m.kind != TT_MEDIUM_HOMOGENEOUS) {
      g_err = "unknown medium kind";
      return false;
    }
    s.media.push_back(md);
  }
  for (uint32_t i = 0; i < d->num_materials; ++i) {
    const tt_material& m = d->materials[i];
    if (m.medium_inside < 0 || m.medium_inside > (int)d->num_media || m.medium_outside < 0 ||
        m.medium_outside > (int)d->num_media) {
      g_err = "medium index out of range";
      return false;
    }
    if (m.diffuse_texture < 0 || m.diffuse_texture > (int)d->num_textures) {
      g_err = "texture index out of range";
      return false;
    }
    s.materials.push_back(Material{m});
  }
  for (uint32_t t = 0; t < d->num_triangles; ++t) {
    for (int k = 0; k < 3; ++k)
      if (s.idx[3 * t + k] >= d->num_vertices) { g_err = "vertex index out of range"; return false; }
    if (s.mat_of_tri[t] >= d->num_materials) { g_err = "material index out of range"; return false; }
    s.tv0.push_back(VertD(s, s.idx[3 * t]));
    s.tv1.push_back(VertD(s, s.idx[3 * t + 1]));
    s.tv2.push_back(VertD(s, s.idx[3 * t + 2]));
    const tt_material& m = s.materials[s.mat_of_tri[t]].m;
    if (m.volume_boundary) {
      s.vol.tris.push_back((int)t);
    } else {
      s.surf.tris.push_back((int)t);
      if (m.emissive) s.area_lights.push_back((int)t);
    }
  }
  s.ntri = d->num_triangles;
  if (d->num_spheres > 0 && (!d->spheres || !d->sphere_material_ids)) { g_err = "sphere arrays missing"; return false; }
  for (uint32_t i = 0; i < d->num_spheres; ++i) {
    const float* q = d->spheres + 4 * (size_t)i;
    const uint32_t mat = d->sphere_material_ids[i];
    if (mat >= d->num_materials) { g_err = "sphere material index out of range"; return false; }
    if (!(q[3] > 0.f)) { g_err = "sphere radius must be positive"; return false; }
    s.sph_c.push_back({q[0], q[1], q[2]});
    s.sph_r.push_back(q[3]);
    s.mat_of_tri.push_back(mat);
    const int prim = (int)(d->num_triangles + i);
    const tt_material& m = s.materials[mat].m;
    if (m.volume_boundary) {
      s.vol.tris.push_back(prim);
    } else {
      s.surf.tris.push_back(prim);
      if (m.emissive) s.area_lights.push_back(prim);
    }
  }
  for (int k = 0; k < 3; ++k) { s.bb_lo[k] = 1e300; s.bb_hi[k] = -1e300; }
  for (auto& v : s.vert) {
    double c[3] = {v.x, v.y, v.z};
    for (int k = 0; k < 3; ++k) { s.bb_lo[k] = std::min(s.bb_lo[k], c[k]); s.bb_hi[k] = std::max(s.bb_hi[k], c[k]); }
  }
  for (size_t i = 0; i < s.sph_c.size(); ++i)
    for (int k = 0; k < 3; ++k) {
      s.bb_lo[k] = std::min(s.bb_lo[k], s.sph_c[i][k] - s.sph_r[i]);
      s.bb_hi[k] = std::max(s.bb_hi[k], s.sph_c[i][k] + s.sph_r[i]);
    }
  if (s.vert.empty() && s.sph_c.empty()) for (int k = 0; k < 3; ++k) { s.bb_lo[k] = 0; s.bb_hi[k] = 0; }
  s.diag = std::sqrt(Sqr(s.bb_hi[0] - s.bb_lo[0]) + Sqr(s.bb_hi[1] - s.bb_lo[1]) + Sqr(s.bb_hi[2] - s.bb_lo[2]));
  s.long_distance = 10. * s.diag;
  s.box_center = {0.5 * (s.bb_lo[0] + s.bb_hi[0]), 0.5 * (s.bb_lo[1] + s.bb_hi[1]), 0.5 * (s.bb_lo[2] + s.bb_hi[2])};
  for (uint32_t i = 0; i < d->num_point_lights; ++i) s.points.push_back(d->point_lights[i]);
  for (uint32_t i = 0; i < d->num_env_lights; ++i) {
    const tt_env_light& e = d->env_lights[i];
    EnvLight L;
    L.kind = e.kind;
    for (int b = 0; b < NBINS; ++b) L.spectrum[b] = e.spectrum[b];
    L.dir = {e.dir[0], e.dir[1], e.dir[2]};
    L.scalar = e.scalar;
    L.scalar2 = e.scalar2;
    if (e.kind == TT_ENV_SUN) {
      // Sun::Sun, light.hxx:253-263.
      L.cos_opening = std::cos(Pi / 180. * L.scalar2);
      L.pdf_val = 1. / (2. * Pi * (1. - L.cos_opening));
      L.frame = OrthogonalSystemZAligned(Normalized(L.dir));
      for (int b = 0; b < NBINS; ++b) L.sun_emission[b] = kSunSpectrum[b] * L.scalar * L.pdf_val;
    } else if (e.kind == TT_ENV_DOME) {
      L.down_dir = -Normalized(L.dir);
      L.frame = OrthogonalSystemZAligned(L.down_dir);
    } else if (e.kind == TT_ENV_DIRECTIONAL) {
      L.dir = Normalized(L.dir);
    } else if (e.kind == TT_ENV_MAP) {
      if (!e.tex_rgb || e.tex_width <= 0 || e.tex_height <= 0) { g_err = "env map without texture"; return false; }
      L.w = e.tex_width;
      L.h = e.tex_height;
      L.tex.assign(e.tex_rgb, e.tex_rgb + 3 * (size_t)L.w * L.h);
      // Float frame, EnvMapLight ctor (light.cxx:88-115).
      float up[3] = {(float)L.dir.x, (float)L.dir.y, (float)L.dir.z};
      float sign = std::copysign(1.0f, up[2]);
      const float a = -1.0f / (sign + up[2]);
      const float b = up[0] * up[1] * a;
      float X[3] = {1.0f + sign * up[0] * up[0] * a, sign * b, -sign * up[0]};
      float Y[3] = {b, sign + up[1] * up[1] * a, -up[1]};
      for (int k = 0; k < 3; ++k) { L.fX[k] = X[k]; L.fY[k] = Y[k]; L.fZ[k] = up[k]; }
      L.cmf_rows.assign(L.h, 0.f);
      L.cmf_cols.assign((size_t)L.w * L.h, 0.f);
      for (int y = 0; y < L.h; ++y) {
        double row_weight = 0.;
        for (int x = 0; x < L.w; ++x) {
          const float* px = &L.tex[3 * ((size_t)y * L.w + x)];
          double mean = ((double)px[0] + px[1] + px[2]) / 3.;
          // PixelCenterToUv + UvToSpherical: theta = v * pi, v = (h - 1 - y + 0.5) / h.
          float v = ((float)(L.h - 1 - y) + 0.5f) / L.h;
          float theta = v * (float)Pi;
          double weight = std::sin(theta) * mean;
          row_weight += weight;
          L.cmf_cols[(size_t)y * L.w + x] = (float)row_weight;
        }
        for (int x = 0; x < L.w; ++x) L.cmf_cols[(size_t)y * L.w + x] /= (float)row_weight;
        L.cmf_rows[y] = (float)row_weight;
      }
      for (int y = 1; y < L.h; ++y) L.cmf_rows[y] += L.cmf_rows[y - 1];
      float inv = 1.f / L.cmf_rows[L.h - 1];
      for (int y = 0; y < L.h; ++y) L.cmf_rows[y] *= inv;
    } else {
      g_err = "unknown env light kind";
      return false;
    }
    s.env.push_back(std::move(L));
  }
  // TrivialLightPicker ctor, lightpicker_trivial.cxx:11-31.
  const double nl = (double)s.points.size(), ne = s.env.empty() ? 0. : 1., na = (double)s.area_lights.size();
  const double norm = 1. / (nl + ne + na);
  s.type_probs[0] = ne * norm;
  s.type_probs[1] = na * norm;
  s.type_probs[2] = nl * norm;
  s.type_probs[3] = 0.;
  s.in_class[0] = ne > 0 ? 1. / ne : NAN;
  s.in_class[1] = na > 0 ? 1. / na : NAN;
  s.in_class[2] = nl > 0 ? 1. / nl : NAN;
  s.in_class[3] = 0;
  // Camera (camera.hxx:38-108, 159-175).
  const tt_camera& c = d->camera;
  Camera& cam = s.cam;
  cam.kind = c.kind;
  cam.pos = {c.pos[0], c.pos[1], c.pos[2]};
  cam.xres = c.xres;
  cam.yres = c.yres;
  if (c.xres <= 0 || c.yres <= 0) { g_err = "bad camera resolution"; return false; }
  V3 up = Normalized(V3{c.up[0], c.up[1], c.up[2]});
  V3 dir = Normalized(V3{c.dir[0], c.dir[1], c.dir[2]});
  double r = Dot(dir, up);
  if (!(std::abs(r) > 1.0 - Eps)) up = Normalized(up - r * dir);
  cam.up = up;
  cam.dir = dir;
  cam.right = Cross(up, dir);
  double fov = c.fov_deg * Pi / 180.;
  double aspect = (double)c.yres / c.xres;
  double a = std::tan(fov * 0.5);
  double b = a * aspect;
  cam.xmin = -a;
  cam.ymin = -b;
  cam.xperpixel = 2. * a / c.xres;
  cam.yperpixel = 2. * b / c.yres;
  cam.per_pixel_delta = 2. / std::min(c.xres, c.yres);
  BuildBvh(s, s.surf);
  BuildBvh(s, s.vol);
  return true;
}

}  // namespace orc

using namespace orc;

struct or_scene {
  Scene s;
};

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

or_scene* or_create(const tt_scene_desc* scene, const tt_params* params) {
  auto* o = new or_scene;
  if (!BuildScene(o->s, scene, params)) {
    delete o;
    return nullptr;
  }
  return o;
}

void or_destroy(or_scene* s) { delete s; }

int or_intersect(or_scene* s, const double* rays, int n, int brute_force, int32_t* prim, double* t, double* u,
                 double* v) {
  for (int i = 0; i < n; ++i) {
    const double* r = rays + 8 * (size_t)i;
    V3 org{r[0], r[1], r[2]}, dir{r[4], r[5], r[6]};
    double tt = 0, uu = 0, vv = 0;
    int p = brute_force ? TraceBrute(s->s, s->s.surf, org, dir, r[3], r[7], &tt, &uu, &vv)
                        : Trace(s->s, s->s.surf, org, dir, r[3], r[7], false, &tt, &uu, &vv);
    prim[i] = p;
    t[i] = p >= 0 ? tt : -1;
    u[i] = uu;
    v[i] = vv;
  }
  return 0;
}

int or_occluded(or_scene* s, const double* rays, int n, uint8_t* occluded) {
  for (int i = 0; i < n; ++i) {
    const double* r = rays + 8 * (size_t)i;
    double tt, uu, vv;
    occluded[i] = Trace(s->s, s->s.surf, {r[0], r[1], r[2]}, {r[4], r[5], r[6]}, r[3], r[7], true, &tt, &uu, &vv) >= 0;
  }
  return 0;
}

int or_render(or_scene* os, int spp, uint64_t seed, int sample_offset, int pixel_begin, int pixel_end, int nthreads,
              double* accum, double* light_accum, uint64_t* splat_count) {
  const Scene& sc = os->s;
  const int npix = sc.cam.xres * sc.cam.yres;
  if (pixel_begin < 0 || pixel_end > npix || pixel_begin > pixel_end) { g_err = "bad pixel range"; return 2; }
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int> next{pixel_begin};
  constexpr int CHUNK = 64;
  // Splats land on arbitrary pixels: each thread records (pixel, rgb) and the records are
  // added to light_accum after the threads join.
  struct Splat { int unit; double rgb[3]; };
  std::vector<std::vector<Splat>> splats(nthreads);
  auto body = [&](int tid) {
    Worker w(sc);
    Worker2 w2(sc);
    const bool pt2 = sc.params.algo == TT_ALGO_PT2;
    std::vector<double> scratch;
    for (;;) {
      int p0 = next.fetch_add(CHUNK);
      if (p0 >= pixel_end) break;
      int p1 = std::min(pixel_end, p0 + CHUNK);
      for (int p = p0; p < p1; ++p) {
        for (int sidx = 0; sidx < spp; ++sidx) {
          uint64_t sample = (uint64_t)sample_offset + sidx;
          double rgb[3];
          if (pt2) {
            SeedPath(w2.smp.g, seed, sample * (uint64_t)npix + (uint64_t)p);
            if (!sc.sobol.empty()) {
              // SetPixelIndex / SetPointNum (renderingalgorithms_pathtracing2.cxx:345-352).
              const int px = p % sc.cam.xres, py = p / sc.cam.xres;
              const int r = (px % TT_ROTATION_BLOCK) + (py % TT_ROTATION_BLOCK) * TT_ROTATION_BLOCK;
              w2.smp.qmc = sc.sobol.data();
              w2.smp.point = (uint32_t)sample;
              w2.smp.rot[0] = tt_rotation_offsets[2 * r];
              w2.smp.rot[1] = tt_rotation_offsets[2 * r + 1];
              w2.smp.offset = 0;
              w2.smp.sub = 0;
            }
            w2.RenderPixel(p, rgb);
          } else {
            SeedPath(w.smp.g, seed, sample * (uint64_t)npix + (uint64_t)p);
            w.RenderPixel(p, rgb, &splats[tid]);
          }
          for (int k = 0; k < 3; ++k) accum[3 * (size_t)p + k] += rgb[k];
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads; ++i) th.emplace_back(body, i);
  for (auto& t : th) t.join();
  for (int i = 0; i < nthreads; ++i)
    for (const auto& sp : splats[i])
      for (int k = 0; k < 3; ++k) light_accum[3 * (size_t)sp.unit + k] += sp.rgb[k];
  *splat_count += (uint64_t)spp * (uint64_t)(pixel_end - pixel_begin);
  return 0;
}

static Surf ZUpSurface(V3 wi) {
  Surf si;
  si.prim = 0;
  si.geometry_normal = {0, 0, 1};
  si.smooth_normal = {0, 0, 1};
  const double sign = -Sign(Dot(-wi, si.geometry_normal));
  si.normal = sign * si.geometry_normal;
  si.shading_normal = sign * si.smooth_normal;
  return si;
}

int or_sample_bsdf(or_scene* s, int material, const double* wi, const int32_t* lambda_idx, int n, uint64_t seed,
                   double* out_dir, double* out_value, double* out_pdf) {
  if (material < 0 || material >= (int)s->s.materials.size()) return 2;
  const tt_material& m = s->s.materials[material].m;
  V3 w{wi[0], wi[1], wi[2]};
  Surf si = ZUpSurface(w);
  for (int i = 0; i < n; ++i) {
    Sampler smp;
    SeedPath(smp.g, seed, (uint64_t)i);
    ScatterSample ss = SampleBSDF(m, w, si, smp, lambda_idx);
    out_dir[3 * i] = ss.dir.x; out_dir[3 * i + 1] = ss.dir.y; out_dir[3 * i + 2] = ss.dir.z;
    for (int k = 0; k < 3; ++k) out_value[3 * i + k] = ss.value[k];
    out_pdf[i] = ss.delta ? -ss.pdf : ss.pdf;
  }
  return 0;
}

int or_eval_bsdf(or_scene* s, int material, const double* wi, const int32_t* lambda_idx, const double* dirs, int n,
                 double* out_value, double* out_pdf) {
  if (material < 0 || material >= (int)s->s.materials.size()) return 2;
  const tt_material& m = s->s.materials[material].m;
  V3 w{wi[0], wi[1], wi[2]};
  Surf si = ZUpSurface(w);
  for (int i = 0; i < n; ++i) {
    V3 o{dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
    double pdf = 0;
    S3 val = EvaluateBSDF(m, w, si, o, lambda_idx, &pdf);
    for (int k = 0; k < 3; ++k) out_value[3 * i + k] = val[k];
    out_pdf[i] = pdf;
  }
  return 0;
}

void or_rgb_to_spectrum(const double* rgb, double* out) {
  SmitsCases(rgb[0], rgb[1], rgb[2], [&](double a, int ia, double b, int ib, double c, int ic) {
    LinCombN(out, a, kSmitsBasis[ia], b, kSmitsBasis[ib], c, kSmitsBasis[ic]);
  });
}
void or_spectrum_to_rgb(const double* spec, double* rgb) {
  for (int i = 0; i < 3; ++i) {
    rgb[i] = 0;
    for (int b = 0; b < NBINS; ++b) rgb[i] += spec[b] * kSpectrumToRgb[i][b];
  }
}
void or_selection_to_rgb(const double* val3, const int32_t* idx3, double* rgb) {
  SpectralSelectionToRGB(S3(val3[0], val3[1], val3[2]), idx3, rgb);
}
void or_rgb_to_selection(const double* rgb, const int32_t* idx3, double* val3) {
  S3 r = RGBToSpectralSelection(rgb, idx3);
  for (int k = 0; k < 3; ++k) val3[k] = r[k];
}
void or_reflected(const double* wi, const double* n, double* out) {
  V3 r = Reflected({wi[0], wi[1], wi[2]}, {n[0], n[1], n[2]});
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
int or_refracted(const double* wi, const double* n, double eta, double* out) {
  V3 r;
  if (!Refracted({wi[0], wi[1], wi[2]}, {n[0], n[1], n[2]}, eta, &r)) return 0;
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
  return 1;
}
void or_half_vector(const double* wi, const double* wo, double* out) {
  V3 r = HalfVector({wi[0], wi[1], wi[2]}, {wo[0], wo[1], wo[2]});
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
int or_half_vector_refracted(const double* wi, const double* wo, double eta, double* out) {
  V3 r;
  if (!HalfVectorRefracted({wi[0], wi[1], wi[2]}, {wo[0], wo[1], wo[2]}, eta, &r)) return 0;
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
  return 1;
}
double or_fresnel(double cos_i, double eta) { return FresnelReflectivityWalter(cos_i, eta); }
void or_pcg32_stream(uint64_t initstate, uint64_t initseq, int n, uint32_t* out) {
  Pcg32 g;
  g.Seed(initstate, initseq);
  for (int i = 0; i < n; ++i) out[i] = g.NextUInt();
}
double or_pcg32_nextdouble_first(uint64_t initstate, uint64_t initseq) {
  Pcg32 g;
  g.Seed(initstate, initseq);
  return g.NextDouble();
}
int or_uniform_int_stream(uint64_t initstate, uint64_t initseq, int a, int b, int n, int32_t* out) {
  Sampler s;
  s.g.Seed(initstate, initseq);
  for (int i = 0; i < n; ++i) out[i] = s.UniformInt(a, b);
  return 0;
}
void or_tables(double* smits, double* m, double* sun) {
  std::memcpy(smits, kSmitsBasis, sizeof(kSmitsBasis));
  std::memcpy(m, kSpectrumToRgb, sizeof(kSpectrumToRgb));
  std::memcpy(sun, kSunSpectrum, sizeof(kSunSpectrum));
}
int or_eval_env(or_scene* s, const double* dir_out, const int32_t* lambda_idx, double* value3, double* pdf) {
  V3 d{dir_out[0], dir_out[1], dir_out[2]};
  S3 v = EnvEvaluateTotal(s->s, d, lambda_idx);
  for (int k = 0; k < 3; ++k) value3[k] = v[k];
  *pdf = EnvEvaluatePdfTotal(s->s, d);
  return 0;
}
// Medium-tracker walk along a ray: initializes the tracker at the origin and records the
// current medium (-1 = vacuum) after each volume-boundary crossing (MediaTransmission
// tests, tests3.cxx:70-152).  Returns the number of crossings written.
int or_medium_walk(or_scene* os, const double* org3, const double* dir3, double tfar, int max, int32_t* media,
                   double* ts, int32_t* initial) {
  const Scene& sc = os->s;
  MediumTracker mt;
  V3 o{org3[0], org3[1], org3[2]}, d{dir3[0], dir3[1], dir3[2]};
  InitializeMediumTracker(sc, mt, o);
  *initial = mt.current;
  std::vector<Crossing> hits;
  AllHits(sc, sc.vol, o, d, 0., tfar, hits);
  int n = 0;
  for (const auto& h : hits) {
    if (n >= max) break;
    GoingThroughSurface(sc, mt, d, h.n, h.material);
    media[n] = mt.current;
    ts[n] = h.t;
    ++n;
  }
  return n;
}

// TransmittanceEstimate along a segment starting at org with a tracker initialized there.
int or_transmittance(or_scene* os, const double* org3, const double* dir3, double length, const int32_t* idx,
                     uint64_t seed, double* T3, double* coeff3) {
  Worker w(os->s);
  std::memcpy(w.ctx.idx, idx, 3 * sizeof(int32_t));
  MediumTracker mt;
  V3 o{org3[0], org3[1], org3[2]}, d{dir3[0], dir3[1], dir3[2]};
  InitializeMediumTracker(os->s, mt, o);
  VolCoeffs c;
  Sampler shadow;
  SeedPath(shadow.g, seed, 0u);
  S3 T = w.TransmittanceEstimate(o, d, length, mt, &c, shadow);
  for (int k = 0; k < 3; ++k) T3[k] = T[k];
  coeff3[0] = c.fwd; coeff3[1] = c.bwd; coeff3[2] = c.tr;
  return 0;
}

// n independent TrackToNextInteraction samples from org along dir (stream i = sample i):
// out[11 i ..] = interacted, distance, weight[3], sigma_s[3], coeff fwd, bwd, transmittance.
int or_track(or_scene* os, const double* org3, const double* dir3, const int32_t* idx, int n, uint64_t seed,
             double* out) {
  for (int i = 0; i < n; ++i) {
    Worker w(os->s);
    std::memcpy(w.ctx.idx, idx, 3 * sizeof(int32_t));
    SeedPath(w.smp.g, seed, (uint64_t)i);
    Node src;
    src.type = CAMERA;  // a point source that is not a surface: no offset, no passage
    src.coords = {org3[0], org3[1], org3[2]};
    MediumTracker mt;
    InitializeMediumTracker(os->s, mt, src.coords);
    // Track along the given direction: emulate TakeRandomWalkStep after the direction is
    // chosen by calling the tracking part through a one-off source with a fixed ray.
    V3 d{dir3[0], dir3[1], dir3[2]};
    auto st = w.TrackFrom(src.coords, d, mt);
    double* o = out + 11 * (size_t)i;
    o[0] = st.node.type == VOLUME_SCATTER ? 1. : 0.;
    o[1] = st.seg_len;
    for (int k = 0; k < 3; ++k) { o[2 + k] = st.beta_factor[k]; o[5 + k] = st.node.sigma_s[k]; }
    o[8] = st.coeff.fwd;
    o[9] = st.coeff.bwd;
    o[10] = st.coeff.tr;
  }
  return 0;
}

// n phase-function samples about the reverse incident direction wi (the direction back
// towards the previous vertex) plus the pdf and value of each sampled direction.
int or_phase_sample(int kind, double g, const double* wi3, int n, uint64_t seed, double* dirs, double* pdf,
                    double* value) {
  MediumDesc m{};
  m.phase = kind;
  m.g = g;
  const V3 wi{wi3[0], wi3[1], wi3[2]};
  for (int i = 0; i < n; ++i) {
    Sampler smp;
    SeedPath(smp.g, seed, (uint64_t)i);
    const ScatterSample s = PhaseSample(m, wi, smp);
    dirs[3 * i] = s.dir.x; dirs[3 * i + 1] = s.dir.y; dirs[3 * i + 2] = s.dir.z;
    pdf[i] = s.pdf;
    value[i] = PhaseEvaluate(m, wi, s.dir);
  }
  return 0;
}

// Atmosphere model of medium `medium` (tests): out[0] altitude of pos, out[1..3] lowest
// point of the segment (org, dir, length), out[4..6] sigma_s and out[7..9] sigma_t at pos,
// out[10..12] molecular and out[13..15] aerosol sigma_s at pos, out[16] the segment
// majorant, out[17] the majorant at pos's altitude.
int or_atmosphere_query(or_scene* os, int medium, const double* pos3, const double* org3, const double* dir3,
                        double length, const int32_t* idx, double* out) {
  const Scene& sc = os->s;
  if (medium < 0 || medium >= (int)sc.media.size() || sc.media[medium].kind != TT_MEDIUM_ATMOSPHERE) return 2;
  const MediumDesc& m = sc.media[medium];
  const V3 pos{pos3[0], pos3[1], pos3[2]}, org{org3[0], org3[1], org3[2]}, dir{dir3[0], dir3[1], dir3[2]};
  out[0] = Altitude(m, pos);
  const V3 lp = LowestPoint(m, org, dir, length);
  out[1] = lp.x; out[2] = lp.y; out[3] = lp.z;
  S3 ss, st, c[2];
  AtmCoeffs(m, out[0], idx, &ss, &st);
  AtmSigmaS(m, out[0], idx, c);
  for (int k = 0; k < 3; ++k) {
    out[4 + k] = ss[k];
    out[7 + k] = st[k];
    out[10 + k] = c[0][k];
    out[13 + k] = c[1][k];
  }
  out[16] = AtmSegmentMajorant(m, org, dir, length);
  out[17] = AtmMajorant(m, out[0]);
  return 0;
}

// n phase samples of medium `medium` at a volume vertex at pos (the atmosphere's phase
// function depends on the altitude): directions, values per wavelength and pdfs.
int or_medium_phase_sample(or_scene* os, int medium, const double* pos3, const double* wi3, const int32_t* idx, int n,
                           uint64_t seed, double* dirs, double* value3, double* pdf) {
  const Scene& sc = os->s;
  if (medium < 0 || medium >= (int)sc.media.size()) return 2;
  const V3 pos{pos3[0], pos3[1], pos3[2]}, wi{wi3[0], wi3[1], wi3[2]};
  for (int i = 0; i < n; ++i) {
    Sampler smp;
    SeedPath(smp.g, seed, (uint64_t)i);
    const ScatterSample s = MediumPhaseSample(sc.media[medium], pos, wi, smp, idx);
    dirs[3 * i] = s.dir.x; dirs[3 * i + 1] = s.dir.y; dirs[3 * i + 2] = s.dir.z;
    for (int k = 0; k < 3; ++k) value3[3 * i + k] = s.value[k];
    pdf[i] = s.pdf;
  }
  return 0;
}

int or_scene_info(or_scene* s, double* bbox6, int32_t* counts4) {
  for (int k = 0; k < 3; ++k) { bbox6[k] = s->s.bb_lo[k]; bbox6[3 + k] = s->s.bb_hi[k]; }
  counts4[0] = (int32_t)s->s.tv0.size();
  counts4[1] = (int32_t)s->s.area_lights.size();
  counts4[2] = (int32_t)s->s.env.size();
  counts4[3] = (int32_t)s->s.surf.nodes.size();
  return 0;
}

int or_sobol(int dim, int n, const uint32_t* points, double* out) {
  static std::vector<uint32_t> mats;
  static std::once_flag once;
  std::call_once(once, [] { SobolMatrices(mats); });
  if (dim < 0 || dim >= TT_SOBOL_DIMS) { g_err = "dimension out of range"; return 2; }
  for (int i = 0; i < n; ++i) out[i] = SobolMult(points[i], &mats[32 * (size_t)dim]);
  return 0;
}

void or_sobol_matrix(int s, int a, const uint16_t* m, uint32_t* out32) { SobolMatrix(s, a, m, out32); }

int or_qmc_draws(int px, int py, uint32_t point, int n_ops, const int32_t* ops, uint64_t pcg_seed, double* out) {
  static std::vector<uint32_t> mats;
  static std::once_flag once;
  std::call_once(once, [] { SobolMatrices(mats); });
  Sampler smp;
  SeedPath(smp.g, pcg_seed, 0);
  const int r = (px % TT_ROTATION_BLOCK) + (py % TT_ROTATION_BLOCK) * TT_ROTATION_BLOCK;
  smp.qmc = mats.data();
  smp.point = point;
  smp.rot[0] = tt_rotation_offsets[2 * r];
  smp.rot[1] = tt_rotation_offsets[2 * r + 1];
  int k = 0;
  for (int i = 0; i < n_ops; ++i) {
    if (ops[i] == 0) {
      out[k++] = smp.Uniform01();
    } else if (ops[i] == 1) {
      smp.UniformUnitSquare(out + k);
      k += 2;
    } else {
      if (ops[i] - 2 >= 64) { g_err = "subsequence id out of range"; return 2; }
      smp.SetSubsequenceId((uint32_t)(ops[i] - 2));
    }
  }
  return 0;
}

}  // extern "C"
