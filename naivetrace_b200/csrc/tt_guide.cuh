// Learned path guiding: a small MLP maps an encoded surface point (position, normal,
// outgoing direction) to an 8-lobe von Mises-Fisher mixture and to the probability of
// sampling that mixture instead of the BSDF.  It stands in for the reference's guided path
// tracer (renderingalgorithms_pathtracing_guided.cxx), whose per-cell vMF mixtures are
// fitted from radiance records (path_guiding.cxx); the mixture is combined with the BSDF
// by the one-sample MIS of SampleWithBinaryMixtureDensity / EvaluateWithBinaryMixtureDensity
// (renderingalgorithms_pathtracing_guided.cxx:474-544).  vMF density and sampling follow
// distribution_mixture_models.cxx:93-152.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tt_device.cuh"

namespace tt {

// Network shape: 82 input features padded to 96, four hidden layers of 64, 41 outputs
// (8 lobes x (weight logit, mean xyz, concentration) + 1 MIS logit) padded to 48.
constexpr int kGIn = 96;
constexpr int kGHid = 64;
constexpr int kGOut = 48;
constexpr int kGLobes = 8;
constexpr int kGFreq = 12;
constexpr int kGLayers = 5;  // weight matrices
// Parameter offsets in the flat FP32 / BF16 parameter arrays.  Layer l has weights W_l
// (stored [out][in], input index contiguous) and bias b_l.
__host__ __device__ constexpr int guide_in(int l) { return l == 0 ? kGIn : kGHid; }
__host__ __device__ constexpr int guide_out(int l) { return l == kGLayers - 1 ? kGOut : kGHid; }
__host__ __device__ constexpr int guide_w_offset(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += guide_in(i) * guide_out(i) + guide_out(i);
  return o;
}
__host__ __device__ constexpr int guide_b_offset(int l) { return guide_w_offset(l) + guide_in(l) * guide_out(l); }
constexpr int kGParams = guide_w_offset(kGLayers);

// Output maps.  Smooth, so that no output sits in a dead zone without gradient:
//   c       = 0.05 + 0.9 sigmoid(o)                 probability of sampling the mixture
//   log k   = M + H tanh((o - M) / H)               kappa in (0.05, 40), slope 1 at o = M
// The upper limit 40 is the reference's concentration limit (distribution_mixture_models.hxx:12-14).
constexpr float kGGuideProbMin = 0.05f;
constexpr float kGGuideProbSpan = 0.9f;
constexpr float kGLogKappaMid = 0.34657359f;   // (log 0.05 + log 40) / 2
constexpr float kGLogKappaHalf = 3.34236985f;  // (log 40 - log 0.05) / 2

// Frequency multiplier of band j: 2^(j/8) (eighth octaves, 1 .. 2^1.375).  A smooth
// encoding (finest period about 0.8 of the scene box; the ReLU layers add the sharper
// features) generalised best from the few records that carry light: with octave-spaced
// bands the network fitted single records and lost to plain BSDF sampling on held-out data.
__host__ __device__ __forceinline__ float guide_freq(int j) {
  const int q = j & 7;
  const float f = q == 0 ? 1.f
                  : q == 1 ? 1.09050773f
                  : q == 2 ? 1.18920712f
                  : q == 3 ? 1.29683955f
                  : q == 4 ? 1.41421356f
                  : q == 5 ? 1.54221083f
                  : q == 6 ? 1.68179283f
                           : 1.83400809f;
  return f * (float)(1 << (j >> 3));
}

// Input features of a surface point (guide_feature_pair builds them): sin and cos of
// pi 2^(j/8) x for the 12 bands j of each coordinate x of the position normalised to the
// scene box (72), the normalised position (3), the shading normal (3), the outgoing
// direction (3) and a constant 1 (82), zero padded to 96.

// Decoded mixture of one query.
struct GuideMixture {
  float w[kGLobes];      // weights (softmax)
  float3 mu[kGLobes];    // unit means
  float kappa[kGLobes];  // concentrations
  float c;               // probability of sampling the mixture (vs. the BSDF)
};

__device__ __forceinline__ GuideMixture guide_decode(const float* o) {
  GuideMixture m;
  float mx = -INFINITY;
#pragma unroll
  for (int k = 0; k < kGLobes; ++k) mx = fmaxf(mx, o[5 * k]);
  float sum = 0.f;
#pragma unroll
  for (int k = 0; k < kGLobes; ++k) {
    m.w[k] = __expf(o[5 * k] - mx);
    sum += m.w[k];
  }
#pragma unroll
  for (int k = 0; k < kGLobes; ++k) {
    m.w[k] /= sum;
    float3 v = f3(o[5 * k + 1], o[5 * k + 2], o[5 * k + 3]);
    const float l = len3(v);
    m.mu[k] = l > 1e-12f ? v * (1.f / l) : f3(0.f, 0.f, 1.f);
    m.kappa[k] = __expf(kGLogKappaMid + kGLogKappaHalf * tanhf((o[5 * k + 4] - kGLogKappaMid) / kGLogKappaHalf));
  }
  m.c = kGGuideProbMin + kGGuideProbSpan / (1.f + __expf(-o[5 * kGLobes]));
  return m;
}

// vMF density k / (2 pi (1 - exp(-2k))) exp(k (mu.x - 1)).
__device__ __forceinline__ float vmf_pdf(float3 mu, float k, float3 x) {
  return k / (2.f * kPi * (1.f - __expf(-2.f * k))) * __expf(k * (dot3(mu, x) - 1.f));
}

__device__ __forceinline__ float guide_mixture_pdf(const GuideMixture& m, float3 x) {
  float p = 0.f;
#pragma unroll
  for (int k = 0; k < kGLobes; ++k) p += m.w[k] * vmf_pdf(m.mu[k], m.kappa[k], x);
  return p;
}

// Lobe by tower sampling of the weights, then w = 1 + log(r2 + (1 - r2) exp(-2k)) / k about
// the lobe's mean.
__device__ __forceinline__ float3 guide_mixture_sample(const GuideMixture& m, Rng& rng) {
  float r = rng.uniform();
  float3 mu = m.mu[kGLobes - 1];
  float kp = m.kappa[kGLobes - 1];
  bool found = false;
#pragma unroll
  for (int k = 0; k < kGLobes - 1; ++k) {
    if (!found && r < m.w[k]) {
      mu = m.mu[k];
      kp = m.kappa[k];
      found = true;
    }
    r -= m.w[k];
  }
  float rr[2];
  rng.square(rr);
  const float w = 1.f + __logf(rr[1] + (1.f - rr[1]) * __expf(-2.f * kp)) / kp;
  const float rho = sqrtf(fmaxf(0.f, 1.f - w * w));
  float sn, cs;
  sincosf(2.f * kPi * rr[0], &sn, &cs);
  const Frame fr = frame_z(mu);
  return normalize3(fr.to_world(f3(rho * cs, rho * sn, w)));
}

// ---- Fused MLP on warp-level tensor-core MMA -------------------------------------------
// One warp runs the five layers for a tile of 16 rows with mma.sync m16n8k16 (BF16 inputs,
// FP32 accumulation).  The weights sit in shared memory with rows padded by 8 BF16 (the
// fragment loads of the 8 row groups then fall into distinct banks); activations stay in
// registers from layer to layer: the accumulator fragment of two adjacent 8-column tiles is,
// after bias, ReLU and rounding to BF16, exactly the A fragment of the next layer's 16-wide
// K chunk.  Fragment layouts (PTX ISA, mma.m16n8k16): lane = 4 g + t; A holds rows (g, g+8)
// x columns (2t, 2t+1, 2t+8, 2t+9) of its 16 x 16 chunk, B columns n = g with rows
// (2t, 2t+1, 2t+8, 2t+9), C rows (g, g+8) x columns (2t, 2t+1).
constexpr int kGPad = 8;
__host__ __device__ constexpr int guide_sm_stride(int l) { return guide_in(l) + kGPad; }
__host__ __device__ constexpr int guide_sm_w(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += guide_out(i) * guide_sm_stride(i);
  return o;
}
__host__ __device__ constexpr int guide_sm_b(int l) { return l * kGHid; }
constexpr int kGSmW = guide_sm_w(kGLayers);                   // BF16 weight elements
constexpr int kGSmB = (kGLayers - 1) * kGHid + kGOut;         // FP32 biases
constexpr int kGSmBytes = kGSmW * 2 + kGSmB * 4;              // 49088
constexpr int kGInputs = 9;                                   // p01 xyz, normal xyz, wo xyz
constexpr int kGOutStride = kGOut + 4;                        // FP32 output row in shared memory
static_assert(kGSmBytes % 16 == 0, "shared-memory regions after the weights stay 16-byte aligned");

__device__ __forceinline__ void mma_bf16_16816(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// Copies the BF16 weights (flat layout of guide_w_offset) and the FP32 biases into shared
// memory (16-byte copies; every layer's weights start on a 16-byte boundary).
__device__ __forceinline__ void guide_smem_load(const __nv_bfloat16* __restrict__ w16, const float* __restrict__ w32,
                                                __nv_bfloat16* sw, float* sb) {
#pragma unroll 1
  for (int l = 0; l < kGLayers; ++l) {
    const int cpr = guide_in(l) / 8;
    const uint4* src = reinterpret_cast<const uint4*>(w16 + guide_w_offset(l));
    for (int e = threadIdx.x; e < guide_out(l) * cpr; e += blockDim.x) {
      const int r = e / cpr, c = e - r * cpr;
      *reinterpret_cast<uint4*>(sw + guide_sm_w(l) + r * guide_sm_stride(l) + c * 8) = __ldg(src + e);
    }
    for (int e = threadIdx.x; e < guide_out(l); e += blockDim.x) sb[guide_sm_b(l) + e] = __ldg(w32 + guide_b_offset(l) + e);
  }
}

// Packed BF16 pair of input features (col, col + 1), col even, of a point with inputs
// q = (p01 xyz, normal xyz, wo xyz).  The arguments stay within |x| <= 2.6 pi, where the
// hardware sine and cosine (__sincosf) are accurate to about 1e-6, below the BF16 step.
__device__ __forceinline__ uint32_t guide_feature_pair(const float* q, int col) {
  float x = 0.f, y = 0.f;
  if (col < 6 * kGFreq) {
    const int a = col / (2 * kGFreq), j = (col - a * 2 * kGFreq) >> 1;
    __sincosf((kPi * q[a]) * guide_freq(j), &x, &y);
  } else if (col < 6 * kGFreq + 10) {
    const int i = col - 6 * kGFreq;
    x = q[i];
    y = i + 1 < kGInputs ? q[i + 1] : 1.f;
  }
  return pack_bf16x2(x, y);
}

// Optional global copies of a tile's activations (training keeps them for the backward
// pass).  Row r of the tile is row `row0 + r` of each array.
struct GuideTileStore {
  __nv_bfloat16* x;      // kGIn per row
  __nv_bfloat16* h[4];   // kGHid per row
  int row0, rows;        // rows past `rows` are not stored
};

// Stores A-fragment rows (g, g + 8) of a 16-row tile: NK chunks of 16 columns.
template <int NK>
__device__ __forceinline__ void guide_store_frags(__nv_bfloat16* base, int ld, const uint32_t (&f)[NK][4], int row0,
                                                  int rows) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int ra = row0 + g, rb = ra + 8;
#pragma unroll
  for (int kc = 0; kc < NK; ++kc) {
    const int c = kc * 16 + 2 * t;
    if (g < rows) {
      *reinterpret_cast<uint32_t*>(base + (size_t)ra * ld + c) = f[kc][0];
      *reinterpret_cast<uint32_t*>(base + (size_t)ra * ld + c + 8) = f[kc][2];
    }
    if (g + 8 < rows) {
      *reinterpret_cast<uint32_t*>(base + (size_t)rb * ld + c) = f[kc][1];
      *reinterpret_cast<uint32_t*>(base + (size_t)rb * ld + c + 8) = f[kc][3];
    }
  }
}

// Bias, ReLU and rounding of a 64-wide accumulator into the next layer's A fragments.
__device__ __forceinline__ void guide_relu_frags(const float (&acc)[8][4], const float* bias, uint32_t (&hf)[4][4]) {
  const int t = threadIdx.x & 3;
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    const float* b = bias + kc * 16 + 2 * t;
    hf[kc][0] = pack_bf16x2(fmaxf(acc[2 * kc][0] + b[0], 0.f), fmaxf(acc[2 * kc][1] + b[1], 0.f));
    hf[kc][1] = pack_bf16x2(fmaxf(acc[2 * kc][2] + b[0], 0.f), fmaxf(acc[2 * kc][3] + b[1], 0.f));
    hf[kc][2] = pack_bf16x2(fmaxf(acc[2 * kc + 1][0] + b[8], 0.f), fmaxf(acc[2 * kc + 1][1] + b[9], 0.f));
    hf[kc][3] = pack_bf16x2(fmaxf(acc[2 * kc + 1][2] + b[8], 0.f), fmaxf(acc[2 * kc + 1][3] + b[9], 0.f));
  }
}

// Five layers for the 16-row tile whose input fragments are `xf` (6 K chunks); FP32
// outputs with bias to out[r * ldo + col] for the tile's rows r (all 16 rows written).
__device__ __forceinline__ void guide_mlp_tile(const __nv_bfloat16* sw, const float* sb, const uint32_t (&xf)[6][4],
                                               float* out, int ldo, const GuideTileStore* st) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t hf[4][4];
  {
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const __nv_bfloat16* w = sw + guide_sm_w(0) + g * guide_sm_stride(0) + 2 * t;
#pragma unroll
    for (int kc = 0; kc < 6; ++kc)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const __nv_bfloat16* wr = w + j * 8 * guide_sm_stride(0) + kc * 16;
        mma_bf16_16816(acc[j], xf[kc], ld_u32(wr), ld_u32(wr + 8));
      }
    guide_relu_frags(acc, sb + guide_sm_b(0), hf);
  }
  if (st) guide_store_frags<6>(st->x, kGIn, xf, st->row0, st->rows);
#pragma unroll 1
  for (int l = 1; l < kGLayers - 1; ++l) {
    if (st) guide_store_frags<4>(st->h[l - 1], kGHid, hf, st->row0, st->rows);
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const __nv_bfloat16* w = sw + guide_sm_w(l) + g * guide_sm_stride(l) + 2 * t;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const __nv_bfloat16* wr = w + j * 8 * guide_sm_stride(l) + kc * 16;
        mma_bf16_16816(acc[j], hf[kc], ld_u32(wr), ld_u32(wr + 8));
      }
    guide_relu_frags(acc, sb + guide_sm_b(l), hf);
  }
  if (st) guide_store_frags<4>(st->h[kGLayers - 2], kGHid, hf, st->row0, st->rows);
  {
    constexpr int L = kGLayers - 1;
    float acc[6][4];
#pragma unroll
    for (int j = 0; j < 6; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const __nv_bfloat16* w = sw + guide_sm_w(L) + g * guide_sm_stride(L) + 2 * t;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const __nv_bfloat16* wr = w + j * 8 * guide_sm_stride(L) + kc * 16;
        mma_bf16_16816(acc[j], hf[kc], ld_u32(wr), ld_u32(wr + 8));
      }
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const int c = j * 8 + 2 * t;
      const float b0 = sb[guide_sm_b(L) + c], b1 = sb[guide_sm_b(L) + c + 1];
      *reinterpret_cast<float2*>(out + g * ldo + c) = make_float2(acc[j][0] + b0, acc[j][1] + b1);
      *reinterpret_cast<float2*>(out + (g + 8) * ldo + c) = make_float2(acc[j][2] + b0, acc[j][3] + b1);
    }
  }
}

// Input fragments of a 16-row tile from per-row inputs q (kGInputs floats, stride qs).
__device__ __forceinline__ void guide_tile_features(const float* q, int qs, uint32_t (&xf)[6][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const float* qa = q + g * qs;
  const float* qb = q + (g + 8) * qs;
#pragma unroll
  for (int kc = 0; kc < 6; ++kc) {
    const int c0 = kc * 16 + 2 * t;
    xf[kc][0] = guide_feature_pair(qa, c0);
    xf[kc][1] = guide_feature_pair(qb, c0);
    xf[kc][2] = guide_feature_pair(qa, c0 + 8);
    xf[kc][3] = guide_feature_pair(qb, c0 + 8);
  }
}

// Input fragments of a 16-row tile from BF16 feature rows x (kGIn per row); rows past
// `rows` read zeros.
__device__ __forceinline__ void guide_tile_load_x(const __nv_bfloat16* x, int rows, uint32_t (&xf)[6][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int kc = 0; kc < 6; ++kc) {
    const int c0 = kc * 16 + 2 * t;
    xf[kc][0] = g < rows ? ld_u32(x + (size_t)g * kGIn + c0) : 0u;
    xf[kc][1] = g + 8 < rows ? ld_u32(x + (size_t)(g + 8) * kGIn + c0) : 0u;
    xf[kc][2] = g < rows ? ld_u32(x + (size_t)g * kGIn + c0 + 8) : 0u;
    xf[kc][3] = g + 8 < rows ? ld_u32(x + (size_t)(g + 8) * kGIn + c0 + 8) : 0u;
  }
}

}  // namespace tt
