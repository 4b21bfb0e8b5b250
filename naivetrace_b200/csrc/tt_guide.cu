// Training and batch evaluation of the guiding network on the GPU.  Training follows the
// KL-divergence objective of neural importance sampling (Mueller et al. 2019): for a record
// sampled with density q at direction wi with target value F, minimise -(F / q) log p(wi)
// with p = (1 - c) p_bsdf + c p_vmf, which also learns the selection probability c.
//
// One training step is two launches with the default (tcgen05) network kernels:
//   k_step_tc      persistent over tiles of 128 records: features, the five layers, the loss
//                  gradient per record, the backward pass and the weight and bias gradients,
//                  the tile's activations in shared memory and the CTA's weight gradients in
//                  tensor memory, written once per CTA as a partial sum;
//   k_reduce_adam  sum of the CTAs' partials with the Adam step fused in (k_reduce and k_adam
//                  separately when the gradient alone is asked for).
// With the warp-level mma.sync kernels it is three:
//   k_train   persistent; per warp 16 records: features in registers, the five layers
//             (activations kept in global memory for the weight gradients), the loss gradient
//             per record, and the backward pass through the layers on the same tensor-core
//             tiles (B fragments of W^T by ldmatrix.trans from the forward weight image),
//             storing each layer's output gradient;
//   k_wgrad   dW_l = sum over records of dH_l^T X_l and the bias sums, split over chunks of
//             128 records (ldmatrix.trans fragments of both operands);
//   k_reduce_adam  as above.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "tt_guide.cuh"
#include "tt_guide.h"
#include "tt_guide_tc.cuh"
#include "tt_internal.h"

namespace tt {
namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ void ldsm_x4_trans(uint32_t (&r)[4], const void* row) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(row));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ float lo_bf16(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float hi_bf16(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// Loss -(F/q) log p(wi), p = (1 - c) p_bsdf + c p_vmf, of one record with network outputs o,
// and its gradient with respect to the 41 outputs into d[0..47] (padded columns zero).
__device__ float guide_loss_row(const GuideRecord& r, const float* o, float* d) {
  const float w = r.f_over_q;
  const float3 x = f3(r.wi[0], r.wi[1], r.wi[2]);
  float mx = -INFINITY;
  for (int k = 0; k < kGLobes; ++k) mx = fmaxf(mx, o[5 * k]);
  float pi_[kGLobes], sum = 0.f;
  for (int k = 0; k < kGLobes; ++k) {
    pi_[k] = expf(o[5 * k] - mx);
    sum += pi_[k];
  }
  float v[kGLobes], pv = 0.f, mlen[kGLobes], kap[kGLobes], kslope[kGLobes];
  float3 mu[kGLobes];
  for (int k = 0; k < kGLobes; ++k) {
    pi_[k] /= sum;
    const float3 m = f3(o[5 * k + 1], o[5 * k + 2], o[5 * k + 3]);
    mlen[k] = len3(m);
    mu[k] = mlen[k] > 1e-12f ? m * (1.f / mlen[k]) : f3(0.f, 0.f, 1.f);
    const float th = tanhf((o[5 * k + 4] - kGLogKappaMid) / kGLogKappaHalf);
    kslope[k] = 1.f - th * th;  // d log kappa / d output
    kap[k] = expf(kGLogKappaMid + kGLogKappaHalf * th);
    v[k] = kap[k] / (2.f * kPi * (1.f - expf(-2.f * kap[k]))) * expf(kap[k] * (dot3(mu[k], x) - 1.f));
    pv += pi_[k] * v[k];
  }
  const float sg = 1.f / (1.f + expf(-o[5 * kGLobes]));
  const float c = kGGuideProbMin + kGGuideProbSpan * sg;
  const float pp = fmaxf((1.f - c) * r.p_bsdf + c * pv, 1e-20f);
  const float loss = w > 0.f ? -w * logf(pp) : 0.f;
  const float dLdp = w > 0.f ? -w / pp : 0.f;
  const float dLdpv = dLdp * c;
  for (int k = 0; k < kGLobes; ++k) {
    // Softmax: d pv / d a_k = pi_k (v_k - pv).
    d[5 * k] = dLdpv * pi_[k] * (v[k] - pv);
    // d v_k / d mu_k = v_k kappa_k x, projected through the normalisation of m.
    const float s = dLdpv * pi_[k] * v[k] * kap[k];
    float3 dm = f3(0.f, 0.f, 0.f);
    if (mlen[k] > 1e-12f) {
      const float3 gx = x * s;
      dm = (gx - mu[k] * dot3(mu[k], gx)) * (1.f / mlen[k]);
    }
    d[5 * k + 1] = dm.x;
    d[5 * k + 2] = dm.y;
    d[5 * k + 3] = dm.z;
    // d log v_k / d kappa = 1/kappa - 2 exp(-2 kappa) / (1 - exp(-2 kappa)) + (mu.x - 1),
    // times d kappa / d output = kappa kslope.
    const float e2 = expf(-2.f * kap[k]);
    const float dlogv = 1.f / kap[k] - 2.f * e2 / (1.f - e2) + (dot3(mu[k], x) - 1.f);
    d[5 * k + 4] = dLdpv * pi_[k] * v[k] * dlogv * kap[k] * kslope[k];
  }
  d[5 * kGLobes] = dLdp * (pv - r.p_bsdf) * kGGuideProbSpan * sg * (1.f - sg);
  for (int k = 5 * kGLobes + 1; k < kGOut; ++k) d[k] = 0.f;
  return loss;
}

struct TrainBufs {
  bf16* x;       // features (kGIn per record)
  bf16* h[4];    // hidden activations (kGHid)
  bf16* dh[4];   // gradients of the hidden layers' pre-activations (kGHid)
  bf16* dy;      // gradient of the outputs (kGOut)
  float* loss;   // mean loss
};

// Backward pass of one 16-row tile: dY (shared memory, 16 x kGOut BF16, row stride dys)
// through layers 4..1: dH_{l-1} = (dH_l W_l) masked by H_{l-1} > 0, rounded to BF16,
// stored for the weight gradients.
__device__ __forceinline__ void guide_bwd_tile(const bf16* sw, const bf16* dyt, int dys, const TrainBufs& b,
                                               int row0, int rows) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t af[4][4];
#pragma unroll
  for (int kc = 0; kc < 3; ++kc) {
    const int c = kc * 16 + 2 * t;
    af[kc][0] = ld_u32(dyt + g * dys + c);
    af[kc][1] = ld_u32(dyt + (g + 8) * dys + c);
    af[kc][2] = ld_u32(dyt + g * dys + c + 8);
    af[kc][3] = ld_u32(dyt + (g + 8) * dys + c + 8);
  }
  af[3][0] = af[3][1] = af[3][2] = af[3][3] = 0u;
  // ldmatrix lane roles: matrix mi = lane / 8 gets its row (lane % 8) address from this lane.
  const int mi = lane >> 3, mr = lane & 7;
#pragma unroll 1
  for (int l = kGLayers - 1; l >= 1; --l) {
    const int nk = l == kGLayers - 1 ? 3 : 4;  // K chunks over this layer's outputs
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const bf16* w = sw + guide_sm_w(l);
    const int ws = guide_sm_stride(l);
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      if (kc >= nk) break;
#pragma unroll
      for (int jp = 0; jp < 4; ++jp) {
        // Blocks of W (rows k = outputs, columns n = inputs): (k 0-7, n 0-7), (k 8-15, n 0-7),
        // (k 0-7, n 8-15), (k 8-15, n 8-15): b0, b1 of n-tile 2jp, then of 2jp + 1.
        uint32_t bf[4];
        ldsm_x4_trans(bf, w + (kc * 16 + (mi & 1) * 8 + mr) * ws + jp * 16 + (mi >> 1) * 8);
        mma_bf16_16816(acc[2 * jp], af[kc], bf[0], bf[1]);
        mma_bf16_16816(acc[2 * jp + 1], af[kc], bf[2], bf[3]);
      }
    }
    // Mask by the ReLU of H_{l-1}, read in the A-fragment layout that matches the
    // accumulator of the two 8-column tiles 2kc and 2kc + 1.
    const bf16* hp = b.h[l - 1];
    const int ra = row0 + g, rb = ra + 8;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      const int c = kc * 16 + 2 * t;
      const uint32_t h0 = g < rows ? ld_u32(hp + (size_t)ra * kGHid + c) : 0u;
      const uint32_t h1 = g + 8 < rows ? ld_u32(hp + (size_t)rb * kGHid + c) : 0u;
      const uint32_t h2 = g < rows ? ld_u32(hp + (size_t)ra * kGHid + c + 8) : 0u;
      const uint32_t h3 = g + 8 < rows ? ld_u32(hp + (size_t)rb * kGHid + c + 8) : 0u;
      af[kc][0] = pack_bf16x2(lo_bf16(h0) > 0.f ? acc[2 * kc][0] : 0.f, hi_bf16(h0) > 0.f ? acc[2 * kc][1] : 0.f);
      af[kc][1] = pack_bf16x2(lo_bf16(h1) > 0.f ? acc[2 * kc][2] : 0.f, hi_bf16(h1) > 0.f ? acc[2 * kc][3] : 0.f);
      af[kc][2] = pack_bf16x2(lo_bf16(h2) > 0.f ? acc[2 * kc + 1][0] : 0.f, hi_bf16(h2) > 0.f ? acc[2 * kc + 1][1] : 0.f);
      af[kc][3] = pack_bf16x2(lo_bf16(h3) > 0.f ? acc[2 * kc + 1][2] : 0.f, hi_bf16(h3) > 0.f ? acc[2 * kc + 1][3] : 0.f);
    }
    guide_store_frags<4>(b.dh[l - 1], kGHid, af, row0, rows);
  }
}

constexpr int kTrainWarps = 4;
constexpr int kTrainRows = 16;        // records per warp iteration (one tile)
constexpr int kDyStride = kGOut + 8;  // BF16 output-gradient row in shared memory
constexpr int kTrainWarpBytes = kTrainRows * (kGInputs * 4 + kGOutStride * 4 + kDyStride * 2);
constexpr int kTrainSmem = kGSmBytes + kTrainWarps * kTrainWarpBytes;
static_assert(kTrainWarpBytes % 16 == 0, "per-warp regions stay 16-byte aligned");

// Record i of the batch is rec[i], or with pool_n > 0 the i-th record of a mini-batch drawn
// uniformly with replacement from the pool, rec[h(seed, i) mod pool_n] with h the SplitMix64
// finalizer, read straight from the pool.
__global__ void __launch_bounds__(kTrainWarps * 32) k_train(const GuideRecord* __restrict__ rec, int n,
                                                            const bf16* __restrict__ w16,
                                                            const float* __restrict__ w32, TrainBufs b, int pool_n,
                                                            unsigned long long seed) {
  extern __shared__ __align__(16) unsigned char tsm[];
  bf16* sw = reinterpret_cast<bf16*>(tsm);
  float* sb = reinterpret_cast<float*>(tsm + kGSmW * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* wsm = tsm + kGSmBytes + warp * kTrainWarpBytes;
  float* q = reinterpret_cast<float*>(wsm);
  float* o = q + kTrainRows * kGInputs;
  bf16* dys = reinterpret_cast<bf16*>(o + kTrainRows * kGOutStride);
  if (blockIdx.x * kTrainWarps * kTrainRows >= n) return;
  guide_smem_load(w16, w32, sw, sb);
  __syncthreads();
  const float inv_n = 1.f / (float)n;
  float lsum = 0.f;
  for (int base = (blockIdx.x * kTrainWarps + warp) * kTrainRows; base < n;
       base += gridDim.x * kTrainWarps * kTrainRows) {
    const int i = base + lane;
    const bool mine = lane < kTrainRows && i < n;  // lanes 0..15 own the tile's records
    GuideRecord r{};
    if (mine) {
      const int src =
          pool_n > 0 ? (int)(Rng::splitmix64(seed ^ Rng::splitmix64((unsigned long long)i)) % (unsigned long long)pool_n)
                     : i;
      r = rec[src];
    }
    if (lane < kTrainRows) {
      float* qr = q + lane * kGInputs;
      qr[0] = r.pos[0]; qr[1] = r.pos[1]; qr[2] = r.pos[2];
      qr[3] = r.n[0]; qr[4] = r.n[1]; qr[5] = r.n[2];
      qr[6] = r.wo[0]; qr[7] = r.wo[1]; qr[8] = r.wo[2];
    }
    __syncwarp();
    {
      GuideTileStore st{b.x, {b.h[0], b.h[1], b.h[2], b.h[3]}, base, n - base};
      uint32_t xf[6][4];
      guide_tile_features(q, kGInputs, xf);
      guide_mlp_tile(sw, sb, xf, o, kGOutStride, &st);
    }
    __syncwarp();
    // Loss and output gradient of record `lane`, divided by n and rounded to BF16.
    if (lane < kTrainRows) {
      float d[kGOut];
      if (mine) {
        lsum += guide_loss_row(r, o + lane * kGOutStride, d);
      } else {
#pragma unroll
        for (int k = 0; k < kGOut; ++k) d[k] = 0.f;
      }
      uint32_t pk[kGOut / 2];
#pragma unroll
      for (int k = 0; k < kGOut / 2; ++k) pk[k] = pack_bf16x2(d[2 * k] * inv_n, d[2 * k + 1] * inv_n);
      uint4* srow = reinterpret_cast<uint4*>(dys + lane * kDyStride);
#pragma unroll
      for (int k = 0; k < kGOut / 8; ++k) srow[k] = make_uint4(pk[4 * k], pk[4 * k + 1], pk[4 * k + 2], pk[4 * k + 3]);
      if (mine) {
        uint4* grow = reinterpret_cast<uint4*>(b.dy + (size_t)i * kGOut);
#pragma unroll
        for (int k = 0; k < kGOut / 8; ++k) grow[k] = srow[k];
      }
    }
    __syncwarp();
    guide_bwd_tile(sw, dys, kDyStride, b, base, n - base);
    __syncwarp();
  }
  for (int s = 16; s > 0; s >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, s);
  if (lane == 0 && lsum != 0.f) atomicAdd(b.loss, lsum * inv_n);
}

// Weight and bias gradients of layer blockIdx.y over records [blockIdx.x * kWgChunk, +kWgChunk):
// dW[o][i] = sum_r G[r][o] X[r][i] (G = the layer's output gradient, X its input) as an
// M = outputs, N = inputs, K = records product; both operands are staged record-major in
// shared memory and read transposed by ldmatrix.trans.  Partials go to
// partial[blockIdx.x][guide_w_offset / guide_b_offset].
constexpr int kWgRows = 32;
constexpr int kWgChunk = 128;
constexpr int kWgGs = kGHid + 8;
constexpr int kWgXs = kGIn + 8;

__global__ void __launch_bounds__(128) k_wgrad(int n, TrainBufs b, float* __restrict__ partial) {
  __shared__ __align__(16) bf16 Gs[kWgRows * kWgGs];
  __shared__ __align__(16) bf16 Xs[kWgRows * kWgXs];
  const int l = blockIdx.y;
  const int out = guide_out(l), in = guide_in(l);
  const bf16* G = l == kGLayers - 1 ? b.dy : b.dh[l];
  const bf16* X = l == 0 ? b.x : b.h[l - 1];
  const int r0 = blockIdx.x * kWgChunk, r1 = min(n, r0 + kWgChunk);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int mi = lane >> 3, mr = lane & 7;
  const bool active = warp * 16 < out;
  float acc[12][4];
#pragma unroll
  for (int j = 0; j < 12; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  float bsum = 0.f;
  const int gch = out / 8, xch = in / 8;  // 16-byte chunks per row
  for (int rr = r0; rr < r1; rr += kWgRows) {
    for (int e = tid; e < kWgRows * gch; e += blockDim.x) {
      const int r = e / gch, c = e - r * gch;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (rr + r < r1) v = *reinterpret_cast<const uint4*>(G + (size_t)(rr + r) * out + c * 8);
      *reinterpret_cast<uint4*>(Gs + r * kWgGs + c * 8) = v;
    }
    for (int e = tid; e < kWgRows * xch; e += blockDim.x) {
      const int r = e / xch, c = e - r * xch;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (rr + r < r1) v = *reinterpret_cast<const uint4*>(X + (size_t)(rr + r) * in + c * 8);
      *reinterpret_cast<uint4*>(Xs + r * kWgXs + c * 8) = v;
    }
    __syncthreads();
    if (tid < out)
      for (int r = 0; r < kWgRows; ++r) bsum += __bfloat162float(Gs[r * kWgGs + tid]);
    if (active) {
#pragma unroll
      for (int ks = 0; ks < kWgRows; ks += 16) {
        // A(m = output, k = record) from Gs[record][output]: blocks (m 0-7, k 0-7),
        // (m 8-15, k 0-7), (m 0-7, k 8-15), (m 8-15, k 8-15).
        uint32_t a[4];
        ldsm_x4_trans(a, Gs + (ks + (mi >> 1) * 8 + mr) * kWgGs + warp * 16 + (mi & 1) * 8);
#pragma unroll
        for (int jp = 0; jp < 6; ++jp) {
          if (jp * 16 >= in) break;
          // B(k = record, n = input) from Xs[record][input]: blocks (k 0-7, n 0-7),
          // (k 8-15, n 0-7), (k 0-7, n 8-15), (k 8-15, n 8-15).
          uint32_t bb[4];
          ldsm_x4_trans(bb, Xs + (ks + (mi & 1) * 8 + mr) * kWgXs + jp * 16 + (mi >> 1) * 8);
          mma_bf16_16816(acc[2 * jp], a, bb[0], bb[1]);
          mma_bf16_16816(acc[2 * jp + 1], a, bb[2], bb[3]);
        }
      }
    }
    __syncthreads();
  }
  float* pw = partial + (size_t)blockIdx.x * kGParams;
  if (active) {
    const int m = warp * 16 + g;
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      if (j * 8 >= in) break;
      const int c = j * 8 + 2 * t;
      pw[guide_w_offset(l) + m * in + c] = acc[j][0];
      pw[guide_w_offset(l) + m * in + c + 1] = acc[j][1];
      pw[guide_w_offset(l) + (m + 8) * in + c] = acc[j][2];
      pw[guide_w_offset(l) + (m + 8) * in + c + 1] = acc[j][3];
    }
  }
  if (tid < out) pw[guide_b_offset(l) + tid] = bsum;
}

// The gradient of a training step in one kernel on the tcgen05 tensor cores.  A CTA of 128
// threads (four warps) walks the mini-batch in tiles of 128 records, thread t owning record
// t of the tile, and keeps the whole tile on chip: the features and the four hidden
// activations in shared memory, the ReLU masks in registers, the per-layer accumulator and
// the CTA's weight gradients of all five layers in tensor memory (64 + 304 of 512 columns).
// Every GEMM has M = 128 and BF16 operands in the core-matrix layout of tt_guide_tc.cuh:
//   forward   H_l = ReLU(H_{l-1} W_l^T + b_l): A = the input tile (K-major over features),
//             B = W_l as stored ([out][in], K-major);
//   backward  dH_{l-1} = (dH_l W_l) masked by H_{l-1} > 0: A = the gradient tile (K-major
//             over the layer's outputs), B = W_l^T (a transposed copy made when the CTA
//             loads the weights);
//   weights   dW_l += H_{l-1}^T dH_l over the tile's 128 records, D[m = input][n = output]:
//             A = the input tile read MN-major (the same bytes: 8 consecutive features of a
//             record form a 16-byte core-matrix row, 8 records its 8 rows), B = the gradient
//             tile read MN-major.  The hidden tiles carry a column of ones after the 64
//             activations, so row 64 of D is the bias gradient; layer 0's inputs hold the
//             network's constant feature (column kGOneFeature), whose row is its bias gradient.
//             Rows of D past a layer's inputs (M = 128 reads on into the next core-matrix
//             rows of the tile) are not used.
// The loss and its output gradient per record are guide_loss_row's, rounded to BF16 after the
// division by n as in k_train; hidden gradients are rounded to BF16 as there.  At the end the
// CTA writes its weight and bias gradients to partial[blockIdx.x] (k_reduce_adam sums them).
constexpr int kFhK = kGHid + 8;                                   // hidden tile row: 64 + ones + 7 zeros
constexpr int kGOneFeature = 6 * kGFreq + kGInputs;              // the constant-1 input feature
static_assert(kGOneFeature < kGIn, "the constant feature is one of layer 0's inputs");
constexpr int kFwBytes = kGHid * kGIn * 2 + 3 * kGHid * kGHid * 2 + kGOut * kGHid * 2;
constexpr int kFwtBytes = 3 * kGHid * kGHid * 2 + kGHid * kGOut * 2;
constexpr int kFX = 0;                                            // 128 x 96 features
constexpr int kFHBytes = kTcRows * kFhK * 2;
constexpr int kFH = kFX + kTcRows * kGIn * 2;                     // 4 tiles of 128 x 72
constexpr int kFD = kFH + 4 * kFHBytes;                           // 128 x (48 or 64) gradients
constexpr int kFW = kFD + kTcRows * kGHid * 2;                    // forward weights
constexpr int kFWt = kFW + kFwBytes;                              // W_l^T, l = 1..4
constexpr int kFBias = kFWt + kFwtBytes;
constexpr int kFBar = kFBias + (4 * kGHid + kGOut) * 4;
constexpr int kFTmem = kFBar + 8;
constexpr int kFSmem = kFTmem + 8;
constexpr int kFCols = 512;                                       // tensor-memory columns of the CTA
static_assert(kFH % 16 == 0 && kFHBytes % 16 == 0 && kFD % 16 == 0 && kFW % 16 == 0 && kFWt % 16 == 0 &&
                  kFBar % 8 == 0 && kFSmem <= 227 * 1024,
              "fused training layout: operands 16-byte aligned, mbarrier 8-byte aligned, within a CTA's limit");
// An MN-major read with M = 128 reaches up to 16 core-matrix rows (2 KB) past a tile's last
// record group; the buffers after each tile cover that.
static_assert(kFH + 4 * kFHBytes + 16 * 128 <= kFW, "MN-major reads stay inside the CTA's buffers");
static_assert(64 + 4 * kGHid + kGOut <= kFCols, "accumulator and weight gradients fit the tensor-memory allocation");

__device__ __forceinline__ int f_w(int l) { return kFW + (l == 0 ? 0 : kGHid * kGIn * 2 + (l - 1) * kGHid * kGHid * 2); }
__device__ __forceinline__ int f_wt(int l) { return kFWt + (l - 1) * kGHid * kGHid * 2; }  // l = 1..4
__device__ __forceinline__ int f_act(int l) { return l == 0 ? kFX : kFH + (l - 1) * kFHBytes; }  // layer l's input
__device__ __forceinline__ int f_act_k(int l) { return l == 0 ? kGIn : kFhK; }                   // its row length
__device__ __forceinline__ uint32_t f_dw_col(int l) { return 64u + 64u * (uint32_t)l; }

// Instruction descriptor of kind::f16 with both operands MN-major.
__host__ __device__ constexpr uint32_t tc_idesc_mn(int M, int N) { return tc_idesc(M, N) | (1u << 15) | (1u << 16); }

__global__ void __launch_bounds__(kTcRows, 1) k_step_tc(const GuideRecord* __restrict__ rec, int n,
                                                        const bf16* __restrict__ w16, const float* __restrict__ w32,
                                                        float* __restrict__ loss, float* __restrict__ partial,
                                                        int pool_n, unsigned long long seed, unsigned* err) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int t = threadIdx.x;
  const uint32_t bar = tc_smem(sm + kFBar);
  if (t < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(sm + kFTmem)),
                 "r"(kFCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // Weights in the forward layout and, for layers 1..4, transposed; biases in FP32.
  for (int l = 0; l < kGLayers; ++l) {
    const int K = guide_in(l), N = guide_out(l);
    const uint4* w = reinterpret_cast<const uint4*>(w16 + guide_w_offset(l));
    const int per_row = K / 8;
    for (int e = t; e < N * per_row; e += kTcRows) {
      const int o = e / per_row, i = (e - o * per_row) * 8;
      const uint4 v = __ldg(w + e);
      *reinterpret_cast<uint4*>(sm + f_w(l) + tc_off(o, i, K)) = v;
      if (l > 0) {
        const bf16* el = reinterpret_cast<const bf16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; ++j) *reinterpret_cast<bf16*>(sm + f_wt(l) + tc_off(i + j, o, N)) = el[j];
      }
    }
  }
  float* bias = reinterpret_cast<float*>(sm + kFBias);
  for (int l = 0; l < kGLayers; ++l)
    for (int c = t; c < guide_out(l); c += kTcRows) bias[l * kGHid + c] = w32[guide_b_offset(l) + c];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kFTmem);
  const uint32_t lanes = (uint32_t)((t >> 5) * 32) << 16;
  const float inv_n = 1.f / (float)n;
  const int ntiles = (n + kTcRows - 1) / kTcRows;
  uint32_t phase = 0;
  bool ok = true, first = true;
  float lsum = 0.f;

  // Makes every thread's shared-memory writes visible to the tensor cores and ends every
  // thread's reads of the accumulator; thread 0 then issues `issue` and commits it.  Waits
  // (bounded) for the commit; false, the same on every thread, when the wait gave up.
  auto run = [&](auto issue) {
    tc_fence_proxy();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t == 0) {
      issue();
      tc_commit(bar);
    }
    const bool done = __syncthreads_and(tc_wait(bar, phase & 1u) ? 1 : 0) != 0;
    ++phase;
    if (done) tc_fence_after();
    return done;
  };
  // K-major GEMM into the layer accumulator: A at a_off (row length ak), B at b_off (N rows
  // of K columns).
  auto mma_k = [&](int a_off, int ak, int b_off, int K, int N) {
    const uint32_t a0 = tc_smem(sm + a_off), b0 = tc_smem(sm + b_off);
    for (int ks = 0; ks < K / 16; ++ks)
      tc_mma(tmem, tc_desc(a0 + ks * 256, 128, ak * 16), tc_desc(b0 + ks * 256, 128, K * 16), tc_idesc(kTcRows, N),
             ks > 0 ? 1u : 0u);
  };
  // Weight gradient of layer l over the tile: A = its input tile, B = the gradient tile (row
  // length N = the layer's outputs), both MN-major (core matrices adjacent in M or N 128
  // bytes apart, adjacent in K one 8-record group apart), K = 128 records in steps of 16.
  auto mma_dw = [&](int l, bool init) {
    const int ak = f_act_k(l), N = guide_out(l);
    const uint32_t a0 = tc_smem(sm + f_act(l)), b0 = tc_smem(sm + kFD);
    for (int ks = 0; ks < kTcRows / 16; ++ks)
      tc_mma(tmem + f_dw_col(l), tc_desc(a0 + ks * 2 * (ak * 16), ak * 16, 128),
             tc_desc(b0 + ks * 2 * (N * 16), N * 16, 128), tc_idesc_mn(kTcRows, N), (init && ks == 0) ? 0u : 1u);
  };

  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long i = (long long)tile * kTcRows + t;
    const bool has = i < n;
    GuideRecord r{};
    if (has) {
      const long long src =
          pool_n > 0 ? (long long)(Rng::splitmix64(seed ^ Rng::splitmix64((unsigned long long)i)) % (unsigned long long)pool_n)
                     : i;
      r = rec[src];
    }
    {
      const float q[kGInputs] = {r.pos[0], r.pos[1], r.pos[2], r.n[0], r.n[1], r.n[2], r.wo[0], r.wo[1], r.wo[2]};
#pragma unroll
      for (int k = 0; k < kGIn; k += 8) {
        const uint4 v = has ? make_uint4(guide_feature_pair(q, k), guide_feature_pair(q, k + 2),
                                         guide_feature_pair(q, k + 4), guide_feature_pair(q, k + 6))
                            : make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(sm + kFX + tc_off(t, k, kGIn)) = v;
      }
    }
    uint32_t mask[4][2];
    float o[kGOut];
    for (int l = 0; l < kGLayers; ++l) {
      const int N = guide_out(l);
      if (!(ok = run([&] { mma_k(f_act(l), f_act_k(l), f_w(l), guide_in(l), N); }))) break;
      uint32_t v[kGHid];
      const uint32_t taddr = tmem + lanes;
      tc_ld16(taddr, v);
      tc_ld16(taddr + 16, v + 16);
      tc_ld16(taddr + 32, v + 32);
      if (N > 48) tc_ld16(taddr + 48, v + 48);
      tc_ld_wait();
      const float* bl = bias + l * kGHid;
      if (l < kGLayers - 1) {
        unsigned char* hrow = sm + f_act(l + 1);
        mask[l][0] = mask[l][1] = 0u;
#pragma unroll
        for (int k = 0; k < kGHid; k += 8) {
          uint32_t pw[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int c = k + 2 * j;
            pw[j] = pack_bf16x2(fmaxf(__uint_as_float(v[c]) + bl[c], 0.f),
                                fmaxf(__uint_as_float(v[c + 1]) + bl[c + 1], 0.f));
            // ReLU mask of the rounded activations, as the backward pass reads them.
            const uint32_t bits = (lo_bf16(pw[j]) > 0.f ? 1u : 0u) | (hi_bf16(pw[j]) > 0.f ? 2u : 0u);
            mask[l][c >> 5] |= bits << (c & 31);
          }
          *reinterpret_cast<uint4*>(hrow + tc_off(t, k, kFhK)) = make_uint4(pw[0], pw[1], pw[2], pw[3]);
        }
        // The ones column (bias gradients) of a record of the batch, zeros after it.
        *reinterpret_cast<uint4*>(hrow + tc_off(t, kGHid, kFhK)) =
            make_uint4(has ? pack_bf16x2(1.f, 0.f) : 0u, 0u, 0u, 0u);
      } else {
#pragma unroll
        for (int k = 0; k < kGOut; ++k) o[k] = __uint_as_float(v[k]) + bl[k];
      }
    }
    if (!ok) break;
    {
      // Loss and output gradient of this record, divided by n and rounded to BF16.
      float d[kGOut];
      if (has) {
        lsum += guide_loss_row(r, o, d);
      } else {
#pragma unroll
        for (int k = 0; k < kGOut; ++k) d[k] = 0.f;
      }
#pragma unroll
      for (int k = 0; k < kGOut; k += 8)
        *reinterpret_cast<uint4*>(sm + kFD + tc_off(t, k, kGOut)) =
            make_uint4(pack_bf16x2(d[k] * inv_n, d[k + 1] * inv_n), pack_bf16x2(d[k + 2] * inv_n, d[k + 3] * inv_n),
                       pack_bf16x2(d[k + 4] * inv_n, d[k + 5] * inv_n), pack_bf16x2(d[k + 6] * inv_n, d[k + 7] * inv_n));
    }
    for (int l = kGLayers - 1; l >= 1; --l) {
      // dH_{l-1} into the accumulator and dW_l into its columns, both from the gradient tile.
      if (!(ok = run([&] {
              mma_k(kFD, guide_out(l), f_wt(l), guide_out(l), kGHid);
              mma_dw(l, first);
            })))
        break;
      uint32_t v[kGHid];
      const uint32_t taddr = tmem + lanes;
      tc_ld16(taddr, v);
      tc_ld16(taddr + 16, v + 16);
      tc_ld16(taddr + 32, v + 32);
      tc_ld16(taddr + 48, v + 48);
      tc_ld_wait();
#pragma unroll
      for (int k = 0; k < kGHid; k += 8) {
        uint32_t pw[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int c = k + 2 * j;
          const uint32_t m = mask[l - 1][c >> 5] >> (c & 31);
          pw[j] = pack_bf16x2((m & 1u) ? __uint_as_float(v[c]) : 0.f, (m & 2u) ? __uint_as_float(v[c + 1]) : 0.f);
        }
        *reinterpret_cast<uint4*>(sm + kFD + tc_off(t, k, kGHid)) = make_uint4(pw[0], pw[1], pw[2], pw[3]);
      }
    }
    if (!ok) break;
    if (!(ok = run([&] { mma_dw(0, first); }))) break;
    first = false;
  }
  for (int s = 16; s > 0; s >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, s);
  if ((t & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum * inv_n);
  float* pw = partial + (size_t)blockIdx.x * kGParams;
  if (ok && !first) {
    // Lane t of each weight-gradient accumulator: dW_l[o][t] for the layer's inputs t, and
    // the bias gradient in the ones row (layer 0: the constant feature's row).
    for (int l = 0; l < kGLayers; ++l) {
      const int in = guide_in(l), out = guide_out(l);
      uint32_t v[kGHid];
      const uint32_t taddr = tmem + lanes + f_dw_col(l);
      tc_ld16(taddr, v);
      tc_ld16(taddr + 16, v + 16);
      tc_ld16(taddr + 32, v + 32);
      if (out > 48) tc_ld16(taddr + 48, v + 48);
      tc_ld_wait();
      if (t < in)
        for (int c = 0; c < out; ++c) pw[guide_w_offset(l) + c * in + t] = __uint_as_float(v[c]);
      if (t == (l == 0 ? kGOneFeature : kGHid))
        for (int c = 0; c < out; ++c) pw[guide_b_offset(l) + c] = __uint_as_float(v[c]);
    }
  } else {
    // No tile, or a wait gave up: this CTA adds nothing to the step.
    for (int e = t; e < kGParams; e += kTcRows) pw[e] = 0.f;
    if (!ok) {
      if (t == 0) atomicOr(err, kTcErrTimeout);
      if (phase > 0) tc_wait(bar, (phase - 1) & 1u);  // the last commit, before the memory is freed
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFCols));
}

__global__ void k_reduce(const float* __restrict__ part, int z, float* __restrict__ g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGParams; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < z; ++k) s += part[(size_t)k * kGParams + i];
    g[i] = s;
  }
}

// Forward pass of n rows of BF16 features (kGIn per row) into FP32 outputs (kGOut per row).
constexpr int kFwdWarps = 4;
constexpr int kFwdSmem = kGSmBytes + kFwdWarps * 16 * kGOutStride * 4;

__global__ void __launch_bounds__(kFwdWarps * 32) k_forward_x(const bf16* __restrict__ x, int n,
                                                              const bf16* __restrict__ w16,
                                                              const float* __restrict__ w32, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char fsm[];
  bf16* sw = reinterpret_cast<bf16*>(fsm);
  float* sb = reinterpret_cast<float*>(fsm + kGSmW * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* o = reinterpret_cast<float*>(fsm + kGSmBytes) + warp * 16 * kGOutStride;
  guide_smem_load(w16, w32, sw, sb);
  __syncthreads();
  for (int row0 = (blockIdx.x * kFwdWarps + warp) * 16; row0 < n; row0 += gridDim.x * kFwdWarps * 16) {
    uint32_t xf[6][4];
    guide_tile_load_x(x + (size_t)row0 * kGIn, n - row0, xf);
    guide_mlp_tile(sw, sb, xf, o, kGOutStride, nullptr);
    __syncwarp();
    for (int e = lane; e < 16 * kGOut; e += 32) {
      const int r = e / kGOut, c = e - r * kGOut;
      if (row0 + r < n) out[(size_t)(row0 + r) * kGOut + c] = o[r * kGOutStride + c];
    }
    __syncwarp();
  }
}

// The same forward pass on the tcgen05 tensor cores: each CTA (persistent) runs kTcChains
// independent chains of 128-row tiles over one shared copy of the weights.
__global__ void __launch_bounds__(kTcThreads) k_forward_tc(const bf16* __restrict__ x, int n, const bf16* __restrict__ w16,
                                                           const float* __restrict__ w32, float* __restrict__ out,
                                                           unsigned* err) {
  extern __shared__ __align__(128) unsigned char csm[];
  const TcChain c = tc_setup(csm);
  tc_load_weights(w16, w32, csm);
  __syncthreads();
  uint32_t phase = 0;
  bool ok = true;
  const int tiles = (n + kTcRows - 1) / kTcRows;
  const int g = threadIdx.x / kTcRows;
  for (int t = blockIdx.x * kTcChains + g; t < tiles; t += gridDim.x * kTcChains) {
    const long long r0 = (long long)t * kTcRows;
    tc_load_x(x, r0, n, csm, c);
    if (!tc_mlp_tile(csm, c, phase)) {  // the same on every thread of the chain
      ok = false;
      break;
    }
    tc_store_out(csm, r0, n, out, c);
    tc_chain_sync(c);  // the buffer is read out before the next tile's features land there
  }
  if (!ok) {
    atomicOr(err, kTcErrTimeout);
    tc_drain(c, phase);
  }
  tc_teardown(csm);
}

// Feature rows (BF16, kGIn) of n points given as 9 floats (p01, normal, wo): the input
// fragments the kernels above build, stored.
__global__ void __launch_bounds__(128) k_features(const float* __restrict__ pts, int n, bf16* __restrict__ x) {
  __shared__ float q[4][16 * kGInputs];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int row0 = (blockIdx.x * 4 + warp) * 16; row0 < n; row0 += gridDim.x * 4 * 16) {
    for (int e = lane; e < 16 * kGInputs; e += 32) {
      const int r = e / kGInputs;
      q[warp][e] = row0 + r < n ? pts[(size_t)row0 * kGInputs + e] : 0.f;
    }
    __syncwarp();
    uint32_t xf[6][4];
    guide_tile_features(q[warp], kGInputs, xf);
    guide_store_frags<6>(x, kGIn, xf, row0, n - row0);
    __syncwarp();
  }
}

// Adam (Kingma and Ba 2015) on the FP32 master parameters, refreshing the BF16 copy.
struct AdamArgs {
  float* p;
  float* m;
  float* v;
  bf16* w16;
  float lr, b1, b2, eps, bc1, bc2;
};
__device__ __forceinline__ void adam_one(const AdamArgs& a, int i, float gi) {
  const float mi = a.b1 * a.m[i] + (1.f - a.b1) * gi;
  const float vi = a.b2 * a.v[i] + (1.f - a.b2) * gi * gi;
  a.m[i] = mi;
  a.v[i] = vi;
  const float pi = a.p[i] - a.lr * (mi / a.bc1) / (sqrtf(vi / a.bc2) + a.eps);
  a.p[i] = pi;
  a.w16[i] = __float2bfloat16(pi);
}

__global__ void k_adam(AdamArgs a, const float* g, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) adam_one(a, i, g[i]);
}

// k_reduce and k_adam in one pass over the parameters (one launch less per training step).
__global__ void k_reduce_adam(const float* __restrict__ part, int z, float* __restrict__ g, AdamArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGParams; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < z; ++k) s += part[(size_t)k * kGParams + i];
    g[i] = s;
    adam_one(a, i, s);
  }
}

__global__ void k_to_bf16(const float* p, int n, bf16* w16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w16[i] = __float2bfloat16(p[i]);
}

int grid1(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 8192 ? 8192 : g));
}

// Resident-block capacity of a kernel on the current device (SMs x blocks per SM), with its
// dynamic shared-memory limit raised to `smem`; looked up once per kernel, launch shape and
// device, as a training step launches its kernels many times per pass.
int persistent_grid(const void* fn, int threads, int smem, long long work_blocks) {
  struct Entry {
    const void* fn;
    int dev, threads, smem;
    long long cap;
  };
  static std::mutex mu;
  static std::vector<Entry> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  long long cap = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : cache)
      if (e.fn == fn && e.dev == dev && e.threads == threads && e.smem == smem) cap = e.cap;
    if (cap == 0) {
      int sms = 0, per_sm = 0;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
      cap = (long long)std::max(1, sms) * (per_sm > 0 ? per_sm : 1);
      cache.push_back(Entry{fn, dev, threads, smem, cap});
    }
  }
  return (int)std::max(1LL, std::min(cap, work_blocks));
}


}  // namespace

// ----------------------------------------------------------------------------------------
GuideNet::~GuideNet() { release(); }

void GuideNet::release() {
  for (void* p : allocs) cudaFree(p);
  allocs.clear();
  for (void* p : scratch) cudaFree(p);
  scratch.clear();
  params = adam_m = adam_v = grad = loss = nullptr;
  params16 = nullptr;
  tc_err = nullptr;
  cap = 0;
}

template <class T>
static T* galloc(std::vector<void*>& allocs, size_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
  allocs.push_back(p);
  return static_cast<T*>(p);
}

bool GuideNet::init(uint64_t seed, std::string* err) {
  release();
  static bool attrs = false;
  if (!attrs) {
    cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
    cudaFuncSetAttribute(k_forward_x, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    attrs = true;
  }
  params = galloc<float>(allocs, kGParams);
  adam_m = galloc<float>(allocs, kGParams);
  adam_v = galloc<float>(allocs, kGParams);
  grad = galloc<float>(allocs, kGParams);
  params16 = galloc<bf16>(allocs, kGParams);
  loss = galloc<float>(allocs, 1);
  if (!params || !adam_m || !adam_v || !grad || !params16 || !loss) {
    *err = "guiding network: device allocation failed";
    return false;
  }
  // He-uniform initialisation (the output layer scaled by 0.1); zero biases.
  std::vector<float> h(kGParams, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kGLayers; ++l) {
    const float lim = std::sqrt(6.f / (float)guide_in(l)) * (l == kGLayers - 1 ? 0.1f : 1.f);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int i = 0; i < guide_in(l) * guide_out(l); ++i) h[guide_w_offset(l) + i] = U(rng);
  }
  cudaMemcpy(params, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(adam_m, 0, kGParams * sizeof(float));
  cudaMemset(adam_v, 0, kGParams * sizeof(float));
  k_to_bf16<<<grid1(kGParams), 256>>>(params, kGParams, params16);
  step = 0;
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    *err = std::string("guiding network init: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool GuideNet::set_params(const float* host, std::string* err) {
  fresh = false;
  cudaMemcpy(params, host, kGParams * sizeof(float), cudaMemcpyHostToDevice);
  k_to_bf16<<<grid1(kGParams), 256>>>(params, kGParams, params16);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool GuideNet::ensure_capacity(int n, std::string* err) {
  if (n <= cap) return true;
  for (void*& p : scratch) cudaFree(p);
  scratch.clear();
  auto al = [&](size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return (void*)nullptr;
    scratch.push_back(p);
    return p;
  };
  const size_t rows = (size_t)n;
  x0 = (bf16*)al(rows * kGIn * sizeof(bf16));
  for (int l = 0; l < 4; ++l) {
    h[l] = (bf16*)al(rows * kGHid * sizeof(bf16));
    dh[l] = (bf16*)al(rows * kGHid * sizeof(bf16));
  }
  out = (float*)al(rows * kGOut * sizeof(float));
  dy = (bf16*)al(rows * kGOut * sizeof(bf16));
  const int z = (n + kWgChunk - 1) / kWgChunk;
  partial = (float*)al((size_t)z * kGParams * sizeof(float));
  bool ok = x0 && out && dy && partial;
  for (int l = 0; l < 4; ++l) ok = ok && h[l] && dh[l];
  if (!ok) {
    for (void*& p : scratch) cudaFree(p);
    scratch.clear();
    cap = 0;
    *err = "guiding network: scratch allocation failed";
    return false;
  }
  cap = n;
  return true;
}

void GuideNet::forward(const bf16* x, int n, float* out_rows, cudaStream_t st) {
  const int grid = persistent_grid((const void*)k_forward_x, kFwdWarps * 32, kFwdSmem,
                                   (n + kFwdWarps * 16 - 1) / (kFwdWarps * 16));
  k_forward_x<<<grid, kFwdWarps * 32, kFwdSmem, st>>>(x, n, params16, params, out_rows);
}

bool GuideNet::forward_tc(const bf16* x, int n, float* out_rows, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    attr = true;
  }
  if (!tc_err) {
    if (cudaMalloc(&tc_err, sizeof(unsigned)) != cudaSuccess) return false;
    allocs.push_back(tc_err);
  }
  cudaMemsetAsync(tc_err, 0, sizeof(unsigned), st);
  const int grid = persistent_grid((const void*)k_forward_tc, kTcThreads, kTcSmem,
                                   (n + kTcThreads - 1) / kTcThreads);
  k_forward_tc<<<grid, kTcThreads, kTcSmem, st>>>(x, n, params16, params, out_rows, tc_err);
  unsigned e = 0;
  cudaMemcpyAsync(&e, tc_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return e == 0;
}

void GuideNet::features(const float* pts, int n, bf16* x, cudaStream_t st) {
  k_features<<<std::max(1, std::min(4096, (n + 63) / 64)), 128, 0, st>>>(pts, n, x);
}

static AdamArgs adam_args(GuideNet& g, float lr) {
  ++g.step;
  g.fresh = false;
  const float b1 = 0.9f, b2 = 0.999f;
  return AdamArgs{g.params, g.adam_m, g.adam_v, g.params16, lr, b1, b2, 1e-8f,
                  1.f - std::pow(b1, (float)g.step), 1.f - std::pow(b2, (float)g.step)};
}

void GuideNet::gradient(const GuideRecord* rec, int n, cudaStream_t st, bool adam_step, float lr, int pool_n,
                        uint64_t seed) {
  TrainBufs b{x0, {h[0], h[1], h[2], h[3]}, {dh[0], dh[1], dh[2], dh[3]}, dy, loss};
  cudaMemsetAsync(loss, 0, sizeof(float), st);
  if (wgrad_tc && !tc_err) {
    if (cudaMalloc(&tc_err, sizeof(unsigned)) == cudaSuccess) {
      allocs.push_back(tc_err);
      cudaMemsetAsync(tc_err, 0, sizeof(unsigned), st);
    } else {
      tc_err = nullptr;
    }
  }
  int z;
  if (wgrad_tc && tc_err) {
    z = persistent_grid((const void*)k_step_tc, kTcRows, kFSmem, (n + kTcRows - 1) / kTcRows);
    k_step_tc<<<z, kTcRows, kFSmem, st>>>(rec, n, params16, params, loss, partial, pool_n, seed, tc_err);
  } else {
    const int grid = persistent_grid((const void*)k_train, kTrainWarps * 32, kTrainSmem,
                                     (n + kTrainWarps * kTrainRows - 1) / (kTrainWarps * kTrainRows));
    k_train<<<grid, kTrainWarps * 32, kTrainSmem, st>>>(rec, n, params16, params, b, pool_n, seed);
    z = (n + kWgChunk - 1) / kWgChunk;
    k_wgrad<<<dim3(z, kGLayers), 128, 0, st>>>(n, b, partial);
  }
  if (adam_step)
    k_reduce_adam<<<grid1(kGParams), 256, 0, st>>>(partial, z, grad, adam_args(*this, lr));
  else
    k_reduce<<<grid1(kGParams), 256, 0, st>>>(partial, z, grad);
}


unsigned GuideNet::tensor_error(cudaStream_t st) {
  if (!tc_err) return 0u;
  unsigned e = 0u;
  cudaMemcpyAsync(&e, tc_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return e;
}

void GuideNet::adam(float lr, cudaStream_t st) {
  k_adam<<<grid1(kGParams), 256, 0, st>>>(adam_args(*this, lr), grad, kGParams);
}

}  // namespace tt
