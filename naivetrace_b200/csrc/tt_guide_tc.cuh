// The guiding MLP on the 5th-generation tensor cores (tcgen05): a chain of 128 threads (four
// warps) runs the five layers for a tile of 128 rows, and a CTA runs kTcChains chains side
// by side over one copy of the weights, so that one chain's epilogue overlaps another's
// tensor-core work.  Operands sit in shared memory in the K-major
// "interleave" layout of the UMMA shared-memory descriptors (8 x 8 BF16 core matrices of
// 128 bytes; core matrices adjacent in K 128 bytes apart, 8-row groups K * 16 bytes apart),
// the FP32 accumulator of a layer (128 lanes x N columns) lives in tensor memory.  Per
// layer one thread of the chain issues K / 16 tcgen05.mma instructions (M = 128, N = 64 or
// 48, K = 16) and commits them to the chain's mbarrier; after the wait every thread reads its row's
// accumulators with tcgen05.ld, adds the bias, applies the ReLU and writes the BF16 row of
// the next layer's A operand back to shared memory.  Every wait is bounded; a timeout sets
// an error bit and the kernel still frees its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tt_guide.cuh"

namespace tt {

constexpr int kTcRows = 128;
constexpr int kTcChains = 4;                               // independent 128-row tiles per CTA
constexpr int kTcThreads = kTcRows * kTcChains;
constexpr int kTcCols = 64;                                // tensor-memory columns of one chain
// Shared-memory layout (bytes).
constexpr int kTcW0 = 0;                                   // 64 x 96
constexpr int kTcW1 = kTcW0 + kGHid * kGIn * 2;            // 64 x 64 (x3)
constexpr int kTcW4 = kTcW1 + 3 * kGHid * kGHid * 2;       // 48 x 64
// One tile buffer per chain: the features of its tile (128 x 96), then its hidden
// activations (128 x 64, over the features once layer 0 has read them), then the staged
// FP32 outputs (128 x 48).
constexpr int kTcX = kTcW4 + kGOut * kGHid * 2;
constexpr int kTcXBytes = kTcRows * kGIn * 2;
constexpr int kTcBias = kTcX + kTcChains * kTcXBytes;      // 4 x 64 + 48 floats
constexpr int kTcBar = kTcBias + (4 * kGHid + kGOut) * 4;  // one mbarrier (8 bytes) per chain
constexpr int kTcTmem = kTcBar + 8 * kTcChains;            // tensor-memory address
constexpr int kTcSmem = kTcTmem + 8;
constexpr unsigned kTcErrTimeout = 1u << 8;                // error bit: a wait gave up
static_assert(kTcW1 % 16 == 0 && kTcW4 % 16 == 0 && kTcX % 16 == 0 && kTcXBytes % 16 == 0,
              "UMMA operands start on 16-byte boundaries");
static_assert(kTcRows * kGHid * 2 <= kTcXBytes && kTcRows * kGOut * 4 <= kTcXBytes,
              "hidden activations and staged outputs fit in a tile buffer");
static_assert(kTcBar % 8 == 0 && kTcSmem <= 227 * 1024, "mbarriers 8-byte aligned; shared memory within a CTA's limit");
static_assert(kTcChains * kTcCols <= 512 && ((kTcChains * kTcCols) & (kTcChains * kTcCols - 1)) == 0,
              "a tensor-memory allocation is a power of two of at most 512 columns");
static_assert(kGIn % 16 == 0 && kGHid % 16 == 0 && kGOut % 16 == 0, "K and N in steps of 16");

// What one chain (four warps, 128 threads) of the CTA owns.
struct TcChain {
  int xo;          // byte offset of its tile buffer
  uint32_t tmem;   // its accumulator: kTcCols columns
  uint32_t lanes;  // tensor-memory lane offset of this warp (32 * (warp % 4)) << 16
  uint32_t bar;    // shared address of its mbarrier
  int bar_id;      // its named barrier (1 + chain)
  int row;         // this thread's row in the tile
  bool issuer;     // the thread that issues the chain's MMAs
};

// Byte offset of element (r, k) of a K-major operand with K columns.
__device__ __forceinline__ int tc_off(int r, int k, int K) {
  return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, K-major, no swizzle: start address, leading byte offset
// (between the two K-adjacent core matrices of one K = 16 step), stride byte offset
// (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the mbarrier phase; false if it gave up.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase) {
  for (int it = 0; it < (1 << 20); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_chain_sync(const TcChain& c) {
  asm volatile("bar.sync %0, %1;" ::"r"(c.bar_id), "r"(kTcRows) : "memory");
}
// Barrier of the chain that also ANDs `v` over its threads: every thread gets the same answer.
__device__ __forceinline__ bool tc_chain_all(const TcChain& c, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(c.bar_id), "r"(kTcRows)
      : "memory");
  return r != 0;
}

// 16 consecutive FP32 columns of this thread's lane (raw bits; complete after tc_ld_wait).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tc_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Weights (BF16 [out][in] per layer, rows of K a multiple of 8) into the K-major layout in
// 16-byte pieces, biases into FP32.
__device__ __forceinline__ void tc_load_weights(const __nv_bfloat16* __restrict__ w16, const float* __restrict__ w32,
                                                unsigned char* sm) {
  const int offs[5] = {kTcW0, kTcW1, kTcW1 + kGHid * kGHid * 2, kTcW1 + 2 * kGHid * kGHid * 2, kTcW4};
  for (int l = 0; l < kGLayers; ++l) {
    const int K = guide_in(l), N = guide_out(l);
    const uint4* w = reinterpret_cast<const uint4*>(w16 + guide_w_offset(l));
    const int pieces = N * K / 8, per_row = K / 8;
    for (int e = threadIdx.x; e < pieces; e += blockDim.x) {
      const int n = e / per_row, k = (e - n * per_row) * 8;
      *reinterpret_cast<uint4*>(sm + offs[l] + tc_off(n, k, K)) = __ldg(w + e);
    }
  }
  float* b = reinterpret_cast<float*>(sm + kTcBias);
  for (int l = 0; l < kGLayers; ++l) {
    const int N = guide_out(l);
    for (int c = threadIdx.x; c < N; c += blockDim.x) b[l * kGHid + c] = w32[guide_b_offset(l) + c];
  }
}

// Feature tile: rows r0 .. r0 + 127 of x (n x kGIn BF16, rows 16-byte aligned) into the
// chain's buffer, as coalesced 16-byte cp.async copies; rows past n are zeroed.  Complete
// for this thread on return.
__device__ __forceinline__ void tc_load_x(const __nv_bfloat16* __restrict__ x, long long r0, int n, unsigned char* sm,
                                          const TcChain& c) {
  constexpr int kPer = kGIn / 8;
  const uint4* src = reinterpret_cast<const uint4*>(x + r0 * kGIn);
  const long long rows = n - r0;
#pragma unroll 4
  for (int i = c.row; i < kTcRows * kPer; i += kTcRows) {
    const int r = i / kPer, q = i - r * kPer;
    unsigned char* dst = sm + c.xo + tc_off(r, q * 8, kGIn);
    if (r < rows)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc_smem(dst)), "l"(src + i) : "memory");
    else
      *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
  }
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// FP32 output row slot of the tile staged in the buffer at xo (128 x kGOut): 16-byte
// piece q of row r, rotated by r so that the writes of 8 rows spread over the banks.
__device__ __forceinline__ float4* tc_out_slot(unsigned char* sm, int xo, int r, int q) {
  constexpr int kPer = kGOut / 4;
  return reinterpret_cast<float4*>(sm + xo) + r * kPer + (q + r) % kPer;
}

// The staged outputs of rows r0 .. min(n, r0 + 128) - 1 to out (n x kGOut FP32), coalesced.
__device__ __forceinline__ void tc_store_out(unsigned char* sm, long long r0, int n, float* __restrict__ out,
                                             const TcChain& c) {
  constexpr int kPer = kGOut / 4;
  float4* dst = reinterpret_cast<float4*>(out + r0 * kGOut);
  const long long rows = n - r0;
#pragma unroll 4
  for (int i = c.row; i < kTcRows * kPer; i += kTcRows) {
    const int r = i / kPer, q = i - r * kPer;
    if (r < rows) dst[i] = *tc_out_slot(sm, c.xo, r, q);
  }
}

// Five layers on the 128 feature rows of the chain's buffer; the hidden activations
// replace the features there once layer 0 has read them, and the 48 outputs of row t are
// staged there at the end (tc_out_slot).  `phase` counts the chain's mbarrier phases
// (one per committed layer).  Returns false, the same on every thread of the chain, when a
// wait on a layer's commit gave up on any thread; the chain then issues no further MMAs,
// the caller stops using it and drains the outstanding commit with tc_drain before the
// tensor memory is freed.
__device__ __forceinline__ bool tc_mlp_tile(unsigned char* sm, const TcChain& c, uint32_t& phase) {
  const int offs[5] = {kTcW0, kTcW1, kTcW1 + kGHid * kGHid * 2, kTcW1 + 2 * kGHid * kGHid * 2, kTcW4};
  const float* bias = reinterpret_cast<const float*>(sm + kTcBias);
  bool ok = true;
  for (int l = 0; l < kGLayers; ++l) {
    const int K = guide_in(l), N = guide_out(l);
    // The A operand (written by every thread of the chain) is visible to the tensor cores,
    // and the chain's previous reads of its accumulator are done; the vote carries the
    // previous layer's wait.
    tc_fence_proxy();
    tc_fence_before();
    if (!tc_chain_all(c, ok)) return false;
    tc_fence_after();
    if (c.issuer) {
      const uint32_t a0 = tc_smem(sm + c.xo), b0 = tc_smem(sm + offs[l]);
      const uint32_t id = tc_idesc(kTcRows, N);
      for (int ks = 0; ks < K / 16; ++ks)
        tc_mma(c.tmem, tc_desc(a0 + ks * 256, 128, K * 16), tc_desc(b0 + ks * 256, 128, K * 16), id, ks > 0 ? 1u : 0u);
      tc_commit(c.bar);
    }
    // Warp-uniform, as tcgen05.ld is a warp-collective instruction.
    ok = __all_sync(0xffffffffu, tc_wait(c.bar, phase & 1u));
    ++phase;
    if (!ok) continue;  // nothing read from an accumulator that may still be written
    tc_fence_after();
    uint32_t v[kGHid];
    const uint32_t taddr = c.tmem + c.lanes;
    tc_ld16(taddr, v);
    tc_ld16(taddr + 16, v + 16);
    tc_ld16(taddr + 32, v + 32);
    if (N > 48) tc_ld16(taddr + 48, v + 48);
    tc_ld_wait();
    const float* b = bias + l * kGHid;
    if (l < kGLayers - 1) {
#pragma unroll
      for (int k = 0; k < kGHid; k += 8) {
        uint4 p;
        uint32_t* pw = reinterpret_cast<uint32_t*>(&p);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(__uint_as_float(v[k + 2 * j]) + b[k + 2 * j], 0.f),
                                                         fmaxf(__uint_as_float(v[k + 2 * j + 1]) + b[k + 2 * j + 1], 0.f));
          pw[j] = *reinterpret_cast<const uint32_t*>(&h);
        }
        *reinterpret_cast<uint4*>(sm + c.xo + tc_off(c.row, k, kGHid)) = p;
      }
    } else {
#pragma unroll
      for (int q = 0; q < kGOut / 4; ++q)
        *tc_out_slot(sm, c.xo, c.row, q) =
            make_float4(__uint_as_float(v[4 * q]) + b[4 * q], __uint_as_float(v[4 * q + 1]) + b[4 * q + 1],
                        __uint_as_float(v[4 * q + 2]) + b[4 * q + 2], __uint_as_float(v[4 * q + 3]) + b[4 * q + 3]);
    }
  }
  return tc_chain_all(c, ok);  // the staged outputs are complete
}

// After a failed tile: one more bounded wait for the chain's last commit, so that the
// tensor memory is not freed under an MMA that is still writing it.
__device__ __forceinline__ void tc_drain(const TcChain& c, uint32_t phase) {
  if (phase > 0) tc_wait(c.bar, (phase - 1) & 1u);
}

// Tensor-memory allocation of kTcChains * kTcCols columns by warp 0, the address published
// in shared memory; the chains' mbarriers initialised.  Returns this thread's chain.
__device__ __forceinline__ TcChain tc_setup(unsigned char* sm) {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(sm + kTcTmem)),
                 "r"(kTcChains * kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x < kTcChains) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(sm + kTcBar + 8 * threadIdx.x)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const int g = threadIdx.x / kTcRows;
  TcChain c;
  c.xo = kTcX + g * kTcXBytes;
  c.tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTcTmem) + (uint32_t)(g * kTcCols);
  c.lanes = (uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16;
  c.bar = tc_smem(sm + kTcBar + 8 * g);
  c.bar_id = 1 + g;
  c.row = threadIdx.x % kTcRows;
  c.issuer = c.row == 0;
  return c;
}

__device__ __forceinline__ void tc_teardown(unsigned char* sm) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     *reinterpret_cast<volatile uint32_t*>(sm + kTcTmem)),
                 "r"(kTcChains * kTcCols));
}

}  // namespace tt
