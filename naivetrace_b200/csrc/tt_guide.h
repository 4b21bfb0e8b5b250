// Host side of the guiding network (tt_guide.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "tt_internal.h"

namespace tt {

struct GuideNet {
  std::vector<void*> allocs, scratch;
  float* params = nullptr;       // FP32 master parameters (guide_w_offset / guide_b_offset)
  __nv_bfloat16* params16 = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grad = nullptr;
  float* loss = nullptr;         // mean loss of the last gradient
  int step = 0;
  bool fresh = true;             // still the random initial weights (no Adam step, no set_params)
  // Training scratch for up to `cap` records: features, hidden activations, their
  // gradients, output gradients, FP32 outputs (batch forward) and the weight-gradient
  // partials of the record chunks.
  int cap = 0;
  __nv_bfloat16* x0 = nullptr;
  __nv_bfloat16* h[4] = {nullptr, nullptr, nullptr, nullptr};
  __nv_bfloat16* dh[4] = {nullptr, nullptr, nullptr, nullptr};
  float* out = nullptr;
  __nv_bfloat16* dy = nullptr;
  float* partial = nullptr;

  ~GuideNet();
  void release();
  bool init(uint64_t seed, std::string* err);
  bool set_params(const float* host, std::string* err);
  bool ensure_capacity(int n, std::string* err);
  // Forward pass of n rows of BF16 features into FP32 outputs.
  void forward(const __nv_bfloat16* x, int n, float* out_rows, cudaStream_t st);
  // The same on the tcgen05 tensor cores (tt_guide_tc.cuh); synchronous; false when a wait
  // on the tensor cores timed out.
  bool forward_tc(const __nv_bfloat16* x, int n, float* out_rows, cudaStream_t st);
  unsigned* tc_err = nullptr;
  // Training step on the tcgen05 tensor cores (k_step_tc: forward, backward and weight
  // gradients in one kernel; a wait that gave up sets tc_err) or on warp-level mma.sync
  // (k_train + k_wgrad).
  bool wgrad_tc = true;
  // Nonzero when a tcgen05 wait of the network kernels gave up (reads tc_err; synchronous).
  unsigned tensor_error(cudaStream_t st);
  // Feature rows of n points (9 floats each: position in [0,1]^3, normal, outgoing direction).
  void features(const float* pts, int n, __nv_bfloat16* x, cudaStream_t st);
  // Mean-loss gradient over n records into `grad` and the loss into `loss`; with adam_step
  // also the Adam step of size lr (as adam(), fused into the gradient's last kernel).  With
  // pool_n > 0 the records are a mini-batch of n drawn uniformly (with replacement) from
  // rec[0, pool_n) by `seed`, gathered from the pool by the gradient's first kernel.
  void gradient(const GuideRecord* rec, int n, cudaStream_t st, bool adam_step = false, float lr = 0.f,
                int pool_n = 0, uint64_t seed = 0);
  void adam(float lr, cudaStream_t st);
};

}  // namespace tt
