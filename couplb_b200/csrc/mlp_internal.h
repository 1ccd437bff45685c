// mlp_internal.h -- the correction-network handle, shared by mlp.cu and the
// engine (which reads its packed inference form).  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/couplb_b200.h"
#include "mlp_kernels.cuh"

struct couplb_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* w = nullptr;                  // FP32 master parameters (kMlpNParam)
  float* grad = nullptr;               // FP32 gradient accumulator
  float* m1 = nullptr;                 // Adam first moments
  float* m2 = nullptr;                 // Adam second moments
  couplb::MlpPacked* pack = nullptr;   // inference form (BF16 weights)
  double* d_acc = nullptr;             // FP64 loss / scale accumulators (64 doubles)
  double* h_acc = nullptr;             // pinned read-back of d_acc
  double s_in = 1.0, s_out = 1.0;      // input / target normalisation
  long long adam_step = 0;
  std::string err;
};
