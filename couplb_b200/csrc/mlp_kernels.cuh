// mlp_kernels.cuh -- the 84-64-64-3 no-slip correction network: parameter
// layout, the packed inference form and the warp-level forward pass that the
// learned IBM sub-step runs per marker.
//
// Parameters (FP32 master copy, flat): W1[64][84], b1[64], W2[64][64], b2[64],
// W3[3][64], b3[3].  The network computes in FP32 with weights rounded to
// BF16 (round to nearest even) and FP32 biases:
//   h1 = relu(W1 (s_in x) + b1), h2 = relu(W2 h1 + b2), y = (W3 h2 + b3) / s_out.
// x = (u0 at the 27 nodes round(l)-1..round(l)+1 of the marker, node-major
// dz,dy,dx; then v / vel_scale), all
// lattice velocities; y is the force correction over m xi vel_scale / dt.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace couplb {

constexpr int kMlpIn = 84, kMlpHid = 64, kMlpOut = 3, kMlpRow = 88;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpHid * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpHid;
constexpr int kMlpB2 = kMlpW2 + kMlpHid * kMlpHid;
constexpr int kMlpW3 = kMlpB2 + kMlpHid;
constexpr int kMlpB3 = kMlpW3 + kMlpOut * kMlpHid;
constexpr int kMlpNParam = kMlpB3 + kMlpOut;   // 9795

// Inference form, copied whole into shared memory by the learned sub-step.
// Hidden unit pairs (j, j+32) sit in one bf16x2 so lane j reads its two
// weights of an input column as one conflict-free 4-byte word.
struct __align__(16) MlpPacked {
  __nv_bfloat162 w1t[kMlpIn * 32];    // [k][lane] = (W1[lane][k], W1[lane+32][k])
  __nv_bfloat162 w2t[kMlpHid * 32];   // [k][lane] = (W2[lane][k], W2[lane+32][k])
  float b1[kMlpHid];
  float b2[kMlpHid];
  float w3[kMlpOut * kMlpHid];        // BF16-rounded values
  float b3[kMlpOut];
  float s_in, s_out;
  float pad[3];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked is copied in 16-byte words");

__device__ __forceinline__ float bf16_round(float v) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

// Copy the packed network into shared memory (all threads of the block).
__device__ __forceinline__ void mlp_stage(MlpPacked* dst, const MlpPacked* __restrict__ src) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) d[i] = __ldg(s + i);
}

// Forward pass of one sample by one warp.  xs: the warp's 84 inputs in shared
// memory (raw, lattice velocities), hs: 64 floats of warp scratch.  Every lane
// returns the three outputs.
__device__ __forceinline__ void mlp_warp_forward(const MlpPacked& P, const float* xs, float* hs,
                                                 int lane, float y[3]) {
  float a0 = P.b1[lane], a1 = P.b1[lane + 32];
#pragma unroll 4
  for (int k = 0; k < kMlpIn; k++) {
    const float xk = xs[k] * P.s_in;
    const float2 w = __bfloat1622float2(P.w1t[k * 32 + lane]);
    a0 = fmaf(w.x, xk, a0);
    a1 = fmaf(w.y, xk, a1);
  }
  __syncwarp();
  hs[lane] = fmaxf(a0, 0.f);
  hs[lane + 32] = fmaxf(a1, 0.f);
  __syncwarp();
  float c0 = P.b2[lane], c1 = P.b2[lane + 32];
#pragma unroll 4
  for (int k = 0; k < kMlpHid; k++) {
    const float hk = hs[k];
    const float2 w = __bfloat1622float2(P.w2t[k * 32 + lane]);
    c0 = fmaf(w.x, hk, c0);
    c1 = fmaf(w.y, hk, c1);
  }
  c0 = fmaxf(c0, 0.f);
  c1 = fmaxf(c1, 0.f);
#pragma unroll
  for (int c = 0; c < kMlpOut; c++) {
    float p = P.w3[c * kMlpHid + lane] * c0 + P.w3[c * kMlpHid + lane + 32] * c1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    y[c] = (p + P.b3[c]) / P.s_out;
  }
  __syncwarp();
}

}  // namespace couplb
