// mlp_kernels.cuh -- the 84-64-64-3 no-slip correction network: parameter
// layout, the packed inference form and the tensor-core forward pass that the
// learned IBM sub-step runs for the markers of a block.
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
#include <stdint.h>

namespace couplb {

constexpr int kMlpIn = 84, kMlpHid = 64, kMlpOut = 3, kMlpRow = 88;
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpHid * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpHid;
constexpr int kMlpB2 = kMlpW2 + kMlpHid * kMlpHid;
constexpr int kMlpW3 = kMlpB2 + kMlpHid;
constexpr int kMlpB3 = kMlpW3 + kMlpOut * kMlpHid;
constexpr int kMlpNParam = kMlpB3 + kMlpOut;   // 9795

// Inference form, copied whole into shared memory by the learned sub-step:
// BF16 weights row-major [output][input] with rows padded so that the
// tensor-core operand loads of a warp hit 32 distinct banks (stride 104 for
// the 84 inputs, 72 for the 64 hidden units; padding and W3 rows 3..7 are
// zero), FP32 biases.
constexpr int kMlpInPad = 96;     // K of layer 1 rounded up to the MMA k of 16
constexpr int kMlpW1Stride = 104; // bf16 per W1 row (13 x 8: bank-conflict-free B loads)
constexpr int kMlpW2Stride = 72;  // bf16 per W2 / W3 row
struct __align__(16) MlpPacked {
  __nv_bfloat16 w1[kMlpHid * kMlpW1Stride];
  __nv_bfloat16 w2[kMlpHid * kMlpW2Stride];
  __nv_bfloat16 w3[8 * kMlpW2Stride];
  float b1[kMlpHid];
  float b2[kMlpHid];
  float b3[4];
  float s_in, s_out;
  float pad[2];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked is copied in 16-byte words");

__device__ __forceinline__ float bf16_round(float v) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

// Copy the packed network into shared memory (all threads of the block) as
// asynchronous 16-byte copies (cp.async), so that the kernel's first loads
// overlap it; mlp_block_forward waits for this thread's
// copies and its first barrier publishes the block's.  dst and src are
// 16-byte aligned (MlpPacked is, and so is its slot in dynamic shared memory).
__device__ __forceinline__ void mlp_stage_async(MlpPacked* dst, const MlpPacked* __restrict__ src) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(d + i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(s + i) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// ---- block forward pass on the tensor cores -------------------------------
// One block of 8 warps evaluates the network for its 8 markers (one row per
// warp) with mma.sync m16n8k16 (BF16 operands, FP32 accumulation; rows 8-15
// of the M = 16 tile are zero).  The weights are BF16; the activations are
// FP32 and enter the MMA split into three BF16 parts, hi + mid + lo, which
// represent an FP32 value exactly, so every product weight x activation is
// the exact FP32 product and the network computes the same function as an
// FP32 evaluation with BF16 weights (up to the order of the FP32 sums).
constexpr int kMlpXStride = 104;  // floats per input row (84 used, the rest zero)
constexpr int kMlpHStride = 72;   // floats per hidden row
struct MlpBlockScratch {
  float x[8 * kMlpXStride];       // inputs (raw, lattice velocities), one row per warp
  float h1[8 * kMlpHStride];
  float h2[8 * kMlpHStride];
  float y[8 * 4];
};

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 v) {
  uint32_t u;
  memcpy(&u, &v, sizeof u);
  return u;
}

// (x0, x1) -> three BF16 pairs with x = hi + mid + lo exactly (FP32 inputs).
__device__ __forceinline__ void split3(float x0, float x1, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const float r0 = x0 - hf.x, r1 = x1 - hf.y;
  const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
  const float2 mf = __bfloat1622float2(m);
  const __nv_bfloat162 l = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
  hi = bf16x2_bits(h);
  mid = bf16x2_bits(m);
  lo = bf16x2_bits(l);
}

// D += A B for one m16n8k16 tile; a[1], a[3] (rows 8-15) are zero.
__device__ __forceinline__ void mma_rows8(float (&d)[4], uint32_t a0, uint32_t a2, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(0u), "r"(a2), "r"(0u), "r"(b0), "r"(b1));
}

// One k-step of 16 of a tile: the FP32 activations split into three BF16
// parts, each into its own accumulator (three independent MMA chains).
__device__ __forceinline__ void mlp_kstep(float (&ah)[4], float (&am)[4], float (&al)[4], const float* ar,
                                          const __nv_bfloat16* wr, int k0, float sa) {
  const float2 x0 = *reinterpret_cast<const float2*>(ar + k0);
  const float2 x1 = *reinterpret_cast<const float2*>(ar + k0 + 8);
  uint32_t h0, m0, l0, h1, m1, l1;
  split3(x0.x * sa, x0.y * sa, h0, m0, l0);
  split3(x1.x * sa, x1.y * sa, h1, m1, l1);
  const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + k0);
  const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + k0 + 8);
  mma_rows8(ah, h0, h1, b0, b1);
  mma_rows8(am, m0, m1, b0, b1);
  mma_rows8(al, l0, l1, b0, b1);
}

// acc (8 x 8 tile: rows = the block's markers, columns = 8 outputs starting at
// row n0 of W) += A[8][K] W^T, A FP32 rows of stride as (scaled by sa), W BF16
// rows of stride ws.  COMPACT: K at run time and the k loop not unrolled --
// for launches that run once per SM (few markers), whose time goes to
// fetching instructions; otherwise K at compile time, unrolled, for launches
// that loop over many markers.  Same sums in the same order either way.
template <bool COMPACT, int KC = 0>
__device__ __forceinline__ void mlp_tile(float (&acc)[4], const float* A, int as, float sa,
                                         const __nv_bfloat16* W, int ws, int n0, int K, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const float* ar = A + g * as + 2 * t;
  const __nv_bfloat16* wr = W + (n0 + g) * ws + 2 * t;
  float ah[4] = {0.f, 0.f, 0.f, 0.f}, am[4] = {0.f, 0.f, 0.f, 0.f}, al[4] = {0.f, 0.f, 0.f, 0.f};
  if constexpr (COMPACT) {
#pragma unroll 1
    for (int k0 = 0; k0 < K; k0 += 16) mlp_kstep(ah, am, al, ar, wr, k0, sa);
  } else {
#pragma unroll
    for (int k0 = 0; k0 < KC; k0 += 16) mlp_kstep(ah, am, al, ar, wr, k0, sa);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) acc[i] += ah[i] + (am[i] + al[i]);
}

// Output tile of layer `layer` (0, 1, 2) for warp `warp`: warp w forms
// outputs 8w..8w+7 of layers 1 and 2, warp 0 the three of layer 3.
template <bool COMPACT>
__device__ __forceinline__ void mlp_layer(const MlpPacked& P, MlpBlockScratch& S, int layer, int warp, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const bool first = layer == 0;
  const float* A = first ? S.x : (layer == 1 ? S.h1 : S.h2);
  const __nv_bfloat16* W = first ? P.w1 : (layer == 1 ? P.w2 : P.w3);
  const int n0 = layer < 2 ? 8 * warp : 0;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  if (COMPACT || !first)
    mlp_tile<COMPACT, kMlpHid>(acc, A, first ? kMlpXStride : kMlpHStride, first ? P.s_in : 1.f, W,
                               first ? kMlpW1Stride : kMlpW2Stride, n0, first ? kMlpInPad : kMlpHid, lane);
  else
    mlp_tile<false, kMlpInPad>(acc, A, kMlpXStride, P.s_in, W, kMlpW1Stride, n0, kMlpInPad, lane);
  const int j = n0 + 2 * t;
  if (layer < 2) {
    const float* b = first ? P.b1 : P.b2;
    float* H = first ? S.h1 : S.h2;
    H[g * kMlpHStride + j] = fmaxf(acc[0] + b[j], 0.f);
    H[g * kMlpHStride + j + 1] = fmaxf(acc[1] + b[j + 1], 0.f);
  } else {
    if (j < kMlpOut) S.y[g * 4 + j] = (acc[0] + P.b3[j]) / P.s_out;
    if (j + 1 < kMlpOut) S.y[g * 4 + j + 1] = (acc[1] + P.b3[j + 1]) / P.s_out;
  }
}

// Forward pass of the block's 8 rows (all 256 threads call it, after each
// warp has written its row of S.x); every lane of warp w gets row w's outputs.
//   h1 = relu(W1 (s_in x) + b1), h2 = relu(W2 h1 + b2), y = (W3 h2 + b3) / s_out.
// COMPACT (see mlp_tile): one loop over the layers; otherwise unrolled.
template <bool COMPACT>
__device__ __forceinline__ void mlp_block_forward(const MlpPacked& P, MlpBlockScratch& S, int warp,
                                                  int lane, float y[3]) {
  // this thread's part of an asynchronous staging of P (mlp_stage_async;
  // nothing pending otherwise), published to the block by the barrier
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  if constexpr (COMPACT) {
#pragma unroll 1
    for (int layer = 0; layer < 3; layer++) {
      if (layer < 2 || warp == 0) mlp_layer<true>(P, S, layer, warp, lane);
      __syncthreads();
    }
  } else {
#pragma unroll
    for (int layer = 0; layer < 3; layer++) {
      if (layer < 2 || warp == 0) mlp_layer<false>(P, S, layer, warp, lane);
      __syncthreads();
    }
  }
  y[0] = S.y[warp * 4];
  y[1] = S.y[warp * 4 + 1];
  y[2] = S.y[warp * 4 + 2];
}

}  // namespace couplb
