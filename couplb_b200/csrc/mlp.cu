// mlp.cu -- training and inference kernels of the 84-64-64-3 no-slip
// correction network, and its C ABI (couplb_mlp_*).
//
// Training runs on the GPU with the project's own kernels: one block of 256
// threads takes a tile of 64 rows, keeps the BF16 weights, the inputs and
// every activation of the tile in shared memory (118 KB), runs the forward
// pass, the squared-error loss and the backward pass, and adds its partial
// gradient to an FP32 accumulator with atomics; a second kernel applies Adam
// to the FP32 master weights.  The contractions run on the tensor cores
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation): a BF16 weight times
// an FP32 activation uses the exact three-part BF16 split of the activation
// (mlp_kernels.cuh), a product of two FP32 operands (the weight gradients)
// the six leading products of both splits, so every contraction keeps FP32
// accuracy.  The tiny layer-3 products (3 outputs) stay on the FP32 pipe.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mlp_internal.h"

using namespace couplb;

namespace {

constexpr int kTile = 64;
constexpr int kThreads = 256;
constexpr int kXS = kMlpXStride;   // FP32 row stride of the inputs (84 used, rest zero)
constexpr int kHS = kMlpHStride;   // FP32 row stride of the hidden activations / deltas
// shared memory, in bytes: BF16 W1 [64][104], W2 and W2^T [64][72], W3 [8][72];
// FP32 W3 [3][64], b1, b2, b3; X [64][104]; H1, H2, D2 [64][72]; Y, T [64][3]; scratch
constexpr size_t kOffW2 = 2 * kMlpHid * kMlpW1Stride;
constexpr size_t kOffW2T = kOffW2 + 2 * kMlpHid * kMlpW2Stride;
constexpr size_t kOffW3b = kOffW2T + 2 * kMlpHid * kMlpW2Stride;
constexpr size_t kOffF = kOffW3b + 2 * 8 * kMlpW2Stride;   // first FP32 array
constexpr int kTileFloats = kMlpOut * kMlpHid + 2 * kMlpHid + 4 + kTile * kXS + 3 * kTile * kHS +
                            2 * kTile * kMlpOut + 32;
constexpr size_t kTileSmem = kOffF + sizeof(float) * kTileFloats;
constexpr int kAccSlots = 32;

// SplitMix64 (Steele, Lea & Flood, OOPSLA 2014): minibatch row sampling and
// weight initialisation.
__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct TileArgs {
  const float* rows;
  long long base, limit;       // sequential: rows base + 64 b + s below limit
  int random;                  // 1: rows drawn uniformly from [0, n_pick)
  unsigned long long seed;
  long long step, n_pick;
  const float* w;
  float s_in, s_out;
  float inv_norm;              // 1 / (3 B)
  double* loss;                // null: no loss
  float* grad;                 // null: no backward pass
  float* out;                  // null: outputs not stored
};

// ---- tensor-core tiles of the training kernel ------------------------------
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Fragment element pairs of an m16n8k16 tile for lane (g = lane / 4,
// t = lane % 4): A rows g and g + 8, columns 2t, 2t + 1 and 2t + 8, 2t + 9;
// B columns (n) g, rows (k) 2t, 2t + 1 and 2t + 8, 2t + 9.
// A = M[m0.., k0..] of a row-major FP32 array (stride ms), split in three.
__device__ __forceinline__ void frag_a_rows(const float* M, int ms, int m0, int k0, int g, int t,
                                            uint32_t (&h)[4], uint32_t (&m)[4], uint32_t (&l)[4]) {
  const float* r0 = M + (m0 + g) * ms + k0 + 2 * t;
  const float* r1 = r0 + 8 * ms;
  split3(r0[0], r0[1], h[0], m[0], l[0]);
  split3(r1[0], r1[1], h[1], m[1], l[1]);
  split3(r0[8], r0[9], h[2], m[2], l[2]);
  split3(r1[8], r1[9], h[3], m[3], l[3]);
}
// A = M^T[m0.., k0..] of a row-major FP32 array M [k][m] (stride ms), split in three.
__device__ __forceinline__ void frag_a_cols(const float* M, int ms, int m0, int k0, int g, int t,
                                            uint32_t (&h)[4], uint32_t (&m)[4], uint32_t (&l)[4]) {
  const float* c = M + (k0 + 2 * t) * ms + m0 + g;
  split3(c[0], c[ms], h[0], m[0], l[0]);
  split3(c[8], c[ms + 8], h[1], m[1], l[1]);
  split3(c[8 * ms], c[9 * ms], h[2], m[2], l[2]);
  split3(c[8 * ms + 8], c[9 * ms + 8], h[3], m[3], l[3]);
}
// B = M[k0.., n0..] of a row-major FP32 array M [k][n] (stride ms), split in three.
__device__ __forceinline__ void frag_b_rows(const float* M, int ms, int k0, int n0, int g, int t,
                                            uint32_t (&h)[2], uint32_t (&m)[2], uint32_t (&l)[2]) {
  const float* c = M + (k0 + 2 * t) * ms + n0 + g;
  split3(c[0], c[ms], h[0], m[0], l[0]);
  split3(c[8 * ms], c[9 * ms], h[1], m[1], l[1]);
}
// B = W^T[k0.., n0..] of a row-major BF16 array W [n][k] (stride ws): exact.
__device__ __forceinline__ void frag_b_bf16(const __nv_bfloat16* W, int ws, int k0, int n0, int g, int t,
                                            uint32_t& b0, uint32_t& b1) {
  const __nv_bfloat16* r = W + (n0 + g) * ws + k0 + 2 * t;
  b0 = *reinterpret_cast<const uint32_t*>(r);
  b1 = *reinterpret_cast<const uint32_t*>(r + 8);
}

// D[16 x 8] += A (FP32 rows of M, split) * W^T (BF16): three products.
template <int K>
__device__ __forceinline__ void tile_act_w(float (&d)[4], const float* M, int ms, int m0,
                                           const __nv_bfloat16* W, int ws, int n0, int g, int t) {
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t h[4], m[4], l[4], b0, b1;
    frag_a_rows(M, ms, m0, k0, g, t, h, m, l);
    frag_b_bf16(W, ws, k0, n0, g, t, b0, b1);
    mma16816(d, h, b0, b1);
    mma16816(d, m, b0, b1);
    mma16816(d, l, b0, b1);
  }
}

// D[16 x 8] += P^T[m0.., :] Q[:, n0..] over the tile's 64 rows, P and Q FP32
// row-major [row][.] (strides ps, qs): the six leading products of the
// three-part splits (the dropped ones are below 2^-24 relative).
__device__ __forceinline__ void tile_grad(float (&d)[4], const float* Pm, int ps, int m0, const float* Qm,
                                          int qs, int n0, int g, int t) {
#pragma unroll
  for (int k0 = 0; k0 < kTile; k0 += 16) {
    uint32_t ah[4], am[4], al[4], bh[2], bm[2], bl[2];
    frag_a_cols(Pm, ps, m0, k0, g, t, ah, am, al);
    frag_b_rows(Qm, qs, k0, n0, g, t, bh, bm, bl);
    mma16816(d, ah, bh[0], bh[1]);
    mma16816(d, ah, bm[0], bm[1]);
    mma16816(d, am, bh[0], bh[1]);
    mma16816(d, ah, bl[0], bl[1]);
    mma16816(d, am, bm[0], bm[1]);
    mma16816(d, al, bh[0], bh[1]);
  }
}

__global__ void __launch_bounds__(kThreads) k_mlp_tile(const TileArgs A) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __nv_bfloat16* W1b = reinterpret_cast<__nv_bfloat16*>(smraw);
  __nv_bfloat16* W2b = reinterpret_cast<__nv_bfloat16*>(smraw + kOffW2);
  __nv_bfloat16* W2Tb = reinterpret_cast<__nv_bfloat16*>(smraw + kOffW2T);
  __nv_bfloat16* W3b = reinterpret_cast<__nv_bfloat16*>(smraw + kOffW3b);
  float* W3 = reinterpret_cast<float*>(smraw + kOffF);
  float* B1 = W3 + kMlpOut * kMlpHid;
  float* B2 = B1 + kMlpHid;
  float* B3 = B2 + kMlpHid;
  float* X = B3 + 4;
  float* H1 = X + kTile * kXS;
  float* H2 = H1 + kTile * kHS;
  float* D2 = H2 + kTile * kHS;
  float* Y = D2 + kTile * kHS;
  float* T = Y + kTile * kMlpOut;
  float* RED = T + kTile * kMlpOut;
  __shared__ long long idx[kTile];
  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);

  for (int e = t; e < kMlpHid * kMlpW1Stride; e += kThreads) {
    const int n = e / kMlpW1Stride, k = e % kMlpW1Stride;
    W1b[e] = k < kMlpIn ? __float2bfloat16_rn(A.w[kMlpW1 + n * kMlpIn + k]) : zero;
  }
  for (int e = t; e < kMlpHid * kMlpW2Stride; e += kThreads) {
    const int n = e / kMlpW2Stride, k = e % kMlpW2Stride;
    W2b[e] = k < kMlpHid ? __float2bfloat16_rn(A.w[kMlpW2 + n * kMlpHid + k]) : zero;
    W2Tb[e] = k < kMlpHid ? __float2bfloat16_rn(A.w[kMlpW2 + k * kMlpHid + n]) : zero;
  }
  for (int e = t; e < 8 * kMlpW2Stride; e += kThreads) {
    const int n = e / kMlpW2Stride, k = e % kMlpW2Stride;
    W3b[e] = (n < kMlpOut && k < kMlpHid) ? __float2bfloat16_rn(A.w[kMlpW3 + n * kMlpHid + k]) : zero;
  }
  for (int e = t; e < kMlpOut * kMlpHid; e += kThreads) W3[e] = bf16_round(A.w[kMlpW3 + e]);
  if (t < kMlpHid) { B1[t] = A.w[kMlpB1 + t]; B2[t] = A.w[kMlpB2 + t]; }
  if (t < kMlpOut) B3[t] = A.w[kMlpB3 + t];
  if (t < kTile) {
    long long r;
    if (A.random) {
      const unsigned long long h =
          splitmix64(A.seed ^ splitmix64((unsigned long long)A.step * 0x100000001ULL +
                                         (unsigned long long)blockIdx.x * kTile + t));
      r = (long long)(h % (unsigned long long)A.n_pick);
    } else {
      r = A.base + (long long)blockIdx.x * kTile + t;
      if (r >= A.limit) r = -1;
    }
    idx[t] = r;
  }
  __syncthreads();
  for (int e = t; e < kTile * kXS; e += kThreads) {
    const int s = e / kXS, k = e % kXS;
    const long long r = idx[s];
    float v = 0.f;
    if (k < kMlpIn && r >= 0) v = __ldg(A.rows + r * kMlpRow + k) * A.s_in;
    X[e] = v;
  }
  for (int e = t; e < kTile * kMlpOut; e += kThreads) {
    const int s = e / kMlpOut, c = e % kMlpOut;
    const long long r = idx[s];
    T[e] = r >= 0 ? __ldg(A.rows + r * kMlpRow + kMlpIn + c) : 0.f;
  }
  __syncthreads();

  // forward: warp w takes row tile w % 4 and the four column tiles 4 (w / 4) ..
  const int mt = (warp & 3) * 16;
  for (int c = 0; c < 4; c++) {
    const int n0 = ((warp >> 2) * 4 + c) * 8;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_act_w<kMlpInPad>(d, X, kXS, mt, W1b, kMlpW1Stride, n0, g, q);
    const int j = n0 + 2 * q;
    H1[(mt + g) * kHS + j] = fmaxf(d[0] + B1[j], 0.f);
    H1[(mt + g) * kHS + j + 1] = fmaxf(d[1] + B1[j + 1], 0.f);
    H1[(mt + g + 8) * kHS + j] = fmaxf(d[2] + B1[j], 0.f);
    H1[(mt + g + 8) * kHS + j + 1] = fmaxf(d[3] + B1[j + 1], 0.f);
  }
  __syncthreads();
  for (int c = 0; c < 4; c++) {
    const int n0 = ((warp >> 2) * 4 + c) * 8;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_act_w<kMlpHid>(d, H1, kHS, mt, W2b, kMlpW2Stride, n0, g, q);
    const int j = n0 + 2 * q;
    H2[(mt + g) * kHS + j] = fmaxf(d[0] + B2[j], 0.f);
    H2[(mt + g) * kHS + j + 1] = fmaxf(d[1] + B2[j + 1], 0.f);
    H2[(mt + g + 8) * kHS + j] = fmaxf(d[2] + B2[j], 0.f);
    H2[(mt + g + 8) * kHS + j + 1] = fmaxf(d[3] + B2[j + 1], 0.f);
  }
  __syncthreads();
  if (warp < 4) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_act_w<kMlpHid>(d, H2, kHS, mt, W3b, kMlpW2Stride, 0, g, q);
    for (int hrow = 0; hrow < 2; hrow++) {
      const int s = mt + g + 8 * hrow;
      for (int cc = 0; cc < 2; cc++) {
        const int c = 2 * q + cc;
        if (c >= kMlpOut) continue;
        const float a = d[2 * hrow + cc] + B3[c];
        Y[s * kMlpOut + c] = a;
        if (A.out && idx[s] >= 0) A.out[idx[s] * kMlpOut + c] = a / A.s_out;
      }
    }
  }
  __syncthreads();
  if (!A.loss) return;

  // loss (mean squared error of the normalised outputs) and dL/dy
  float lp = 0.f;
  if (t < kTile * kMlpOut) {
    const int s = t / kMlpOut;
    const float e = idx[s] >= 0 ? Y[t] - A.s_out * T[t] : 0.f;
    lp = e * e * A.inv_norm;
    Y[t] = 2.f * e * A.inv_norm;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lp += __shfl_xor_sync(0xffffffffu, lp, o);
  if ((t & 31) == 0) RED[t >> 5] = lp;
  __syncthreads();
  if (t == 0) {
    double sm = 0.0;
    for (int i = 0; i < kThreads / 32; i++) sm += RED[i];
    atomicAdd(A.loss + (blockIdx.x & (kAccSlots - 1)), sm);
  }
  if (!A.grad) return;

  // backward: layer 3 (three outputs: FP32 pipe), then
  // delta2 = (W3^T dy) * relu'(h2)
  if (t < kMlpOut * kMlpHid) {
    const int c = t / kMlpHid, k = t % kMlpHid;
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a = fmaf(Y[s * kMlpOut + c], H2[s * kHS + k], a);
    atomicAdd(A.grad + kMlpW3 + t, a);
  }
  if (t < kMlpOut) {
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a += Y[s * kMlpOut + t];
    atomicAdd(A.grad + kMlpB3 + t, a);
  }
  for (int e = t; e < kTile * kMlpHid; e += kThreads) {
    const int s = e / kMlpHid, k = e % kMlpHid;
    float a = 0.f;
    if (H2[s * kHS + k] > 0.f)
      for (int c = 0; c < kMlpOut; c++) a = fmaf(W3[c * kMlpHid + k], Y[s * kMlpOut + c], a);
    D2[s * kHS + k] = a;
  }
  __syncthreads();
  // layer 2 gradient dW2 = delta2^T h1 (row tile = hidden unit j of layer 2)
  for (int c = 0; c < 4; c++) {
    const int n0 = ((warp >> 2) * 4 + c) * 8;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_grad(d, D2, kHS, mt, H1, kHS, n0, g, q);
    const int j0 = mt + g, k = n0 + 2 * q;
    atomicAdd(A.grad + kMlpW2 + j0 * kMlpHid + k, d[0]);
    atomicAdd(A.grad + kMlpW2 + j0 * kMlpHid + k + 1, d[1]);
    atomicAdd(A.grad + kMlpW2 + (j0 + 8) * kMlpHid + k, d[2]);
    atomicAdd(A.grad + kMlpW2 + (j0 + 8) * kMlpHid + k + 1, d[3]);
  }
  if (t < kMlpHid) {
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a += D2[s * kHS + t];
    atomicAdd(A.grad + kMlpB2 + t, a);
  }
  // delta1 = (W2^T delta2) * relu'(h1), into H2 (h2 is no longer read)
  for (int c = 0; c < 4; c++) {
    const int n0 = ((warp >> 2) * 4 + c) * 8;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_act_w<kMlpHid>(d, D2, kHS, mt, W2Tb, kMlpW2Stride, n0, g, q);
    const int k = n0 + 2 * q;
    for (int hrow = 0; hrow < 2; hrow++) {
      const int s = mt + g + 8 * hrow;
      H2[s * kHS + k] = H1[s * kHS + k] > 0.f ? d[2 * hrow] : 0.f;
      H2[s * kHS + k + 1] = H1[s * kHS + k + 1] > 0.f ? d[2 * hrow + 1] : 0.f;
    }
  }
  __syncthreads();
  // layer 1 gradient dW1 = delta1^T x: 4 row tiles (hidden) x 11 column tiles (inputs)
  for (int tile = warp; tile < 4 * 11; tile += kThreads / 32) {
    const int m0 = (tile & 3) * 16, n0 = (tile >> 2) * 8;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    tile_grad(d, H2, kHS, m0, X, kXS, n0, g, q);
    const int j0 = m0 + g, k = n0 + 2 * q;
    if (k < kMlpIn) {
      atomicAdd(A.grad + kMlpW1 + j0 * kMlpIn + k, d[0]);
      atomicAdd(A.grad + kMlpW1 + (j0 + 8) * kMlpIn + k, d[2]);
    }
    if (k + 1 < kMlpIn) {
      atomicAdd(A.grad + kMlpW1 + j0 * kMlpIn + k + 1, d[1]);
      atomicAdd(A.grad + kMlpW1 + (j0 + 8) * kMlpIn + k + 1, d[3]);
    }
  }
  if (t < kMlpHid) {
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a += H2[s * kHS + t];
    atomicAdd(A.grad + kMlpB1 + t, a);
  }
}

// Adam on the FP32 master weights; clears the gradient it consumed.
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ g, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpNParam) return;
  const float gi = g[i];
  g[i] = 0.f;
  const float m = b1 * m1[i] + (1.f - b1) * gi;
  const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = m;
  m2[i] = v;
  w[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// Inference form (BF16 weights in the padded row-major layout of MlpPacked)
// from the master weights.
__global__ void k_mlp_pack(const float* __restrict__ w, float s_in, float s_out, MlpPacked* P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nt = gridDim.x * blockDim.x;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
  for (int e = t; e < kMlpHid * kMlpW1Stride; e += nt) {
    const int n = e / kMlpW1Stride, k = e % kMlpW1Stride;
    P->w1[e] = k < kMlpIn ? __float2bfloat16_rn(w[kMlpW1 + n * kMlpIn + k]) : zero;
  }
  for (int e = t; e < kMlpHid * kMlpW2Stride; e += nt) {
    const int n = e / kMlpW2Stride, k = e % kMlpW2Stride;
    P->w2[e] = k < kMlpHid ? __float2bfloat16_rn(w[kMlpW2 + n * kMlpHid + k]) : zero;
  }
  for (int e = t; e < 8 * kMlpW2Stride; e += nt) {
    const int n = e / kMlpW2Stride, k = e % kMlpW2Stride;
    P->w3[e] = (n < kMlpOut && k < kMlpHid) ? __float2bfloat16_rn(w[kMlpW3 + n * kMlpHid + k]) : zero;
  }
  for (int e = t; e < kMlpHid; e += nt) {
    P->b1[e] = w[kMlpB1 + e];
    P->b2[e] = w[kMlpB2 + e];
  }
  if (t < 4) P->b3[t] = t < kMlpOut ? w[kMlpB3 + t] : 0.f;
  if (t == 0) {
    P->s_in = s_in;
    P->s_out = s_out;
    P->pad[0] = P->pad[1] = 0.f;
  }
}

// Sums of squares of the inputs (acc[0..31]) and targets (acc[32..63]).
__global__ void k_mlp_scale_sums(const float* __restrict__ rows, long long n, double* acc) {
  double sx = 0.0, st = 0.0;
  const long long total = n * (kMlpIn + kMlpOut);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / (kMlpIn + kMlpOut);
    const int k = (int)(e % (kMlpIn + kMlpOut));
    const double v = rows[r * kMlpRow + k];
    if (k < kMlpIn) sx += v * v; else st += v * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    st += __shfl_xor_sync(0xffffffffu, st, o);
  }
  if ((threadIdx.x & 31) == 0) {
    const int slot = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) & (kAccSlots - 1);
    atomicAdd(acc + slot, sx);
    atomicAdd(acc + kAccSlots + slot, st);
  }
}

int mfail(couplb_mlp* m, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (m) m->err = buf;
  return code;
}

#define MCK(call)                                                                  \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return mfail(m, COUPLB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));   \
  } while (0)

int set_dev(couplb_mlp* m) {
  MCK(cudaSetDevice(m->device));
  return COUPLB_OK;
}

int pack(couplb_mlp* m) {
  k_mlp_pack<<<8, 256, 0, m->stream>>>(m->w, (float)m->s_in, (float)m->s_out, m->pack);
  MCK(cudaGetLastError());
  return COUPLB_OK;
}

int tile_launch(couplb_mlp* m, const TileArgs& a, long long blocks) {
  static_assert(kTileSmem <= 227 * 1024, "tile fits in shared memory");
  MCK(cudaFuncSetAttribute(k_mlp_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
  k_mlp_tile<<<(unsigned)blocks, kThreads, kTileSmem, m->stream>>>(a);
  MCK(cudaGetLastError());
  return COUPLB_OK;
}

// Sum of the first nslots accumulators (synchronises); clears them all.
int read_acc(couplb_mlp* m, int nslots, double* out) {
  MCK(cudaMemcpyAsync(m->h_acc, m->d_acc, sizeof(double) * nslots, cudaMemcpyDeviceToHost, m->stream));
  MCK(cudaMemsetAsync(m->d_acc, 0, sizeof(double) * 2 * kAccSlots, m->stream));
  MCK(cudaStreamSynchronize(m->stream));
  double s = 0.0;
  for (int i = 0; i < nslots; i++) s += m->h_acc[i];
  *out = s;
  return COUPLB_OK;
}

// Loss over rows [base, base + n) (forward only); synchronises.
int eval_loss(couplb_mlp* m, const float* rows, long long base, long long n, double* loss) {
  if (n <= 0) { *loss = 0.0; return COUPLB_OK; }
  TileArgs a{};
  a.rows = rows; a.base = base; a.limit = base + n;
  a.w = m->w; a.s_in = (float)m->s_in; a.s_out = (float)m->s_out;
  a.inv_norm = (float)(1.0 / (3.0 * (double)n));
  a.loss = m->d_acc;
  int rc = tile_launch(m, a, (n + kTile - 1) / kTile);
  if (rc) return rc;
  return read_acc(m, kAccSlots, loss);
}

}  // namespace

extern "C" {

int couplb_mlp_create(int device, unsigned long long seed, couplb_mlp** out) {
  if (!out) return COUPLB_ERR_ARG;
  *out = nullptr;
  couplb_mlp* m = new couplb_mlp();
  m->device = device;
  auto bad = [&](int code) {
    couplb_mlp_destroy(m);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bad(COUPLB_ERR_CUDA);
  const size_t pb = sizeof(float) * kMlpNParam;
  if (cudaMalloc(&m->w, pb) != cudaSuccess || cudaMalloc(&m->grad, pb) != cudaSuccess ||
      cudaMalloc(&m->m1, pb) != cudaSuccess || cudaMalloc(&m->m2, pb) != cudaSuccess ||
      cudaMalloc(&m->pack, sizeof(MlpPacked)) != cudaSuccess ||
      cudaMalloc(&m->d_acc, sizeof(double) * 2 * kAccSlots) != cudaSuccess ||
      cudaMallocHost(&m->h_acc, sizeof(double) * 2 * kAccSlots) != cudaSuccess)
    return bad(COUPLB_ERR_CUDA);
  // He-uniform weights for the ReLU layers, fan-in uniform for the output
  // layer, zero biases.
  std::vector<float> w(kMlpNParam, 0.f);
  unsigned long long st = seed;
  auto uni = [&]() {
    st = splitmix64(st);
    return (double)(st >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  const double a1 = std::sqrt(6.0 / kMlpIn), a2 = std::sqrt(6.0 / kMlpHid), a3 = std::sqrt(1.0 / kMlpHid);
  for (int e = 0; e < kMlpHid * kMlpIn; e++) w[kMlpW1 + e] = (float)(a1 * uni());
  for (int e = 0; e < kMlpHid * kMlpHid; e++) w[kMlpW2 + e] = (float)(a2 * uni());
  for (int e = 0; e < kMlpOut * kMlpHid; e++) w[kMlpW3 + e] = (float)(a3 * uni());
  if (cudaMemcpy(m->w, w.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->grad, 0, pb) != cudaSuccess || cudaMemset(m->m1, 0, pb) != cudaSuccess ||
      cudaMemset(m->m2, 0, pb) != cudaSuccess ||
      cudaMemset(m->d_acc, 0, sizeof(double) * 2 * kAccSlots) != cudaSuccess)
    return bad(COUPLB_ERR_CUDA);
  if (pack(m) || cudaStreamSynchronize(m->stream) != cudaSuccess) return bad(COUPLB_ERR_CUDA);
  *out = m;
  return COUPLB_OK;
}

int couplb_mlp_destroy(couplb_mlp* m) {
  if (!m) return COUPLB_OK;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->w);
  cudaFree(m->grad);
  cudaFree(m->m1);
  cudaFree(m->m2);
  cudaFree(m->pack);
  cudaFree(m->d_acc);
  if (m->h_acc) cudaFreeHost(m->h_acc);
  delete m;
  return COUPLB_OK;
}

const char* couplb_mlp_last_error(const couplb_mlp* m) { return m ? m->err.c_str() : "null network"; }

int couplb_mlp_set_stream(couplb_mlp* m, void* s) {
  if (!m) return COUPLB_ERR_ARG;
  m->stream = (cudaStream_t)s;
  return COUPLB_OK;
}

int couplb_mlp_set_weights(couplb_mlp* m, const float* w, double s_in, double s_out) {
  if (!m || !w) return COUPLB_ERR_ARG;
  if (!(s_in > 0.0) || !(s_out > 0.0) || !std::isfinite(s_in) || !std::isfinite(s_out))
    return mfail(m, COUPLB_ERR_ARG, "scales must be positive and finite");
  int rc = set_dev(m);
  if (rc) return rc;
  MCK(cudaMemcpyAsync(m->w, w, sizeof(float) * kMlpNParam, cudaMemcpyHostToDevice, m->stream));
  MCK(cudaMemsetAsync(m->m1, 0, sizeof(float) * kMlpNParam, m->stream));
  MCK(cudaMemsetAsync(m->m2, 0, sizeof(float) * kMlpNParam, m->stream));
  m->s_in = s_in;
  m->s_out = s_out;
  m->adam_step = 0;
  if ((rc = pack(m))) return rc;
  MCK(cudaStreamSynchronize(m->stream));
  return COUPLB_OK;
}

int couplb_mlp_get_weights(couplb_mlp* m, float* w, double* s_in, double* s_out) {
  if (!m) return COUPLB_ERR_ARG;
  int rc = set_dev(m);
  if (rc) return rc;
  if (w) {
    MCK(cudaMemcpyAsync(w, m->w, sizeof(float) * kMlpNParam, cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
  }
  if (s_in) *s_in = m->s_in;
  if (s_out) *s_out = m->s_out;
  return COUPLB_OK;
}

int couplb_mlp_fit_scales(couplb_mlp* m, const float* d_rows, long long n) {
  if (!m || !d_rows || n <= 0) return COUPLB_ERR_ARG;
  int rc = set_dev(m);
  if (rc) return rc;
  MCK(cudaMemsetAsync(m->d_acc, 0, sizeof(double) * 2 * kAccSlots, m->stream));
  k_mlp_scale_sums<<<296, 256, 0, m->stream>>>(d_rows, n, m->d_acc);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(m->h_acc, m->d_acc, sizeof(double) * 2 * kAccSlots, cudaMemcpyDeviceToHost, m->stream));
  MCK(cudaMemsetAsync(m->d_acc, 0, sizeof(double) * 2 * kAccSlots, m->stream));
  MCK(cudaStreamSynchronize(m->stream));
  double sx = 0.0, st = 0.0;
  for (int i = 0; i < kAccSlots; i++) { sx += m->h_acc[i]; st += m->h_acc[kAccSlots + i]; }
  const double rx = std::sqrt(sx / ((double)n * kMlpIn)), rt = std::sqrt(st / ((double)n * kMlpOut));
  m->s_in = rx > 0.0 ? 1.0 / rx : 1.0;
  m->s_out = rt > 0.0 ? 1.0 / rt : 1.0;
  if ((rc = pack(m))) return rc;
  MCK(cudaStreamSynchronize(m->stream));
  return COUPLB_OK;
}

int couplb_mlp_forward(couplb_mlp* m, const float* d_rows, long long n, float* d_out) {
  if (!m || !d_rows || !d_out || n < 0) return COUPLB_ERR_ARG;
  if (n == 0) return COUPLB_OK;
  int rc = set_dev(m);
  if (rc) return rc;
  TileArgs a{};
  a.rows = d_rows; a.base = 0; a.limit = n;
  a.w = m->w; a.s_in = (float)m->s_in; a.s_out = (float)m->s_out;
  a.out = d_out;
  return tile_launch(m, a, (n + kTile - 1) / kTile);
}

int couplb_mlp_loss_grad(couplb_mlp* m, const float* d_rows, long long n, double* loss,
                         float* grad) {
  if (!m || !d_rows || n <= 0) return COUPLB_ERR_ARG;
  int rc = set_dev(m);
  if (rc) return rc;
  MCK(cudaMemsetAsync(m->grad, 0, sizeof(float) * kMlpNParam, m->stream));
  MCK(cudaMemsetAsync(m->d_acc, 0, sizeof(double) * 2 * kAccSlots, m->stream));
  TileArgs a{};
  a.rows = d_rows; a.base = 0; a.limit = n;
  a.w = m->w; a.s_in = (float)m->s_in; a.s_out = (float)m->s_out;
  a.inv_norm = (float)(1.0 / (3.0 * (double)n));
  a.loss = m->d_acc;
  a.grad = m->grad;
  if ((rc = tile_launch(m, a, (n + kTile - 1) / kTile))) return rc;
  if (grad) MCK(cudaMemcpyAsync(grad, m->grad, sizeof(float) * kMlpNParam, cudaMemcpyDeviceToHost, m->stream));
  double l = 0.0;
  if ((rc = read_acc(m, kAccSlots, &l))) return rc;
  MCK(cudaMemsetAsync(m->grad, 0, sizeof(float) * kMlpNParam, m->stream));
  if (loss) *loss = l;
  return COUPLB_OK;
}

int couplb_mlp_train(couplb_mlp* m, const float* d_rows, long long n,
                     const couplb_mlp_train_params* tp, double* train_loss, double* val_loss) {
  if (!m || !d_rows || !tp) return COUPLB_ERR_ARG;
  const long long n_val = tp->n_val < 0 ? 0 : tp->n_val;
  const long long n_train = n - n_val;
  if (n_train < kTile || tp->epochs < 1 || tp->batch < kTile || tp->batch % kTile)
    return mfail(m, COUPLB_ERR_ARG, "need >= 64 training rows, epochs >= 1, batch a multiple of 64");
  if (!(tp->lr > 0.0) || tp->lr_final < 0.0 || !(tp->beta1 >= 0.0 && tp->beta1 < 1.0) ||
      !(tp->beta2 >= 0.0 && tp->beta2 < 1.0) || !(tp->eps > 0.0))
    return mfail(m, COUPLB_ERR_ARG, "bad Adam parameters");
  int rc = set_dev(m);
  if (rc) return rc;
  const long long spe = n_train / tp->batch > 0 ? n_train / tp->batch : 1;
  const long long total = spe * tp->epochs;
  TileArgs a{};
  a.rows = d_rows;
  a.random = 1;
  a.seed = tp->seed;
  a.n_pick = n_train;
  a.w = m->w; a.s_in = (float)m->s_in; a.s_out = (float)m->s_out;
  a.inv_norm = (float)(1.0 / (3.0 * (double)tp->batch));
  a.loss = m->d_acc + kAccSlots;   // running training loss (not read back per step)
  a.grad = m->grad;
  MCK(cudaFuncSetAttribute(k_mlp_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
  const double pi = 3.14159265358979323846;
  for (long long s = 0; s < total; s++) {
    a.step = s;
    k_mlp_tile<<<tp->batch / kTile, kThreads, kTileSmem, m->stream>>>(a);
    m->adam_step++;
    const double lr = tp->lr_final + 0.5 * (tp->lr - tp->lr_final) * (1.0 + std::cos(pi * (double)s / (double)total));
    const double c1 = 1.0 - std::pow(tp->beta1, (double)m->adam_step);
    const double c2 = 1.0 - std::pow(tp->beta2, (double)m->adam_step);
    k_mlp_adam<<<(kMlpNParam + 255) / 256, 256, 0, m->stream>>>(m->w, m->grad, m->m1, m->m2, (float)lr,
                                                                 (float)tp->beta1, (float)tp->beta2,
                                                                 (float)tp->eps, (float)c1, (float)c2);
  }
  MCK(cudaGetLastError());
  MCK(cudaMemsetAsync(m->d_acc, 0, sizeof(double) * 2 * kAccSlots, m->stream));
  double l = 0.0;
  if ((rc = eval_loss(m, d_rows, 0, n_train, &l))) return rc;
  if (train_loss) *train_loss = l;
  if ((rc = eval_loss(m, d_rows, n_train, n_val, &l))) return rc;
  if (val_loss) *val_loss = l;
  if ((rc = pack(m))) return rc;
  MCK(cudaStreamSynchronize(m->stream));
  return COUPLB_OK;
}

int couplb_mlp_save(couplb_mlp* m, const char* path) {
  if (!m || !path) return COUPLB_ERR_ARG;
  std::vector<float> w(kMlpNParam);
  double si, so;
  int rc = couplb_mlp_get_weights(m, w.data(), &si, &so);
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return mfail(m, COUPLB_ERR_IO, "cannot open %s for writing", path);
  bool ok = std::fwrite("CLBMLP01", 1, 8, f) == 8 && std::fwrite(&si, sizeof si, 1, f) == 1 &&
            std::fwrite(&so, sizeof so, 1, f) == 1 &&
            std::fwrite(w.data(), sizeof(float), kMlpNParam, f) == (size_t)kMlpNParam;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? COUPLB_OK : mfail(m, COUPLB_ERR_IO, "write error on %s", path);
}

int couplb_mlp_load(couplb_mlp* m, const char* path) {
  if (!m || !path) return COUPLB_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return mfail(m, COUPLB_ERR_IO, "cannot open %s", path);
  char magic[8];
  double si = 0, so = 0;
  std::vector<float> w(kMlpNParam);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "CLBMLP01", 8) == 0 &&
            std::fread(&si, sizeof si, 1, f) == 1 && std::fread(&so, sizeof so, 1, f) == 1 &&
            std::fread(w.data(), sizeof(float), kMlpNParam, f) == (size_t)kMlpNParam;
  char extra;
  ok = ok && std::fread(&extra, 1, 1, f) == 0;
  std::fclose(f);
  if (!ok) return mfail(m, COUPLB_ERR_IO, "%s is not a network file of this build", path);
  for (float v : w)
    if (!std::isfinite(v)) return mfail(m, COUPLB_ERR_IO, "%s holds non-finite weights", path);
  return couplb_mlp_set_weights(m, w.data(), si, so);
}

}  // extern "C"
