// mlp.cu -- training and inference kernels of the 84-64-64-3 no-slip
// correction network, and its C ABI (couplb_mlp_*).
//
// Training runs on the GPU with the project's own kernels: one block of 256
// threads takes a tile of 64 rows, keeps the BF16-rounded weights, the inputs
// and every activation of the tile in shared memory (113 KB), runs the forward
// pass, the squared-error loss and the backward pass, and adds its partial
// gradient to an FP32 accumulator with atomics; a second kernel applies Adam
// to the FP32 master weights.  At these sizes (9795 parameters, 64-wide
// layers) a step is latency-bound, so the contractions stay on the FP32 pipe.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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
constexpr int kP1 = kMlpIn + 1;    // padded shared-memory row strides
constexpr int kP2 = kMlpHid + 1;
constexpr int kTileFloats = kMlpHid * kP1 + kMlpHid * kP2 + kMlpOut * kMlpHid + 2 * kMlpHid + 4 +
                            kTile * kP1 + 3 * kTile * kP2 + 2 * kTile * kMlpOut + 32;
constexpr size_t kTileSmem = sizeof(float) * kTileFloats;
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

__global__ void __launch_bounds__(kThreads) k_mlp_tile(const TileArgs A) {
  extern __shared__ float sm[];
  float* W1 = sm;
  float* W2 = W1 + kMlpHid * kP1;
  float* W3 = W2 + kMlpHid * kP2;
  float* B1 = W3 + kMlpOut * kMlpHid;
  float* B2 = B1 + kMlpHid;
  float* B3 = B2 + kMlpHid;
  float* X = B3 + 4;
  float* H1 = X + kTile * kP1;
  float* H2 = H1 + kTile * kP2;
  float* D2 = H2 + kTile * kP2;
  float* Y = D2 + kTile * kP2;
  float* T = Y + kTile * kMlpOut;
  float* RED = T + kTile * kMlpOut;
  __shared__ long long idx[kTile];
  const int t = threadIdx.x;

  for (int e = t; e < kMlpHid * kMlpIn; e += kThreads)
    W1[(e / kMlpIn) * kP1 + e % kMlpIn] = bf16_round(A.w[kMlpW1 + e]);
  for (int e = t; e < kMlpHid * kMlpHid; e += kThreads)
    W2[(e / kMlpHid) * kP2 + e % kMlpHid] = bf16_round(A.w[kMlpW2 + e]);
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
  for (int e = t; e < kTile * (kMlpIn + kMlpOut); e += kThreads) {
    const int s = e / (kMlpIn + kMlpOut), k = e % (kMlpIn + kMlpOut);
    const long long r = idx[s];
    const float v = r >= 0 ? __ldg(A.rows + r * kMlpRow + k) : 0.f;
    if (k < kMlpIn) X[s * kP1 + k] = v * A.s_in;
    else T[s * kMlpOut + k - kMlpIn] = v;
  }
  __syncthreads();

  // forward
  for (int e = t; e < kTile * kMlpHid; e += kThreads) {
    const int s = e / kMlpHid, j = e % kMlpHid;
    const float* wr = W1 + j * kP1;
    const float* xr = X + s * kP1;
    float a = B1[j];
#pragma unroll 4
    for (int k = 0; k < kMlpIn; k++) a = fmaf(wr[k], xr[k], a);
    H1[s * kP2 + j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int e = t; e < kTile * kMlpHid; e += kThreads) {
    const int s = e / kMlpHid, j = e % kMlpHid;
    const float* wr = W2 + j * kP2;
    const float* hr = H1 + s * kP2;
    float a = B2[j];
#pragma unroll 4
    for (int k = 0; k < kMlpHid; k++) a = fmaf(wr[k], hr[k], a);
    H2[s * kP2 + j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  if (t < kTile * kMlpOut) {
    const int s = t / kMlpOut, c = t % kMlpOut;
    const float* wr = W3 + c * kMlpHid;
    const float* hr = H2 + s * kP2;
    float a = B3[c];
#pragma unroll 4
    for (int k = 0; k < kMlpHid; k++) a = fmaf(wr[k], hr[k], a);
    Y[t] = a;
    if (A.out && idx[s] >= 0) A.out[idx[s] * kMlpOut + c] = a / A.s_out;
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
    double s = 0.0;
    for (int i = 0; i < kThreads / 32; i++) s += RED[i];
    atomicAdd(A.loss + (blockIdx.x & (kAccSlots - 1)), s);
  }
  if (!A.grad) return;

  // backward: layer 3, then delta2 = (W3^T dy) * relu'(h2)
  if (t < kMlpOut * kMlpHid) {
    const int c = t / kMlpHid, k = t % kMlpHid;
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a = fmaf(Y[s * kMlpOut + c], H2[s * kP2 + k], a);
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
    if (H2[s * kP2 + k] > 0.f)
      for (int c = 0; c < kMlpOut; c++) a = fmaf(W3[c * kMlpHid + k], Y[s * kMlpOut + c], a);
    D2[s * kP2 + k] = a;
  }
  __syncthreads();
  // layer 2 gradient, and delta1 = (W2^T delta2) * relu'(h1) into H2
  for (int e = t; e < kMlpHid * kMlpHid; e += kThreads) {
    const int j = e / kMlpHid, k = e % kMlpHid;
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a = fmaf(D2[s * kP2 + j], H1[s * kP2 + k], a);
    atomicAdd(A.grad + kMlpW2 + e, a);
  }
  if (t < kMlpHid) {
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a += D2[s * kP2 + t];
    atomicAdd(A.grad + kMlpB2 + t, a);
  }
  for (int e = t; e < kTile * kMlpHid; e += kThreads) {
    const int s = e / kMlpHid, k = e % kMlpHid;
    float a = 0.f;
    if (H1[s * kP2 + k] > 0.f) {
      const float* dr = D2 + s * kP2;
#pragma unroll 4
      for (int j = 0; j < kMlpHid; j++) a = fmaf(W2[j * kP2 + k], dr[j], a);
    }
    H2[s * kP2 + k] = a;
  }
  __syncthreads();
  // layer 1 gradient
  for (int e = t; e < kMlpHid * kMlpIn; e += kThreads) {
    const int j = e / kMlpIn, k = e % kMlpIn;
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a = fmaf(H2[s * kP2 + j], X[s * kP1 + k], a);
    atomicAdd(A.grad + kMlpW1 + e, a);
  }
  if (t < kMlpHid) {
    float a = 0.f;
    for (int s = 0; s < kTile; s++) a += H2[s * kP2 + t];
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
