// noalloc.cu -- allocation-free variant of the stability-diagnostics
// reduction (max |u|, total mass, total momentum).
//
// Some callers cannot let a library call cudaMalloc: an MD code that owns all
// device memory through its own pool allocator (a stray cudaMalloc fragments
// the pool and cudaFree synchronises the whole device), or a time loop that
// must not stall on the implicit device synchronisation of an allocation.
// couplb_diagnostics() allocates its reduction scratch lazily on the handle;
// couplb_diagnostics_noalloc() takes caller-owned inputs and outputs and
// keeps its scratch in a fixed-size array in device global memory instead, so
// it never allocates.
//
// Scratch: g_diag_scratch below, COUPLB_NOALLOC_MAX_PARTIALS * 5 doubles
// (1.25 MiB), held by every GPU that loads this library until the process
// exits.  One block reduces COUPLB_NOALLOC_CHUNK consecutive nodes into one
// 5-double slot, so a call handles at most
// COUPLB_NOALLOC_MAX_PARTIALS * COUPLB_NOALLOC_CHUNK nodes.  Every slot a call
// reads is written earlier in the same call, so nothing in the scratch has to
// start at zero; but all calls share the one array, so calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.
//
// Unlike couplb_diagnostics, which follows the reference's max_velocity
// (std::max drops a NaN speed, and non-finite densities are counted in the
// status word instead), the maximum here propagates NaN: this entry point
// returns no non-finite count, so a caller watching max |u| for stability
// sees NaN as soon as one node's velocity is NaN.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/couplb_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// max that keeps a NaN of either argument (fmax and a plain comparison drop it)
__device__ __forceinline__ double max_keep_nan(double a, double b) {
  if (a != a) return a;
  return (b != b || b > a) ? b : a;
}

static __device__ __align__(256) double g_diag_scratch[COUPLB_NOALLOC_MAX_PARTIALS * 5];

// Per-device device address of g_diag_scratch.  In host code the name
// g_diag_scratch is only a host-side stand-in for the symbol, not a device
// address, so it is never passed to a kernel; the address is looked up with
// cudaGetSymbolAddress once per device, with that device current.
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_address(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_diag_scratch) != cudaSuccess || !p) return COUPLB_ERR_CUDA;
    g_scratch_addr[device] = p;
  }
  *out = static_cast<double*>(g_scratch_addr[device]);
  return COUPLB_OK;
}

// One block reduces nodes [b*CHUNK, min((b+1)*CHUNK, n)) into slot b.
template <class A, bool kShift>
__global__ void __launch_bounds__(kThreads) k_diag_chunks(long long n, double rho0,
                                                          const A* __restrict__ rho,
                                                          const A* __restrict__ ux,
                                                          const A* __restrict__ uy,
                                                          const A* __restrict__ uz,
                                                          double* __restrict__ part) {
  const long long lo = (long long)blockIdx.x * COUPLB_NOALLOC_CHUNK;
  const long long hi = lo + COUPLB_NOALLOC_CHUNK < n ? lo + COUPLB_NOALLOC_CHUNK : n;
  double m2 = 0, sm = 0, px = 0, py = 0, pz = 0;
  for (long long i = lo + threadIdx.x; i < hi; i += kThreads) {
    double r = double(rho[i]);
    if (kShift) r += rho0;
    const double a = double(ux[i]), b = double(uy[i]), c = double(uz[i]);
    const double u2 = a * a + b * b + c * c;
    m2 = max_keep_nan(m2, u2);
    sm += r;
    px += r * a; py += r * b; pz += r * c;
  }
  __shared__ double sh[5][kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m2 = max_keep_nan(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
    px += __shfl_xor_sync(0xffffffffu, px, o);
    py += __shfl_xor_sync(0xffffffffu, py, o);
    pz += __shfl_xor_sync(0xffffffffu, pz, o);
  }
  if (lane == 0) { sh[0][wid] = m2; sh[1][wid] = sm; sh[2][wid] = px; sh[3][wid] = py; sh[4][wid] = pz; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double o[5] = {0, 0, 0, 0, 0};
    for (int w = 0; w < kThreads / 32; w++) {
      o[0] = max_keep_nan(o[0], sh[0][w]);
      for (int c = 1; c < 5; c++) o[c] += sh[c][w];
    }
    for (int c = 0; c < 5; c++) part[blockIdx.x * 5 + c] = o[c];
  }
}

// One block sums the slots: thread t takes slots t, t + 256, ... in slot
// order, then a fixed-shape shared-memory tree combines the 256 partials, so
// the result does not depend on scheduling.
__global__ void __launch_bounds__(kThreads) k_diag_finish(int nparts, const double* __restrict__ part,
                                                          double* __restrict__ out) {
  double o[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nparts; b += kThreads) {
    o[0] = max_keep_nan(o[0], part[b * 5]);
    for (int c = 1; c < 5; c++) o[c] += part[b * 5 + c];
  }
  __shared__ double sh[5][kThreads];
  for (int c = 0; c < 5; c++) sh[c][threadIdx.x] = o[c];
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sh[0][threadIdx.x] = max_keep_nan(sh[0][threadIdx.x], sh[0][threadIdx.x + h]);
      for (int c = 1; c < 5; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sqrt(sh[0][0]);
    for (int c = 1; c < 5; c++) out[c] = sh[c][0];
  }
}

}  // namespace

extern "C" int couplb_diagnostics_noalloc(const void* d_rho, const void* d_ux, const void* d_uy,
                                          const void* d_uz, long long n, int precision, double rho0,
                                          double* d_out, void* stream) {
  if (!d_rho || !d_ux || !d_uy || !d_uz || !d_out || n <= 0) return COUPLB_ERR_ARG;
  if (precision != COUPLB_FP64 && precision != COUPLB_FP32_SHIFTED && precision != COUPLB_FP16_SHIFTED)
    return COUPLB_ERR_ARG;
  if (n > COUPLB_NOALLOC_MAX_NODES) return COUPLB_ERR_TOO_LARGE;
  const long long nparts = (n + COUPLB_NOALLOC_CHUNK - 1) / COUPLB_NOALLOC_CHUNK;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return COUPLB_ERR_CUDA;
  double* part = nullptr;
  int rc = scratch_address(device, &part);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == COUPLB_FP64)
    k_diag_chunks<double, false><<<(unsigned)nparts, kThreads, 0, s>>>(
        n, rho0, (const double*)d_rho, (const double*)d_ux, (const double*)d_uy, (const double*)d_uz, part);
  else
    k_diag_chunks<float, true><<<(unsigned)nparts, kThreads, 0, s>>>(
        n, rho0, (const float*)d_rho, (const float*)d_ux, (const float*)d_uy, (const float*)d_uz, part);
  if (cudaGetLastError() != cudaSuccess) return COUPLB_ERR_CUDA;
  k_diag_finish<<<1, kThreads, 0, s>>>((int)nparts, part, d_out);
  if (cudaGetLastError() != cudaSuccess) return COUPLB_ERR_CUDA;
  return COUPLB_OK;
}
