// engine_common.cuh -- helpers shared by the translation units of the lattice
// engine (engine.cu: lattice, LB step, moments, I/O; engine_ibm.cu: the
// immersed-boundary sub-steps).  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/couplb_b200.h"
#include "engine_internal.h"
#include "ibm_kernels.cuh"
#include "ibm_methods.cuh"
#include "lbm_kernels.cuh"

namespace couplb {
namespace eng {

inline thread_local std::string g_create_error;

inline int fail(couplb_handle* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  else g_create_error = buf;
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(h, COUPLB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define CK_LAUNCH()                                                                \
  do {                                                                             \
    cudaError_t e_ = cudaGetLastError();                                           \
    if (e_ != cudaSuccess)                                                         \
      return fail(h, COUPLB_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_)); \
  } while (0)

template <class Fn>
void with_types(int dim, int prec, Fn&& fn) {
  if (dim == 3) {
    if (prec == COUPLB_FP64) fn(D3Q19{}, StoreF64{});
    else if (prec == COUPLB_FP32_SHIFTED) fn(D3Q19{}, StoreF32S{});
    else fn(D3Q19{}, StoreF16S{});
  } else {
    if (prec == COUPLB_FP64) fn(D2Q9{}, StoreF64{});
    else if (prec == COUPLB_FP32_SHIFTED) fn(D2Q9{}, StoreF32S{});
    else fn(D2Q9{}, StoreF16S{});
  }
}

inline size_t elem_bytes_pop(int prec) { return prec == COUPLB_FP64 ? 8 : (prec == COUPLB_FP32_SHIFTED ? 4 : 2); }
inline size_t elem_bytes_aux(int prec) { return prec == COUPLB_FP64 ? 8 : 4; }

inline Geom make_geom(const couplb_handle* h) {
  Geom g;
  g.nx = h->p.nx; g.ny = h->p.ny; g.nz = h->p.nz;
  g.qs = (long long)h->qs;
  for (int f = 0; f < 6; f++) g.face[f] = h->p.wall[f];
  if (h->p.dim == 2) g.face[4] = g.face[5] = 0;
  for (int d = 0; d < 3; d++) g.uw[d] = h->p.wall_vel[d];
  if (h->p.dim == 2) g.uw[2] = 0.0;
  g.rho0 = h->p.rho0;
  g.halo[0] = h->halo[0];
  g.halo[1] = h->halo[1];
  return g;
}

inline void row_launch(const couplb_handle* h, dim3* grid, dim3* block) {
  const int bx = std::min(256, ((h->p.nx + 31) / 32) * 32);
  *block = dim3(bx, 1, 1);
  *grid = dim3((h->p.nx + bx - 1) / bx, h->p.ny, h->p.nz);
}

inline unsigned flat_blocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Force flags: one byte per 8 consecutive interior nodes (n >> 3).
inline size_t seg_bytes(const couplb_handle* h) { return (h->N + 7) / 8; }

inline int dalloc(couplb_handle* h, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess)
    return fail(h, COUPLB_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  h->device_bytes += bytes;
  return COUPLB_OK;
}

inline void dfree(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

inline int ensure_macro(couplb_handle* h) {
  if (h->macro[0]) return COUPLB_OK;
  const size_t b = h->qs * elem_bytes_aux(h->p.precision);
  for (int c = 0; c < 4; c++) {
    int rc = dalloc(h, &h->macro[c], b);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->macro[c], 0, b, h->stream));
  }
  return COUPLB_OK;
}

inline int ensure_staging(couplb_handle* h, size_t bytes) {
  if (h->staging_bytes >= bytes) return COUPLB_OK;
  dfree(h->d_staging);
  h->staging_bytes = 0;
  int rc = dalloc(h, &h->d_staging, bytes);
  if (rc) return rc;
  h->staging_bytes = bytes;
  return COUPLB_OK;
}

// Stencil velocity records of the IBM sub-step, one per marker slot
// (StencilKey + 64 x {ux, uy, uz, rho}).  Keys start with epoch 0xffffffff, which
// cur_epoch never takes, so a fresh record never hits.
inline int ensure_stencil_cache(couplb_handle* h, int n) {
  if (h->stencil_cap >= n) return COUPLB_OK;
  dfree(h->sbuf);
  void* k = h->skey;
  dfree(k);
  h->skey = nullptr;
  h->stencil_cap = 0;
  const int cap = std::max(n, 1024);
  int rc;
  if ((rc = dalloc(h, &h->sbuf, elem_bytes_aux(h->p.precision) * kRecStride * (size_t)cap))) return rc;
  if ((rc = dalloc(h, (void**)&h->skey, sizeof(couplb::StencilKey) * (size_t)cap))) return rc;
  CK(cudaMemsetAsync(h->skey, 0xff, sizeof(couplb::StencilKey) * (size_t)cap, h->stream));
  h->stencil_cap = cap;
  return COUPLB_OK;
}

// The population state changed: every cached stencil velocity is stale.
inline void bump_epoch(couplb_handle* h) {
  if (++h->cur_epoch == 0xffffffffu) {
    h->cur_epoch = 0;
    if (h->skey) cudaMemsetAsync(h->skey, 0xff, sizeof(couplb::StencilKey) * (size_t)h->stencil_cap, h->stream);
  }
}

// Per-marker buffers of the correction passes and their state block.
inline int ensure_method_buffers(couplb_handle* h, int n) {
  if (!h->d_pass) {
    int rc = dalloc(h, &h->d_pass, 2 * sizeof(PassState));
    if (rc) return rc;
    CK(cudaMemsetAsync(h->d_pass, 0, 2 * sizeof(PassState), h->stream));
    h->pass_cur = 0;
  }
  if (h->method_cap >= n) return COUPLB_OK;
  void* p = h->d_corr; dfree(p); h->d_corr = nullptr;
  p = h->d_dF; dfree(p); h->d_dF = nullptr;
  h->method_cap = 0;
  const int cap = std::max(n, 1024);
  int rc;
  if ((rc = dalloc(h, (void**)&h->d_corr, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, (void**)&h->d_dF, sizeof(double) * 3 * cap))) return rc;
  h->method_cap = cap;
  return COUPLB_OK;
}

inline int ensure_atoms(couplb_handle* h, int n) {
  if (h->atom_cap >= n) return COUPLB_OK;
  dfree(h->d_x); dfree(h->d_v); dfree(h->d_m); dfree(h->d_fout); dfree(h->d_active);
  if (h->h_fout) { cudaFreeHost(h->h_fout); h->h_fout = nullptr; }
  if (h->h_mass) { cudaFreeHost(h->h_mass); h->h_mass = nullptr; }
  if (h->h_active) { cudaFreeHost(h->h_active); h->h_active = nullptr; }
  const int cap = std::max(n, 1024);
  int rc;
  if ((rc = dalloc(h, &h->d_x, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_v, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_m, sizeof(double) * cap))) return rc;
  if ((rc = dalloc(h, &h->d_fout, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_active, sizeof(int) * cap))) return rc;
  CK(cudaMallocHost(&h->h_fout, sizeof(double) * 3 * cap));
  CK(cudaMallocHost(&h->h_mass, sizeof(double) * cap));
  CK(cudaMallocHost(&h->h_active, sizeof(int) * cap));
  h->atom_cap = cap;
  h->statics_n = -1;
  return COUPLB_OK;
}

inline int set_device(couplb_handle* h) {
  CK(cudaSetDevice(h->p.device));
  return COUPLB_OK;
}

}  // namespace eng
}  // namespace couplb
