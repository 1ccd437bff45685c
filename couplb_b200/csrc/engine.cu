// engine.cu -- layer 1 of the C ABI (include/couplb_b200.h): one handle per
// LBM subdomain, all state resident in device memory, kernels on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/couplb_b200.h"
#include "engine_internal.h"
#include "ibm_kernels.cuh"
#include "ibm_methods.cuh"
#include "lbm_kernels.cuh"
#include "lbm_packed.cuh"
#include "mlp_internal.h"

using namespace couplb;

namespace {

thread_local std::string g_create_error;

int fail(couplb_handle* h, int code, const char* fmt, ...) {
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

// Copy of the status word (clamp and non-finite counts) into a posted slot of
// mapped pinned host memory; read by the host after the slot's event.
__global__ void k_status_publish(const int* __restrict__ st, int* ring_slot) {
  if (threadIdx.x < 2) ring_slot[threadIdx.x] = st[threadIdx.x];
}

size_t elem_bytes_pop(int prec) { return prec == COUPLB_FP64 ? 8 : (prec == COUPLB_FP32_SHIFTED ? 4 : 2); }
size_t elem_bytes_aux(int prec) { return prec == COUPLB_FP64 ? 8 : 4; }

Geom make_geom(const couplb_handle* h) {
  Geom g;
  g.nx = h->p.nx; g.ny = h->p.ny; g.nz = h->p.nz;
  g.qs = (long long)h->qs;
  for (int f = 0; f < 6; f++) g.face[f] = h->p.wall[f];
  if (h->p.dim == 2) g.face[4] = g.face[5] = 0;
  for (int d = 0; d < 3; d++) g.uw[d] = h->p.wall_vel[d];
  if (h->p.dim == 2) g.uw[2] = 0.0;
  g.rho0 = h->p.rho0;
  return g;
}

void row_launch(const couplb_handle* h, dim3* grid, dim3* block) {
  const int bx = std::min(256, ((h->p.nx + 31) / 32) * 32);
  *block = dim3(bx, 1, 1);
  *grid = dim3((h->p.nx + bx - 1) / bx, h->p.ny, h->p.nz);
}

unsigned flat_blocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Force flags: one byte per 8 consecutive interior nodes (n >> 3).
size_t seg_bytes(const couplb_handle* h) { return (h->N + 7) / 8; }

int dalloc(couplb_handle* h, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess)
    return fail(h, COUPLB_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  h->device_bytes += bytes;
  return COUPLB_OK;
}

void dfree(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int ensure_macro(couplb_handle* h) {
  if (h->macro[0]) return COUPLB_OK;
  const size_t b = h->qs * elem_bytes_aux(h->p.precision);
  for (int c = 0; c < 4; c++) {
    int rc = dalloc(h, &h->macro[c], b);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->macro[c], 0, b, h->stream));
  }
  return COUPLB_OK;
}

int ensure_staging(couplb_handle* h, size_t bytes) {
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
int ensure_stencil_cache(couplb_handle* h, int n) {
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
void bump_epoch(couplb_handle* h) {
  if (++h->cur_epoch == 0xffffffffu) {
    h->cur_epoch = 0;
    if (h->skey) cudaMemsetAsync(h->skey, 0xff, sizeof(couplb::StencilKey) * (size_t)h->stencil_cap, h->stream);
  }
}

// Per-marker buffers of the correction passes and their state block.
int ensure_method_buffers(couplb_handle* h, int n) {
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

int ensure_atoms(couplb_handle* h, int n) {
  if (h->atom_cap >= n) return COUPLB_OK;
  dfree(h->d_x); dfree(h->d_v); dfree(h->d_m); dfree(h->d_fout); dfree(h->d_active);
  if (h->h_fout) { cudaFreeHost(h->h_fout); h->h_fout = nullptr; }
  const int cap = std::max(n, 1024);
  int rc;
  if ((rc = dalloc(h, &h->d_x, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_v, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_m, sizeof(double) * cap))) return rc;
  if ((rc = dalloc(h, &h->d_fout, sizeof(double) * 3 * cap))) return rc;
  if ((rc = dalloc(h, &h->d_active, sizeof(int) * cap))) return rc;
  CK(cudaMallocHost(&h->h_fout, sizeof(double) * 3 * cap));
  h->atom_cap = cap;
  return COUPLB_OK;
}

int set_device(couplb_handle* h) {
  CK(cudaSetDevice(h->p.device));
  return COUPLB_OK;
}

// Launch of the bulk-copy staged fused kernel: returns false (nothing
// launched) when the row layout does not meet the copy alignment rules or the
// stages do not fit in shared memory, so the caller uses the plain kernel.
template <class L, class S, int STAGES>
bool launch_staged(couplb_handle* h, const LBArgs<S>& a) {
  using T = typename S::T;
  const size_t row_bytes = (size_t)h->p.nx * sizeof(T);
  if (row_bytes % 16 != 0 || (h->qs * sizeof(T)) % 16 != 0) return false;
  if (h->p.wall[0] != 0 || h->p.wall[1] != 0) return false;   // no interior rows
  const size_t smem = (size_t)STAGES * L::Q * row_bytes;
  if (smem > 200 * 1024) return false;
  static bool configured = false;   // per template instance
  auto kern = k_stream_collide_tma<L, S, STAGES>;
  if (!configured) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return false;
    configured = true;
  } else {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  const int threads = std::min(256, ((h->p.nx + 31) / 32) * 32);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
    return false;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->p.device);
  const long long rows = (long long)h->p.ny * h->p.nz;
  const int grid = (int)std::min<long long>(rows, (long long)sms * per_sm);
  kern<<<grid, threads, smem, h->stream>>>(a);
  return true;
}

// Populations as post-stream state in buffer `cur` (materialise if needed).
int materialize(couplb_handle* h) {
  if (h->poststream) return COUPLB_OK;
  dim3 grid, block;
  row_launch(h, &grid, &block);
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using T = typename S::T;
    k_materialize<L, S><<<grid, block, 0, h->stream>>>(g, (const T*)h->f[h->cur],
                                                       (const typename S::A*)h->rho_field,
                                                       (T*)h->f[1 - h->cur]);
  });
  CK_LAUNCH();
  h->cur = 1 - h->cur;
  h->poststream = 1;
  return COUPLB_OK;
}

}  // namespace

// ===========================================================================
// internal entry points shared with the fix core and the profile writer
namespace couplb {

int engine_macro(couplb_handle* h) {
  int rc = ensure_macro(h);
  if (rc) return rc;
  CK(cudaMemsetAsync(h->d_status + kStMacroClamps, 0, sizeof(int), h->stream));
  dim3 grid, block;
  row_launch(h, &grid, &block);
  const Geom g = make_geom(h);
  const bool pull = !h->poststream;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using T = typename S::T;
    using A = typename S::A;
    MacroArgs<S> a;
    a.g = g;
    a.fin = (const T*)h->f[h->cur];
    a.rho_field = (const A*)h->rho_field;
    a.rho = (A*)h->macro[0]; a.ux = (A*)h->macro[1]; a.uy = (A*)h->macro[2]; a.uz = (A*)h->macro[3];
    a.status = h->d_status;
    if (pull) k_macro<L, S, true><<<grid, block, 0, h->stream>>>(a);
    else k_macro<L, S, false><<<grid, block, 0, h->stream>>>(a);
  });
  CK_LAUNCH();
  h->macro_valid = 1;
  if (h->p.body_force) h->rho_state = kRhoCurrent;
  return COUPLB_OK;
}

}  // namespace couplb

// ===========================================================================
extern "C" {

int couplb_version(void) { return COUPLB_ABI_VERSION; }

size_t couplb_struct_size(int which) {
  switch (which) {
    case 0: return sizeof(couplb_lattice_params);
    case 1: return sizeof(couplb_ibm_params);
    case 2: return sizeof(couplb_diag);
    case 3: return sizeof(couplb_fix_config);
    case 4: return sizeof(couplb_domain);
    case 5: return sizeof(couplb_atoms);
    case 6: return sizeof(couplb_ibm_method);
    case 7: return sizeof(couplb_mlp_train_params);
    default: return 0;
  }
}

const char* couplb_last_error(const couplb_handle* h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

int couplb_create(const couplb_lattice_params* p, couplb_handle** out) {
  couplb_handle* h = nullptr;
  if (!p || !out) return fail(nullptr, COUPLB_ERR_ARG, "couplb_create: null argument");
  *out = nullptr;
  if (p->dim != 2 && p->dim != 3) return fail(nullptr, COUPLB_ERR_ARG, "dim must be 2 or 3");
  if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return fail(nullptr, COUPLB_ERR_ARG, "grid dimensions must be positive");
  if (p->dim == 2 && p->nz != 1) return fail(nullptr, COUPLB_ERR_ARG, "nz must be 1 for dim 2");
  if (!(p->tau > 0.5) || !std::isfinite(p->tau)) return fail(nullptr, COUPLB_ERR_ARG, "tau <= 0.5 (unstable)");
  if (!(p->rho0 > 0.0) || !std::isfinite(p->rho0)) return fail(nullptr, COUPLB_ERR_ARG, "rho0 must be positive");
  for (int f = 0; f < 6; f++)
    if (p->wall[f] < 0 || p->wall[f] > 4) return fail(nullptr, COUPLB_ERR_ARG, "wall types must be in [0,4]");
  if (p->precision < COUPLB_FP64 || p->precision > COUPLB_FP16_SHIFTED)
    return fail(nullptr, COUPLB_ERR_ARG, "unknown precision %d", p->precision);
  const long long N = (long long)p->nx * p->ny * p->nz;
  const int Q = p->dim == 3 ? 19 : 9;
  if (N * Q >= (1LL << 40)) return fail(nullptr, COUPLB_ERR_ARG, "grid too large");

  h = new couplb_handle();
  h->p = *p;
  h->Q = Q;
  h->N = (size_t)N;
  h->qs = ((size_t)N + 63) / 64 * 64;
  {
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) {
      delete h;
      return fail(nullptr, COUPLB_ERR_CUDA, "cudaSetDevice(%d) failed: %s", p->device, cudaGetErrorString(e));
    }
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete h;
      return fail(nullptr, COUPLB_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
    }
    h->own_stream = true;
  }
  const size_t pb = elem_bytes_pop(p->precision), ab = elem_bytes_aux(p->precision);
  int rc = COUPLB_OK;
  for (int b = 0; b < 2 && !rc; b++) rc = dalloc(h, &h->f[b], pb * Q * h->qs);
  if (!rc) rc = dalloc(h, &h->F, 4 * ab * h->qs);
  h->moving_walls = false;
  for (int f = 0; f < (p->dim == 3 ? 6 : 4); f++) h->moving_walls |= (p->wall[f] == 2);
  if (!rc && (p->body_force || h->moving_walls)) rc = dalloc(h, &h->rho_field, ab * h->qs);
  h->idx32 = ((unsigned long long)Q * h->qs < (1ULL << 32));
  if (!rc) rc = dalloc(h, (void**)&h->d_status, sizeof(int) * 8);
  if (!rc) rc = dalloc(h, (void**)&h->d_ftot, sizeof(double) * 4 * kFtotSlots);
  if (!rc) rc = dalloc(h, (void**)&h->seg_force, seg_bytes(h));
  static_assert(sizeof(double) * 4 * kFtotSlots <= 4096, "h_small holds the force accumulators");
  if (!rc && cudaMallocHost(&h->h_small, 4096) != cudaSuccess)
    rc = fail(h, COUPLB_ERR_CUDA, "cudaMallocHost failed");
  // mapped, so that status_post publishes with a one-warp kernel instead of a
  // copy-engine transfer (a small D2H copy on the stream left a gap of ~10 us
  // before the next step's kernel)
  if (!rc && cudaHostAlloc((void**)&h->h_status_ring, sizeof(int) * 16, cudaHostAllocMapped) != cudaSuccess)
    rc = fail(h, COUPLB_ERR_CUDA, "cudaHostAlloc failed");
  if (!rc && cudaHostGetDevicePointer((void**)&h->d_status_ring, h->h_status_ring, 0) != cudaSuccess)
    rc = fail(h, COUPLB_ERR_CUDA, "cudaHostGetDevicePointer failed");
  for (int e = 0; e < 2 && !rc; e++)
    if (cudaEventCreateWithFlags(&h->status_ev[e], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(h, COUPLB_ERR_CUDA, "cudaEventCreate failed");
  if (rc) {
    g_create_error = h->err;
    couplb_destroy(h);
    return rc;
  }
  if (!rc && cudaMemsetAsync(h->F, 0, 4 * ab * h->qs, h->stream) != cudaSuccess) rc = COUPLB_ERR_CUDA;
  if (!rc && cudaMemsetAsync(h->d_status, 0, sizeof(int) * 8, h->stream) != cudaSuccess) rc = COUPLB_ERR_CUDA;
  if (!rc && cudaMemsetAsync(h->d_ftot, 0, sizeof(double) * 4 * kFtotSlots, h->stream) != cudaSuccess)
    rc = COUPLB_ERR_CUDA;
  if (!rc) rc = couplb_init_equilibrium(h, p->rho0, 0.0, 0.0, 0.0);
  if (rc) {
    g_create_error = h->err.empty() ? "device initialisation failed" : h->err;
    couplb_destroy(h);
    return rc ? rc : COUPLB_ERR_CUDA;
  }
  *out = h;
  return COUPLB_OK;
}

int couplb_destroy(couplb_handle* h) {
  if (!h) return COUPLB_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int b = 0; b < 2; b++) dfree(h->f[b]);
  dfree(h->F);
  for (int c = 0; c < 4; c++) dfree(h->macro[c]);
  dfree(h->rho_field);
  void* p = h->d_status; dfree(p);
  p = h->seg_force; dfree(p);
  p = h->skey; dfree(p);
  dfree(h->sbuf);
  p = h->d_ftot; dfree(p);
  p = h->d_corr; dfree(p);
  p = h->d_dF; dfree(p);
  dfree(h->d_pass);
  dfree(h->d_staging);
  dfree(h->d_scratch);
  dfree(h->d_x); dfree(h->d_v); dfree(h->d_m); dfree(h->d_fout); dfree(h->d_active);
  if (h->h_fout) cudaFreeHost(h->h_fout);
  if (h->h_small) cudaFreeHost(h->h_small);
  if (h->h_status_ring) cudaFreeHost(h->h_status_ring);
  for (int e = 0; e < 2; e++)
    if (h->status_ev[e]) cudaEventDestroy(h->status_ev[e]);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return COUPLB_OK;
}

int couplb_set_stream(couplb_handle* h, void* s) {
  if (!h) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->stream = (cudaStream_t)s;
  h->own_stream = false;
  return COUPLB_OK;
}

int couplb_synchronize(couplb_handle* h) {
  if (!h) return COUPLB_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

size_t couplb_ghost_nodes(const couplb_handle* h) {
  if (!h) return 0;
  return (size_t)(h->p.nx + 2) * (h->p.ny + 2) * (h->p.dim == 3 ? h->p.nz + 2 : 1);
}

size_t couplb_device_bytes(const couplb_handle* h) { return h ? h->device_bytes : 0; }

int couplb_init_equilibrium(couplb_handle* h, double rho, double ux, double uy, double uz) {
  if (!h) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  const Geom g = make_geom(h);
  const long long N = (long long)h->N;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    k_init_eq<L, S><<<flat_blocks(N, 256), 256, 0, h->stream>>>(
        g, (typename S::T*)h->f[0], rho, ux, uy, h->p.dim == 3 ? uz : 0.0,
        (typename S::A*)h->rho_field);
  });
  CK_LAUNCH();
  h->cur = 0;
  h->poststream = 1;
  const size_t ab = elem_bytes_aux(h->p.precision);
  CK(cudaMemsetAsync(h->F, 0, 4 * ab * h->qs, h->stream));
  CK(cudaMemsetAsync(h->seg_force, 0, seg_bytes(h), h->stream));
  h->force_dirty = 0;
  h->force_rows_all = 0;
  h->rho_state = h->p.body_force ? kRhoField : kRhoNone;
  h->macro_valid = 0;
  bump_epoch(h);
  return COUPLB_OK;
}

int couplb_set_populations(couplb_handle* h, const double* f_host) {
  if (!h || !f_host) return fail(h, COUPLB_ERR_ARG, "null argument");
  int rc = set_device(h);
  if (rc) return rc;
  const size_t G = couplb_ghost_nodes(h);
  const size_t bytes = sizeof(double) * h->Q * G;
  if ((rc = ensure_staging(h, bytes))) return rc;
  CK(cudaMemcpyAsync(h->d_staging, f_host, bytes, cudaMemcpyHostToDevice, h->stream));
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    k_import_f<L, S><<<flat_blocks((long long)h->N, 256), 256, 0, h->stream>>>(
        g, (const double*)h->d_staging, (long long)G, (typename S::T*)h->f[0]);
  });
  CK_LAUNCH();
  h->cur = 0;
  h->poststream = 1;
  bump_epoch(h);
  // like IO::read_checkpoint: moments recomputed without the Guo term
  rc = engine_macro(h);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_get_populations(couplb_handle* h, double* f_host) {
  if (!h || !f_host) return fail(h, COUPLB_ERR_ARG, "null argument");
  int rc = set_device(h);
  if (rc) return rc;
  if ((rc = materialize(h))) return rc;
  const size_t G = couplb_ghost_nodes(h);
  const size_t bytes = sizeof(double) * h->Q * G;
  if ((rc = ensure_staging(h, bytes))) return rc;
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    k_export_f<L, S><<<flat_blocks((long long)G, 256), 256, 0, h->stream>>>(
        g, (const typename S::T*)h->f[h->cur], (long long)G, (double*)h->d_staging);
  });
  CK_LAUNCH();
  CK(cudaMemcpyAsync(f_host, h->d_staging, bytes, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_lbm_step(couplb_handle* h, const double* g_lb) {
  if (!h) return COUPLB_ERR_ARG;
  if (g_lb && !h->p.body_force)
    return fail(h, COUPLB_ERR_STATE, "gravity given to a lattice created with body_force = 0");
  int rc = set_device(h);
  if (rc) return rc;
  const bool g_active = g_lb && !(std::fabs(g_lb[0]) < ZERO_TOL && std::fabs(g_lb[1]) < ZERO_TOL &&
                                  std::fabs(g_lb[2]) < ZERO_TOL);
  dim3 grid, block;
  row_launch(h, &grid, &block);
  const Geom g = make_geom(h);
  const bool pull = !h->poststream;
  const int rho_mode = !g_active ? kRhoNone : (h->rho_state == kRhoCurrent ? kRhoCurrent : kRhoField);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using T = typename S::T;
    using A = typename S::A;
    LBArgs<S> a;
    a.g = g;
    a.fin = (const T*)h->f[h->cur];
    a.fout = (T*)h->f[1 - h->cur];
    a.F = h->force_dirty ? (A*)h->F : nullptr;
    a.seg_force = h->force_rows_all ? nullptr : h->seg_force;
    a.rho_field = (A*)h->rho_field;
    a.rho_mode = rho_mode;
    a.write_rho = h->p.body_force ? 2 : (h->moving_walls ? 1 : 0);
    for (int d = 0; d < 3; d++) a.grav[d] = g_active ? g_lb[d] : 0.0;
    for (int d = 0; d < 3; d++) h->g_lb[d] = a.grav[d];
    a.omega = 1.0 / h->p.tau;
    a.status = h->d_status;
    // kernel choice: packed (shifted formats, pull, even nx, 32-bit indices),
    // else staged (when asked for), else plain
    int used = kKernelPlain;
    int want = h->kernel;
    if (want == kKernelAuto) want = S::kShift ? kKernelPacked : kKernelPlain;
    if constexpr (S::kShift) {
      if (want == kKernelPacked && pull && h->idx32 && h->p.nx % 2 == 0) {
        const int pairs = h->p.nx / 2;
        const dim3 pg((pairs + 127) / 128, h->p.ny, h->p.nz);
        k_stream_collide_x2<L, S><<<pg, 128, 0, h->stream>>>(a);
        used = kKernelPacked;
      }
    }
    if (used == kKernelPlain && want == kKernelStaged && pull) {
      bool ok;
      // the staged kernel copies plane rows: plane-major storage only
      if constexpr (S::kTile == 0) {
        if constexpr (sizeof(typename S::T) == 8) ok = launch_staged<L, S, 2>(h, a);
        else ok = launch_staged<L, S, 3>(h, a);
      } else {
        ok = false;
      }
      if (ok) used = kKernelStaged;
    }
    if (used == kKernelPlain) {
      if (h->idx32) {
        if (pull) k_stream_collide<L, S, unsigned, true><<<grid, block, 0, h->stream>>>(a);
        else k_stream_collide<L, S, unsigned, false><<<grid, block, 0, h->stream>>>(a);
      } else {
        if (pull) k_stream_collide<L, S, size_t, true><<<grid, block, 0, h->stream>>>(a);
        else k_stream_collide<L, S, size_t, false><<<grid, block, 0, h->stream>>>(a);
      }
    }
    h->last_kernel = used;
  });
  CK_LAUNCH();
  h->cur = 1 - h->cur;
  h->poststream = 0;
  h->lbm_steps++;
  if (h->force_dirty) {
    // the kernel zeroed every force it read (clear_forces); reset the flags
    CK(cudaMemsetAsync(h->seg_force, 0, seg_bytes(h), h->stream));
    h->force_dirty = 0;
    h->force_rows_all = 0;
  }
  h->rho_state = h->p.body_force ? kRhoField : kRhoNone;
  h->macro_valid = 0;
  bump_epoch(h);
  return COUPLB_OK;
}

int couplb_macroscopic(couplb_handle* h) {
  if (!h) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  return engine_macro(h);
}

int couplb_get_macroscopic(couplb_handle* h, double* rho, double* ux, double* uy, double* uz) {
  if (!h) return COUPLB_ERR_ARG;
  if (!h->macro_valid) return fail(h, COUPLB_ERR_STATE, "moments not computed: call couplb_macroscopic first");
  int rc = set_device(h);
  if (rc) return rc;
  const size_t G = couplb_ghost_nodes(h);
  if ((rc = ensure_staging(h, sizeof(double) * 4 * G))) return rc;
  double* st = (double*)h->d_staging;
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using S = decltype(s);
    using A = typename S::A;
    (void)l;
    k_export_macro<S><<<flat_blocks((long long)G, 256), 256, 0, h->stream>>>(
        g, h->p.dim, (const A*)h->macro[0], (const A*)h->macro[1], (const A*)h->macro[2],
        (const A*)h->macro[3], (long long)G, st, st + G, st + 2 * G, st + 3 * G);
  });
  CK_LAUNCH();
  double* outs[4] = {rho, ux, uy, uz};
  for (int c = 0; c < 4; c++)
    if (outs[c]) CK(cudaMemcpyAsync(outs[c], st + c * G, sizeof(double) * G, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_get_force_field(couplb_handle* h, double* fx, double* fy, double* fz) {
  if (!h || !fx || !fy || !fz) return fail(h, COUPLB_ERR_ARG, "null argument");
  int rc = set_device(h);
  if (rc) return rc;
  const size_t G = couplb_ghost_nodes(h);
  if ((rc = ensure_staging(h, sizeof(double) * 3 * G))) return rc;
  double* st = (double*)h->d_staging;
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using S = decltype(s);
    using A = typename S::A;
    (void)l;
    k_export_force<S><<<flat_blocks((long long)G, 256), 256, 0, h->stream>>>(
        g, h->p.dim, (const A*)h->F, (long long)G, st,
        st + G, st + 2 * G);
  });
  CK_LAUNCH();
  double* outs[3] = {fx, fy, fz};
  for (int c = 0; c < 3; c++)
    CK(cudaMemcpyAsync(outs[c], st + c * G, sizeof(double) * G, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_set_force_field(couplb_handle* h, const double* fx, const double* fy, const double* fz) {
  if (!h || !fx || !fy || !fz) return fail(h, COUPLB_ERR_ARG, "null argument");
  int rc = set_device(h);
  if (rc) return rc;
  const size_t G = couplb_ghost_nodes(h);
  if ((rc = ensure_staging(h, sizeof(double) * 3 * G))) return rc;
  double* st = (double*)h->d_staging;
  const double* ins[3] = {fx, fy, fz};
  for (int c = 0; c < 3; c++)
    CK(cudaMemcpyAsync(st + c * G, ins[c], sizeof(double) * G, cudaMemcpyHostToDevice, h->stream));
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using S = decltype(s);
    using A = typename S::A;
    (void)l;
    k_import_force<S><<<flat_blocks((long long)h->N, 256), 256, 0, h->stream>>>(
        g, h->p.dim, st, st + G, st + 2 * G, (A*)h->F);
  });
  CK_LAUNCH();
  h->force_dirty = 1;
  h->force_rows_all = 1;   // the segment flags know nothing of these forces
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_diagnostics(couplb_handle* h, couplb_diag* out) {
  if (!h || !out) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (!h->macro_valid) return fail(h, COUPLB_ERR_STATE, "moments not computed: call couplb_macroscopic first");
  int rc = set_device(h);
  if (rc) return rc;
  const int nb = std::min<long long>(1184, std::max<long long>(1, ((long long)h->N + 255) / 256));
  if (!h->d_scratch || h->scratch_blocks < nb) {
    dfree(h->d_scratch);
    if ((rc = dalloc(h, &h->d_scratch, sizeof(double) * (5 * nb + 8)))) return rc;
    h->scratch_blocks = nb;
  }
  double* part = (double*)h->d_scratch;
  double* res = part + 5 * nb;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using S = decltype(s);
    using A = typename S::A;
    (void)l;
    k_diag_partial<S><<<nb, 256, 0, h->stream>>>((long long)h->N, h->p.rho0, (const A*)h->macro[0],
                                                 (const A*)h->macro[1], (const A*)h->macro[2],
                                                 (const A*)h->macro[3], part);
  });
  CK_LAUNCH();
  k_reduce_final<<<1, 32, 0, h->stream>>>(nb, part, res);
  CK_LAUNCH();
  double* hs = (double*)h->h_small;
  CK(cudaMemcpyAsync(hs, res, sizeof(double) * 5, cudaMemcpyDeviceToHost, h->stream));
  int* hi = (int*)(hs + 8);
  CK(cudaMemcpyAsync(hi, h->d_status, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  out->umax = hs[0];
  out->mass = hs[1];
  out->mom[0] = hs[2]; out->mom[1] = hs[3]; out->mom[2] = hs[4];
  out->clamps = hi[kStMacroClamps];
  out->nonfinite = hi[kStNonfinite];
  return COUPLB_OK;
}

int couplb_y_profile(couplb_handle* h, double* ux_sum, double* uy_sum, double* rho_sum) {
  if (!h || !ux_sum || !uy_sum || !rho_sum) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (!h->macro_valid) return fail(h, COUPLB_ERR_STATE, "moments not computed: call couplb_macroscopic first");
  int rc = set_device(h);
  if (rc) return rc;
  const int ny = h->p.ny;
  if ((rc = ensure_staging(h, sizeof(double) * 3 * ny))) return rc;
  double* st = (double*)h->d_staging;
  const Geom g = make_geom(h);
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using S = decltype(s);
    using A = typename S::A;
    (void)l;
    k_y_profile<S><<<ny, 256, 0, h->stream>>>(g, (const A*)h->macro[0], (const A*)h->macro[1],
                                              (const A*)h->macro[2], st);
  });
  CK_LAUNCH();
  CK(cudaMemcpyAsync(ux_sum, st, sizeof(double) * ny, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(uy_sum, st + ny, sizeof(double) * ny, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(rho_sum, st + 2 * ny, sizeof(double) * ny, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return COUPLB_OK;
}

int couplb_read_status(couplb_handle* h, int* clamps, int* nonfinite, int reset) {
  if (!h) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  int* hi = (int*)h->h_small;
  CK(cudaMemcpyAsync(hi, h->d_status, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CK(cudaMemsetAsync(h->d_status, 0, sizeof(int) * 2, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (clamps) *clamps = hi[kStClamps];
  if (nonfinite) *nonfinite = hi[kStNonfinite];
  return COUPLB_OK;
}

int couplb_status_post(couplb_handle* h) {
  if (!h) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  const int slot = (int)(h->status_posts & 1);
  k_status_publish<<<1, 32, 0, h->stream>>>(h->d_status, h->d_status_ring + 8 * slot);
  CK_LAUNCH();
  CK(cudaEventRecord(h->status_ev[slot], h->stream));
  h->status_posts++;
  return COUPLB_OK;
}

int couplb_status_last(couplb_handle* h, int* clamps, int* nonfinite) {
  if (!h) return COUPLB_ERR_ARG;
  int c = 0, nf = 0;
  if (h->status_posts > 0) {
    const long long want = h->status_posts >= 2 ? h->status_posts - 2 : 0;
    const int slot = (int)(want & 1);
    CK(cudaEventSynchronize(h->status_ev[slot]));
    const volatile int* ring = h->h_status_ring;
    c = ring[8 * slot + kStClamps];
    nf = ring[8 * slot + kStNonfinite];
  }
  if (clamps) *clamps = c;
  if (nonfinite) *nonfinite = nf;
  return COUPLB_OK;
}

int couplb_set_option(couplb_handle* h, const char* name, long long value) {
  if (!h || !name) return COUPLB_ERR_ARG;
  if (!std::strcmp(name, "kernel")) {
    if (value < kKernelAuto || value > kKernelPacked)
      return fail(h, COUPLB_ERR_ARG, "kernel must be -1 (auto), 0 (plain), 1 (staged) or 2 (packed)");
    h->kernel = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_resident")) {
    if (value != 0 && value != 1) return fail(h, COUPLB_ERR_ARG, "ibm_resident must be 0 or 1");
    h->ibm_resident = (int)value;
    return COUPLB_OK;
  }
  return fail(h, COUPLB_ERR_ARG, "unknown or read-only option '%s'", name);
}

int couplb_get_option(couplb_handle* h, const char* name, long long* value) {
  if (!h || !name || !value) return COUPLB_ERR_ARG;
  if (!std::strcmp(name, "kernel")) { *value = h->kernel; return COUPLB_OK; }
  if (!std::strcmp(name, "last_kernel")) { *value = h->last_kernel; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_resident")) { *value = h->ibm_resident; return COUPLB_OK; }
  if (!std::strcmp(name, "timeouts")) {
    int rc = set_device(h);
    if (rc) return rc;
    int* hi = (int*)h->h_small;
    CK(cudaMemcpyAsync(hi, h->d_status, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *value = hi[kStTimeout];
    return COUPLB_OK;
  }
  return fail(h, COUPLB_ERR_ARG, "unknown option '%s'", name);
}

int couplb_set_ibm_params(couplb_handle* h, const couplb_ibm_params* ip) {
  if (!h || !ip) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (ip->md_per_lb < 1) return fail(h, COUPLB_ERR_ARG, "md_per_lb must be >= 1");
  if (ip->delta != COUPLB_DELTA_ROMA && ip->delta != COUPLB_DELTA_PESKIN4)
    return fail(h, COUPLB_ERR_ARG, "unknown delta kernel %d", ip->delta);
  if (!(ip->dx > 0) || !(ip->dt_lbm > 0) || !(ip->force_scale > 0))
    return fail(h, COUPLB_ERR_ARG, "dx, dt_lbm and force_scale must be positive");
  h->ip = *ip;
  h->ip_set = 1;
  return COUPLB_OK;
}

}  // extern "C"

namespace couplb {

// Shared body of the host- and device-array IBM sub-step.
// Blocks of a cooperative kernel that fit on the device at once (cached).
template <class K>
int coop_resident(couplb_handle* h, K kern, size_t smem, int slot, int* out) {
  int& resident = h->coop_blocks[slot];
  if (resident == 0) {
    int coop = 0, sms = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->p.device));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->p.device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (!coop || per_sm < 1)
      return fail(h, COUPLB_ERR_UNSUPPORTED, "the device cannot run the cooperative IBM kernel");
    resident = per_sm * sms;
  }
  *out = resident;
  return COUPLB_OK;
}

// Cooperative launch of one ITERATIVE / LEARNED sub-step (all blocks
// resident at once, which its grid barriers need).  In 3D, when every marker
// gets a warp of its own, the register-resident form runs.
template <class L, class S>
int launch_method(couplb_handle* h, PassArgs<S>& P, int delta, bool learned, int n) {
  using K = void (*)(const PassArgs<S>);
  const bool roma = delta == COUPLB_DELTA_ROMA;
  const int di = (learned ? 2 : 0) + (roma ? 0 : 1);
  const size_t smem = learned ? kLearnedSmem : 0;
  const long long want = ((long long)n * 32 + 255) / 256;
  void* args[] = {&P};
  int rc, resident = 0;
  if constexpr (L::D == 3) {
    if (h->ibm_resident) {
      K kr = learned ? (roma ? k_ibm_method_resident<L, S, 0, true> : k_ibm_method_resident<L, S, 1, true>)
                     : (roma ? k_ibm_method_resident<L, S, 0, false> : k_ibm_method_resident<L, S, 1, false>);
      if ((rc = coop_resident(h, kr, smem, 4 + di, &resident))) return rc;
      if (want <= resident) {
        CK(cudaLaunchCooperativeKernel((const void*)kr, dim3((unsigned)want), dim3(256), args, smem,
                                       h->stream));
        return COUPLB_OK;
      }
    }
  }
  K kern = nullptr;
  if (learned) {
    if constexpr (L::D == 3) kern = roma ? k_ibm_method<L, S, 0, true> : k_ibm_method<L, S, 1, true>;
  } else {
    kern = roma ? k_ibm_method<L, S, 0, false> : k_ibm_method<L, S, 1, false>;
  }
  if (!kern) return fail(h, COUPLB_ERR_UNSUPPORTED, "the learned correction is defined for D3Q19");
  if ((rc = coop_resident(h, kern, smem, di, &resident))) return rc;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(want, resident));
  CK(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(256), args, smem, h->stream));
  return COUPLB_OK;
}

int engine_ibm(couplb_handle* h, int n, const double* d_x, const double* d_v, const double* d_m,
               const int* d_active, double* d_fout, int accumulate, int refresh) {
  // no coupled atoms: the reference returns before refreshing the moments
  // (fix_couplb.cpp:750-753)
  if (n <= 0) return COUPLB_OK;
  const couplb_ibm_params& ip = h->ip;
  const int method = h->ibm_method;
  if (method == COUPLB_IBM_LEARNED && (h->p.dim != 3 || !h->mlp))
    return fail(h, COUPLB_ERR_UNSUPPORTED, "the learned correction needs D3Q19 and a network");
  // The refresh of compute_macroscopic(false) (fix_couplb.cpp:757-760): the
  // velocities are computed on demand by the kernel; the density it would
  // store is what the next LB step's body force reads.
  if (refresh && h->p.body_force) h->rho_state = kRhoCurrent;
  int rc = ensure_stencil_cache(h, n);
  if (rc) return rc;
  bool record = false;
  if (method != COUPLB_IBM_SINGLE) {
    if ((rc = ensure_method_buffers(h, n))) return rc;
    if (h->rec_rows) {
      if (d_active) return fail(h, COUPLB_ERR_STATE, "sample capture needs every atom coupled");
      record = h->rec_count + n <= h->rec_cap;
    }
  }
  const double dxp = ip.dx;
  const double dv = (h->p.dim == 3) ? dxp * dxp * dxp : dxp * dxp;
  const double cell_vol = dxp * dxp * ((h->p.dim == 3) ? dxp : 1.0);
  const Geom g = make_geom(h);
  const int bs = 256;
  const unsigned nb = (unsigned)(((long long)n * 32 + bs - 1) / bs);
  int lrc = COUPLB_OK;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using A = typename S::A;
    IbmArgs<S> a;
    a.g = g;
    a.fin = (const typename S::T*)h->f[h->cur];
    a.rho_field = (const A*)h->rho_field;
    a.pull = h->poststream ? 0 : 1;
    a.cux = (const A*)h->macro[1]; a.cuy = (const A*)h->macro[2]; a.cuz = (const A*)h->macro[3];
    a.all_valid = h->macro_valid;
    a.crho = (const A*)h->macro[0];
    a.sbuf = (A*)h->sbuf;
    a.skey = h->skey;
    a.cur_epoch = h->cur_epoch;
    a.F = (A*)h->F;
    a.seg_force = h->seg_force;
    a.n = n;
    a.x = d_x; a.v = d_v; a.m = d_m; a.active = d_active;
    a.fout = d_fout;
    a.accumulate = accumulate;
    a.ftot = h->d_ftot;
    for (int d = 0; d < 3; d++) { a.lo[d] = ip.domain_lo[d]; a.off[d] = ip.offset[d]; }
    if (h->p.dim == 2) a.off[2] = 0;
    a.inv_dx = 1.0 / dxp;
    a.xi_over_dt = ip.xi_ibm / ip.dt_lbm;
    a.inv_N = 1.0 / (double)ip.md_per_lb;
    a.vs = ip.vel_scale;
    a.fs = ip.force_scale;
    a.dvr = dv / cell_vol;
    a.corr = method != COUPLB_IBM_SINGLE ? h->d_corr : nullptr;
    a.mlp = (method == COUPLB_IBM_LEARNED) ? h->mlp->pack : nullptr;
    if (method == COUPLB_IBM_SINGLE) {
      if (refresh && !a.all_valid) k_ibm_prefetch<L, S><<<nb, bs, 0, h->stream>>>(a);
      if (ip.delta == COUPLB_DELTA_ROMA) k_ibm_substep<L, S, 0><<<nb, bs, 0, h->stream>>>(a);
      else k_ibm_substep<L, S, 1><<<nb, bs, 0, h->stream>>>(a);
    } else {
      PassState* ps = (PassState*)h->d_pass;
      h->pass_cur ^= 1;
      PassArgs<S> P;
      P.a = a;
      P.dF = h->d_dF;
      P.ps = ps + h->pass_cur;
      P.ps_next = ps + (h->pass_cur ^ 1);
      P.fill = refresh && !a.all_valid;
      P.status = h->d_status;
      P.ncorr = h->ibm_passes - 1;
      P.check_first = method == COUPLB_IBM_LEARNED;
      P.slip_tol = h->slip_tol;
      for (int d = 0; d < 3; d++) P.g_lb[d] = h->g_lb[d];
      P.rows = record ? h->rec_rows + h->rec_count * kMlpRow : nullptr;
      lrc = launch_method<L, S>(h, P, ip.delta, method == COUPLB_IBM_LEARNED, n);
    }
  });
  if (lrc) return lrc;
  CK_LAUNCH();
  if (record) h->rec_count += n;
  h->force_dirty = 1;
  return COUPLB_OK;
}

}  // namespace couplb

extern "C" {

int couplb_ibm_substep(couplb_handle* h, int n, const double* x, const double* v,
                       const double* mass, const int* active, double* f_add, int refresh,
                       int* ncoupled) {
  if (!h) return COUPLB_ERR_ARG;
  if (!h->ip_set) return fail(h, COUPLB_ERR_STATE, "couplb_set_ibm_params not called");
  if (n < 0 || (n > 0 && (!x || !v || !mass || !f_add))) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  int rc = set_device(h);
  if (rc) return rc;
  int nc = 0;
  for (int a = 0; a < n; a++) nc += active ? (active[a] != 0) : 1;
  if (ncoupled) *ncoupled = nc;
  if ((rc = ensure_atoms(h, n))) return rc;
  if (n > 0) {
    CK(cudaMemcpyAsync(h->d_x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_v, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_m, mass, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    if (active) CK(cudaMemcpyAsync(h->d_active, active, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
  }
  rc = engine_ibm(h, nc > 0 ? n : 0, (const double*)h->d_x, (const double*)h->d_v,
                  (const double*)h->d_m, active ? (const int*)h->d_active : nullptr,
                  (double*)h->d_fout, 0, refresh);
  if (rc) return rc;
  if (nc > 0) {
    CK(cudaMemcpyAsync(h->h_fout, h->d_fout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int a = 0; a < 3 * n; a++) f_add[a] += h->h_fout[a];
  }
  return COUPLB_OK;
}

int couplb_ibm_substep_device(couplb_handle* h, int n, const double* d_x, const double* d_v,
                              const double* d_mass, const int* d_active, double* d_f_add,
                              int refresh) {
  if (!h) return COUPLB_ERR_ARG;
  if (!h->ip_set) return fail(h, COUPLB_ERR_STATE, "couplb_set_ibm_params not called");
  if (n < 0 || (n > 0 && (!d_x || !d_v || !d_mass || !d_f_add))) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  int rc = set_device(h);
  if (rc) return rc;
  return engine_ibm(h, n, d_x, d_v, d_mass, d_active, d_f_add, 1, refresh);
}

int couplb_set_ibm_method(couplb_handle* h, const couplb_ibm_method* m) {
  if (!h || !m) return COUPLB_ERR_ARG;
  if (m->method < COUPLB_IBM_SINGLE || m->method > COUPLB_IBM_LEARNED)
    return fail(h, COUPLB_ERR_ARG, "unknown IBM method %d", m->method);
  if (m->passes < 1 || m->passes > 64) return fail(h, COUPLB_ERR_ARG, "passes must be 1..64");
  if (m->method == COUPLB_IBM_LEARNED) {
    if (!m->model) return fail(h, COUPLB_ERR_ARG, "the learned method needs a network");
    if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "the learned correction is defined for D3Q19");
    if (m->model->device != h->p.device)
      return fail(h, COUPLB_ERR_ARG, "the network lives on device %d, the lattice on %d", m->model->device,
                  h->p.device);
    if (!(m->slip_tol >= 0.0)) return fail(h, COUPLB_ERR_ARG, "slip_tol must be >= 0");
  }
  h->ibm_method = m->method;
  h->ibm_passes = m->passes;
  h->slip_tol = m->slip_tol;
  h->mlp = m->method == COUPLB_IBM_LEARNED ? m->model : nullptr;
  return COUPLB_OK;
}

int couplb_ibm_slip(couplb_handle* h, double out[8], int reset) {
  if (!h || !out) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  for (int i = 0; i < 8; i++) out[i] = 0.0;
  unsigned char* hs = (unsigned char*)h->h_small;
  static_assert(sizeof(PassState) + 8 * sizeof(int) <= 4096, "h_small holds the pass state");
  if (h->d_pass)
    CK(cudaMemcpyAsync(hs, (PassState*)h->d_pass + h->pass_cur, sizeof(PassState), cudaMemcpyDeviceToHost,
                       h->stream));
  else std::memset(hs, 0, sizeof(PassState));
  int* st = (int*)(hs + sizeof(PassState));
  CK(cudaMemcpyAsync(st, h->d_status, sizeof(int) * 8, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CK(cudaMemsetAsync(h->d_status + kStSlipChecks, 0, sizeof(int) * 2, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  PassState ps;
  std::memcpy(&ps, hs, sizeof ps);
  auto count = [&](int r) {
    int c = 0;
    for (int i = 0; i < kSlipSlots; i++) c += ps.count[r][i];
    return c;
  };
  auto rms = [&](int r) {
    double s = 0.0;
    for (int i = 0; i < kSlipSlots; i++) s += ps.s2[r][i];
    const int c = count(r);
    return c > 0 ? std::sqrt(s / c) : 0.0;
  };
  auto mx = [&](int r) {
    double m = 0.0;
    for (int i = 0; i < kSlipSlots; i++) {
      double v;
      std::memcpy(&v, &ps.max_bits[r][i], sizeof v);
      m = std::max(m, v);
    }
    return m;
  };
  const int r = (ps.checked && !ps.fell_back) ? 0 : 1;
  out[0] = rms(r);
  out[1] = mx(r);
  out[2] = ps.checked ? rms(0) : 0.0;
  out[3] = ps.checked ? mx(0) : 0.0;
  out[4] = count(r);
  out[5] = ps.fell_back;
  out[6] = st[kStSlipChecks];
  out[7] = st[kStFallbacks];
  return COUPLB_OK;
}

int couplb_ibm_record(couplb_handle* h, float* d_rows, long long capacity) {
  if (!h) return COUPLB_ERR_ARG;
  if (d_rows && capacity < 0) return fail(h, COUPLB_ERR_ARG, "negative capacity");
  h->rec_rows = d_rows;
  h->rec_cap = d_rows ? capacity : 0;
  h->rec_count = 0;
  return COUPLB_OK;
}

int couplb_ibm_record_count(couplb_handle* h, long long* rows) {
  if (!h || !rows) return COUPLB_ERR_ARG;
  *rows = h->rec_count;
  return COUPLB_OK;
}

int couplb_ibm_total_force(couplb_handle* h, double out[3], int reset) {
  if (!h || !out) return COUPLB_ERR_ARG;
  int rc = set_device(h);
  if (rc) return rc;
  double* hs = (double*)h->h_small;
  CK(cudaMemcpyAsync(hs, h->d_ftot, sizeof(double) * 4 * kFtotSlots, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CK(cudaMemsetAsync(h->d_ftot, 0, sizeof(double) * 4 * kFtotSlots, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  out[0] = out[1] = out[2] = 0.0;
  for (int s = 0; s < kFtotSlots; s++)
    for (int c = 0; c < 3; c++) out[c] += hs[4 * s + c];
  return COUPLB_OK;
}

}  // extern "C"
