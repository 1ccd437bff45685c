// engine.cu -- layer 1 of the C ABI (include/couplb_b200.h): one handle per
// LBM subdomain, all state resident in device memory, kernels on one stream.
// This file: the lattice (create, LB step, moments, populations, force
// field, diagnostics, options); engine_ibm.cu: the immersed-boundary part.
#include "engine_common.cuh"
#include "lbm_packed.cuh"
#include "mlp_internal.h"

using namespace couplb;
using namespace couplb::eng;

namespace {

// Copy of the status word (clamp and non-finite counts) into a posted slot of
// mapped pinned host memory; read by the host after the slot's event.
__global__ void k_status_publish(const int* __restrict__ st, int* ring_slot) {
  if (threadIdx.x < 2) ring_slot[threadIdx.x] = st[threadIdx.x];
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

int engine_atom_host_buffers(couplb_handle* h, int n, double** mass, int** active) {
  int rc = set_device(h);
  if (rc) return rc;
  if ((rc = ensure_atoms(h, n))) return rc;
  *mass = h->h_mass;
  *active = h->h_active;
  return COUPLB_OK;
}

void engine_atom_host_hint(couplb_handle* h, int n, int count, int unchanged) {
  h->hint_n = n;
  h->hint_count = count;
  h->hint_unchanged = unchanged;
}

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
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  for (int e = 0; e < 2; e++)
    if (h->copy_ev[e]) cudaEventDestroy(h->copy_ev[e]);
  for (cudaEvent_t e : h->fout_ev)
    if (e) cudaEventDestroy(e);
  if (h->h_order_near) cudaFreeHost(h->h_order_near);
  {
    void* p2 = h->d_order; dfree(p2);
    p2 = h->d_order_rank; dfree(p2);
    p2 = h->d_order_count; dfree(p2);
  }
  dfree(h->d_x); dfree(h->d_v); dfree(h->d_m); dfree(h->d_fout); dfree(h->d_active);
  if (h->h_fout) cudaFreeHost(h->h_fout);
  if (h->h_mass) cudaFreeHost(h->h_mass);
  if (h->h_active) cudaFreeHost(h->h_active);
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
  return engine_lbm_step(h, g_lb);
}

}  // extern "C"

namespace couplb {

int engine_lbm_step(couplb_handle* h, const double* g_lb) {
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
    // else plain
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

}  // namespace couplb

extern "C" {

int couplb_halo_attach(couplb_handle* h, int side, const void* d_recv) {
  if (!h) return COUPLB_ERR_ARG;
  if (side != 0 && side != 1) return fail(h, COUPLB_ERR_ARG, "halo side must be 0 (z low) or 1 (z high)");
  if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "halo faces are z faces of a D3Q19 lattice");
  if (d_recv && h->p.wall[4 + side] != COUPLB_WALL_PERIODIC)
    return fail(h, COUPLB_ERR_ARG, "a halo face must not be a wall (z face %d has type %d)", side,
                h->p.wall[4 + side]);
  h->halo[side] = d_recv;
  return COUPLB_OK;
}

size_t couplb_halo_bytes(const couplb_handle* h) {
  if (!h || h->p.dim != 3) return 0;
  return (size_t)kHaloQ * h->p.nx * h->p.ny * elem_bytes_pop(h->p.precision);
}

int couplb_halo_pack(couplb_handle* h, int side, void* d_send) {
  if (!h || !d_send) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return fail(h, COUPLB_ERR_ARG, "halo side must be 0 (z low) or 1 (z high)");
  if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "halo faces are z faces of a D3Q19 lattice");
  if (h->poststream)
    return fail(h, COUPLB_ERR_STATE, "halo pack needs the post-collision state of an LB step");
  int rc = set_device(h);
  if (rc) return rc;
  const Geom g = make_geom(h);
  const long long cnt = (long long)kHaloQ * h->p.nx * h->p.ny;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using T = typename S::T;
    if constexpr (L::D == 3)
      k_halo_pack<L, S><<<flat_blocks(cnt, 256), 256, 0, h->stream>>>(g, (const T*)h->f[h->cur], side,
                                                                      (T*)d_send);
  });
  CK_LAUNCH();
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
  k_reduce_final<<<1, kReduceThreads, 0, h->stream>>>(nb, part, res);
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
    if (value != kKernelAuto && value != kKernelPlain && value != kKernelPacked)
      return fail(h, COUPLB_ERR_ARG, "kernel must be -1 (auto), 0 (plain) or 2 (packed)");
    h->kernel = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_resident")) {
    if (value != 0 && value != 1) return fail(h, COUPLB_ERR_ARG, "ibm_resident must be 0 or 1");
    h->ibm_resident = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_window")) {
    if (value != 0 && value != 1) return fail(h, COUPLB_ERR_ARG, "ibm_window must be 0 (clip) or 1 (wrap)");
    h->ibm_window = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_slip")) {
    if (value != 0 && value != 1) return fail(h, COUPLB_ERR_ARG, "ibm_slip must be 0 or 1");
    h->ibm_slip = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_group")) {
    if (value != 8 && value != 32) return fail(h, COUPLB_ERR_ARG, "ibm_group must be 8 or 32");
    h->ibm_group = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_sort")) {
    if (value < 0 || value > (1 << 30)) return fail(h, COUPLB_ERR_ARG, "ibm_sort must be 0..2^30");
    h->ibm_sort = (int)value;
    h->order_n = -1;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "ibm_block")) {
    if (value != 64 && value != 128 && value != 256)
      return fail(h, COUPLB_ERR_ARG, "ibm_block must be 64, 128 or 256");
    h->ibm_block = (int)value;
    return COUPLB_OK;
  }
  if (!std::strcmp(name, "barrier_spin")) {
    if (value < 0 || value > (1LL << 40)) return fail(h, COUPLB_ERR_ARG, "barrier_spin must be 0..2^40");
    h->barrier_spin = value;
    return COUPLB_OK;
  }
  return fail(h, COUPLB_ERR_ARG, "unknown or read-only option '%s'", name);
}

int couplb_get_option(couplb_handle* h, const char* name, long long* value) {
  if (!h || !name || !value) return COUPLB_ERR_ARG;
  if (!std::strcmp(name, "kernel")) { *value = h->kernel; return COUPLB_OK; }
  if (!std::strcmp(name, "last_kernel")) { *value = h->last_kernel; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_resident")) { *value = h->ibm_resident; return COUPLB_OK; }
  if (!std::strcmp(name, "barrier_spin")) { *value = h->barrier_spin; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_window")) { *value = h->ibm_window; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_group")) { *value = h->ibm_group; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_block")) { *value = h->ibm_block; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_sort")) { *value = h->ibm_sort; return COUPLB_OK; }
  if (!std::strcmp(name, "ibm_slip")) { *value = h->ibm_slip; return COUPLB_OK; }
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

}  // extern "C"
