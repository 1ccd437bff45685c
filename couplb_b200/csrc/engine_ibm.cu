// engine_ibm.cu -- layer 1 of the C ABI, immersed-boundary part: the IBM
// constants, the sub-steps (single pass, iterative and learned methods),
// slip, training-sample capture and the total-force accumulator.
#include "engine_common.cuh"
#include "engine_methods.cuh"
#include "mlp_internal.h"

using namespace couplb;
using namespace couplb::eng;

extern "C" {

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

void engine_note_refresh(couplb_handle* h) {
  if (h->p.body_force) h->rho_state = kRhoCurrent;
}

// The processing order of the markers' refresh and grouped sub-step
// (k_order_count / k_order_scan / k_order_scatter on the lattice's stream).
template <class L, class S>
int make_order(couplb_handle* h, const IbmArgs<S>& a, int n) {
  const int nb = ((L::D == 3 ? h->p.nz : h->p.ny) + kOrderPlanes - 1) / kOrderPlanes;
  if (h->order_cap < n) {
    void* p = h->d_order; dfree(p); h->d_order = nullptr;
    p = h->d_order_rank; dfree(p); h->d_order_rank = nullptr;
    h->order_cap = 0;
    const int cap = std::max(n, 1024);
    int rc;
    if ((rc = dalloc(h, (void**)&h->d_order, sizeof(int) * (size_t)cap))) return rc;
    if ((rc = dalloc(h, (void**)&h->d_order_rank, sizeof(int) * (size_t)cap))) return rc;
    h->order_cap = cap;
  }
  if (h->order_nb < nb) {
    void* p = h->d_order_count; dfree(p); h->d_order_count = nullptr;
    h->order_nb = 0;
    // the band sizes, then the count of markers next to their successor
    int rc = dalloc(h, (void**)&h->d_order_count, sizeof(int) * ((size_t)nb + 1));
    if (rc) return rc;
    h->order_nb = nb;
  }
  if (!h->h_order_near) CK(cudaMallocHost(&h->h_order_near, sizeof(int)));
  CK(cudaMemsetAsync(h->d_order_count, 0, sizeof(int) * ((size_t)nb + 1), h->stream));
  const unsigned g = (unsigned)((n + 255) / 256);
  k_order_count<L, S><<<g, 256, 0, h->stream>>>(a, nb, h->d_order_count, h->d_order_rank);
  k_order_scan<<<1, 256, 0, h->stream>>>(nb, h->d_order_count);
  k_order_scatter<L, S><<<g, 256, 0, h->stream>>>(a, nb, h->d_order_count, h->d_order_rank, h->d_order);
  CK_LAUNCH();
  // the scatter's choice, read back now (one wait per sort, every ibm_sort
  // refreshes): when it kept the index order the refresh is launched
  // without the order, whose lookup would only lengthen each warp's chain
  CK(cudaMemcpyAsync(h->h_order_near, h->d_order_count + nb, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->order_identity = 2LL * *h->h_order_near > n ? 1 : 0;
  h->order_n = n;
  h->order_age = 0;
  return COUPLB_OK;
}

// The order to pass to the refresh: null while none is made, or when the
// last sort kept the index order.
inline const int* refresh_order(couplb_handle* h, int n) {
  if (h->ibm_sort <= 0 || h->order_n != n || h->order_identity != 0) return nullptr;
  return h->d_order;
}

// Shared body of the host- and device-array IBM sub-step.  The launches of
// the method kernels (launch_method) are compiled in engine_methods_*.cu.
int engine_ibm(couplb_handle* h, int n, const double* d_x, const double* d_v, const double* d_m,
               const int* d_active, double* d_fout, int accumulate, int refresh) {
  for (int side = 0; side < 2; side++)
    if (h->halo[side] && !h->ih_vel[side])
      return fail(h, COUPLB_ERR_STATE,
                  "IBM sub-step on a lattice with a halo on z face %d needs couplb_ibm_halo_attach there", side);
  if ((h->halo[0] || h->halo[1]) && h->ibm_method != COUPLB_IBM_SINGLE)
    return fail(h, COUPLB_ERR_UNSUPPORTED,
                "the iterative and learned IBM methods are not decomposed into slabs (single pass only)");
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
    a.spread_c = a.inv_N / a.fs;
    a.dvr = dv / cell_vol;
    a.corr = method != COUPLB_IBM_SINGLE ? h->d_corr : nullptr;
    a.mlp = (method == COUPLB_IBM_LEARNED) ? h->mlp->pack : nullptr;
    a.wrap = 0;
    if (h->ibm_window) {
      if (!g.face[0] && !g.face[1]) a.wrap |= 1;
      if (!g.face[2] && !g.face[3]) a.wrap |= 2;
      // z faces bound to neighbour slabs take the window through their halos
      if (h->p.dim == 3 && !g.face[4] && !g.face[5] && !h->halo[0] && !h->halo[1]) a.wrap |= 4;
    }
    for (int side = 0; side < 2; side++) {
      const bool bound = h->halo[side] && h->ih_vel[side];
      a.vh[side] = bound ? (const A*)h->ih_vel[side] : nullptr;
      a.fh[side] = bound ? (A*)h->ih_force[side] : nullptr;
      a.zplanes[side] = bound ? h->ih_planes[side] : 0;
    }
    if (method == COUPLB_IBM_SINGLE) {
      if (refresh && !a.all_valid) {
        // the marker order is remade every ibm_sort refreshes (and for a new
        // marker count); in between it only gets less local as markers move
        if (h->ibm_sort > 0 && (h->order_n != n || ++h->order_age >= h->ibm_sort)) {
          lrc = make_order<L, S>(h, a, n);
          if (lrc) return;
        }
        a.order = refresh_order(h, n);
        k_ibm_prefetch<L, S><<<nb, bs, 0, h->stream>>>(a);
        // the sub-steps keep the index order: markers that the caller keeps
        // in chain order (rods, filaments) spread onto shared nodes from one
        // warp there, which the cell order would scatter
        a.order = nullptr;
      }
      bool grouped = false;
      if constexpr (L::D == 3) {
        if (h->ibm_group == 8) {
          // four markers per warp of 8 lanes each: ibm_block / 8 markers per block
          const int bs8 = h->ibm_block;
          const unsigned nb8 = (unsigned)(((long long)n * 8 + bs8 - 1) / bs8);
          const bool halo = a.zplanes[0] || a.zplanes[1];
          if (ip.delta == COUPLB_DELTA_ROMA) {
            if (halo) k_ibm_substep8<L, S, 0, true><<<nb8, bs8, 0, h->stream>>>(a);
            else k_ibm_substep8<L, S, 0, false><<<nb8, bs8, 0, h->stream>>>(a);
          } else {
            if (halo) k_ibm_substep8<L, S, 1, true><<<nb8, bs8, 0, h->stream>>>(a);
            else k_ibm_substep8<L, S, 1, false><<<nb8, bs8, 0, h->stream>>>(a);
          }
          grouped = true;
        }
      }
      if (!grouped) {
        if (ip.delta == COUPLB_DELTA_ROMA) k_ibm_substep<L, S, 0><<<nb, bs, 0, h->stream>>>(a);
        else k_ibm_substep<L, S, 1><<<nb, bs, 0, h->stream>>>(a);
      }
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
      // LEARNED with slip_tol >= kNoFallback never falls back: no check, no
      // corrections
      P.check_first = method == COUPLB_IBM_LEARNED && h->slip_tol < kNoFallback;
      P.ncorr = (method == COUPLB_IBM_LEARNED && !P.check_first) ? 0 : h->ibm_passes - 1;
      P.measure_last = h->ibm_slip;
      P.slip_tol = h->slip_tol;
      for (int d = 0; d < 3; d++) P.g_lb[d] = h->g_lb[d];
      P.rows = record ? h->rec_rows + h->rec_count * kMlpRow : nullptr;
      P.spin = h->barrier_spin;
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

namespace {

constexpr int kForceChunks = 4;

int ensure_copy_stream(couplb_handle* h) {
  if (h->copy_stream) return COUPLB_OK;
  CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  for (int e = 0; e < 2; e++) CK(cudaEventCreateWithFlags(&h->copy_ev[e], cudaEventDisableTiming));
  for (int e = 0; e < kForceChunks; e++) CK(cudaEventCreateWithFlags(&h->fout_ev[e], cudaEventDisableTiming));
  return COUPLB_OK;
}

// The sub-step of the staged atoms, then the forces back to the host: the
// copy comes back in kForceChunks pieces and each is added to f_add while the
// next one travels.
int substep_staged(couplb_handle* h, int n, const int* active, int nc, double* f_add, int refresh) {
  int rc = engine_ibm(h, nc > 0 ? n : 0, (const double*)h->d_x, (const double*)h->d_v,
                      (const double*)h->d_m, active ? (const int*)h->d_active : nullptr,
                      (double*)h->d_fout, 0, refresh);
  if (rc) return rc;
  if (nc > 0) {
    const long long tot = 3LL * n;
    const double* d = (const double*)h->d_fout;
    for (int k = 0; k < kForceChunks; k++) {
      const long long lo = tot * k / kForceChunks, hi = tot * (k + 1) / kForceChunks;
      if (hi > lo)
        CK(cudaMemcpyAsync(h->h_fout + lo, d + lo, sizeof(double) * (hi - lo), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaEventRecord(h->fout_ev[k], h->stream));
    }
    for (int k = 0; k < kForceChunks; k++) {
      const long long lo = tot * k / kForceChunks, hi = tot * (k + 1) / kForceChunks;
      CK(cudaEventSynchronize(h->fout_ev[k]));
      for (long long a = lo; a < hi; a++) f_add[a] += h->h_fout[a];
    }
  }
  return COUPLB_OK;
}

int check_host_args(couplb_handle* h, int n, const double* f_add) {
  if (!h) return COUPLB_ERR_ARG;
  if (!h->ip_set) return fail(h, COUPLB_ERR_STATE, "couplb_set_ibm_params not called");
  if (n > 0 && !f_add) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  return set_device(h);
}

}  // namespace

namespace couplb {

int engine_host_begin(couplb_handle* h, bool lbm, const double* g_lb, int n, const double* x, const double* v) {
  if (!h->ip_set) return fail(h, COUPLB_ERR_STATE, "couplb_set_ibm_params not called");
  if (n < 0 || (n > 0 && (!x || !v))) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  int rc = set_device(h);
  if (rc) return rc;
  if ((rc = ensure_atoms(h, n))) return rc;
  if ((rc = ensure_copy_stream(h))) return rc;
  // the copies wait for the lattice's stream to reach this point (the
  // previous sub-step read the same device buffers), then run beside the LB
  // kernel
  CK(cudaEventRecord(h->copy_ev[0], h->stream));
  CK(cudaStreamWaitEvent(h->copy_stream, h->copy_ev[0], 0));
  if (n > 0) {
    CK(cudaMemcpyAsync(h->d_x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->copy_stream));
    CK(cudaMemcpyAsync(h->d_v, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->copy_stream));
  }
  h->staged_n = n;
  return lbm ? engine_lbm_step(h, g_lb) : COUPLB_OK;
}

int engine_host_finish(couplb_handle* h, bool lbm, int n, const double* mass, const int* active, double* f_add,
                       int refresh, int* ncoupled) {
  if (h->staged_n != n) return fail(h, COUPLB_ERR_STATE, "sub-step of %d atoms without their positions", n);
  h->staged_n = -1;
  if (n > 0 && !mass) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  // the fix core's pinned mass / group buffers come with their count and
  // whether they changed since their last device copy
  const bool pinned = mass == h->h_mass && active == h->h_active && h->hint_n == n;
  int c = 0;
  if (pinned) {
    c = h->hint_count;
  } else {
    for (int a = 0; a < n; a++) c += active ? (active[a] != 0) : 1;
  }
  const bool statics_current = pinned && h->hint_unchanged && h->statics_n == n;
  h->hint_n = -1;
  if (ncoupled) *ncoupled = c;
  if (n > 0 && !statics_current) {
    CK(cudaMemcpyAsync(h->d_m, mass, sizeof(double) * n, cudaMemcpyHostToDevice, h->copy_stream));
    if (active) CK(cudaMemcpyAsync(h->d_active, active, sizeof(int) * n, cudaMemcpyHostToDevice, h->copy_stream));
  }
  if (n > 0) h->statics_n = (pinned && active) ? n : -1;
  CK(cudaEventRecord(h->copy_ev[1], h->copy_stream));
  CK(cudaStreamWaitEvent(h->stream, h->copy_ev[1], 0));
  return substep_staged(h, n, active, c, f_add, lbm ? 1 : refresh);
}

}  // namespace couplb

extern "C" {

int couplb_ibm_substep(couplb_handle* h, int n, const double* x, const double* v,
                       const double* mass, const int* active, double* f_add, int refresh,
                       int* ncoupled) {
  int rc = check_host_args(h, n, f_add);
  if (rc) return rc;
  if ((rc = engine_host_begin(h, false, nullptr, n, x, v))) return rc;
  return engine_host_finish(h, false, n, mass, active, f_add, refresh, ncoupled);
}

int couplb_lbm_step_ibm(couplb_handle* h, const double* g_lb, int n, const double* x, const double* v,
                        const double* mass, const int* active, double* f_add, int* ncoupled) {
  int rc = check_host_args(h, n, f_add);
  if (rc) return rc;
  if ((rc = engine_host_begin(h, true, g_lb, n, x, v))) return rc;
  return engine_host_finish(h, true, n, mass, active, f_add, 1, ncoupled);
}

int couplb_lbm_step_ibm_device(couplb_handle* h, const double* g_lb, int n, const double* d_x,
                               const double* d_v, const double* d_mass, const int* d_active,
                               double* d_f_add) {
  if (!h) return COUPLB_ERR_ARG;
  if (!h->ip_set) return fail(h, COUPLB_ERR_STATE, "couplb_set_ibm_params not called");
  if (n < 0 || (n > 0 && (!d_x || !d_v || !d_mass || !d_f_add))) return fail(h, COUPLB_ERR_ARG, "bad atom arrays");
  int rc = set_device(h);
  if (rc) return rc;
  if ((rc = engine_lbm_step(h, g_lb))) return rc;
  return engine_ibm(h, n, d_x, d_v, d_mass, d_active, d_f_add, 1, 1);
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

size_t couplb_ibm_halo_bytes(const couplb_handle* h, int planes) {
  if (!h || h->p.dim != 3 || planes < 1 || planes > 2) return 0;
  return (size_t)planes * h->p.nx * h->p.ny * 4 * elem_bytes_aux(h->p.precision);
}

int couplb_ibm_halo_attach(couplb_handle* h, int side, int planes, const void* d_vel, void* d_force) {
  if (!h) return COUPLB_ERR_ARG;
  if (side != 0 && side != 1) return fail(h, COUPLB_ERR_ARG, "halo side must be 0 (z low) or 1 (z high)");
  if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "halo faces are z faces of a D3Q19 lattice");
  if (!d_vel) {
    h->ih_vel[side] = nullptr;
    h->ih_force[side] = nullptr;
    h->ih_planes[side] = 0;
    return COUPLB_OK;
  }
  if (!d_force) return fail(h, COUPLB_ERR_ARG, "null force halo");
  if (planes < 1 || planes > (side ? 2 : 1))
    return fail(h, COUPLB_ERR_ARG, "an IBM halo holds 1 plane below the low face and 1 or 2 above the high face");
  if (h->p.nz < 2) return fail(h, COUPLB_ERR_ARG, "IBM across slabs needs slabs of at least 2 planes");
  if (h->p.wall[4 + side] != COUPLB_WALL_PERIODIC)
    return fail(h, COUPLB_ERR_ARG, "a halo face must not be a wall (z face %d has type %d)", side,
                h->p.wall[4 + side]);
  h->ih_vel[side] = d_vel;
  h->ih_force[side] = d_force;
  h->ih_planes[side] = planes;
  return COUPLB_OK;
}

int couplb_ibm_halo_moments(couplb_handle* h, int side, int planes, void* d_out) {
  if (!h || !d_out) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return fail(h, COUPLB_ERR_ARG, "halo side must be 0 (z low) or 1 (z high)");
  if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "halo faces are z faces of a D3Q19 lattice");
  if (planes < 1 || planes > (side ? 1 : 2) || planes > h->p.nz)
    return fail(h, COUPLB_ERR_ARG, "the neighbour below reads 1 or 2 planes, the one above 1");
  int rc = set_device(h);
  if (rc) return rc;
  const Geom g = make_geom(h);
  const long long cnt = (long long)planes * h->p.nx * h->p.ny;
  with_types(h->p.dim, h->p.precision, [&](auto l, auto s) {
    using L = decltype(l);
    using S = decltype(s);
    using A = typename S::A;
    if constexpr (L::D == 3) {
      IbmArgs<S> a{};
      a.g = g;
      a.fin = (const typename S::T*)h->f[h->cur];
      a.rho_field = (const A*)h->rho_field;
      a.pull = h->poststream ? 0 : 1;
      k_halo_moments<L, S><<<flat_blocks(cnt, 256), 256, 0, h->stream>>>(a, side, planes, (A*)d_out);
    }
  });
  CK_LAUNCH();
  return COUPLB_OK;
}

int couplb_ibm_halo_fold(couplb_handle* h, int side, int planes, const void* d_in) {
  if (!h || !d_in) return fail(h, COUPLB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return fail(h, COUPLB_ERR_ARG, "halo side must be 0 (z low) or 1 (z high)");
  if (h->p.dim != 3) return fail(h, COUPLB_ERR_UNSUPPORTED, "halo faces are z faces of a D3Q19 lattice");
  if (planes < 1 || planes > (side ? 1 : 2) || planes > h->p.nz)
    return fail(h, COUPLB_ERR_ARG, "the neighbour below spreads onto 1 or 2 planes, the one above onto 1");
  int rc = set_device(h);
  if (rc) return rc;
  const Geom g = make_geom(h);
  const long long cnt = (long long)planes * h->p.nx * h->p.ny;
  with_types(h->p.dim, h->p.precision, [&](auto, auto s) {
    using A = typename decltype(s)::A;
    k_halo_fold<A><<<flat_blocks(cnt, 256), 256, 0, h->stream>>>(g, side, planes, (const A*)d_in, (A*)h->F,
                                                                  h->seg_force);
  });
  CK_LAUNCH();
  h->force_dirty = 1;
  return COUPLB_OK;
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
