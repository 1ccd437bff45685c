/*
 * ref_harness.cpp -- drives the reference's own CoupLB headers
 * (CoupLB/couplb_lattice.h, couplb_collision.h, couplb_streaming.h,
 * couplb_boundary.h, couplb_ibm.h, compiled unmodified from the reference
 * tree) behind the oracle API with prefix ref_ (TEST INFRASTRUCTURE ONLY).
 *
 * The grid layer below calls the reference classes directly.  The few loops
 * that live in fix_couplb.cpp (which needs LAMMPS and cannot be compiled
 * here) are restated: apply_external_force (fix_couplb.cpp:693-707),
 * enforce_wall_ghost_fields (:800-809) and the atom loop of
 * do_ibm_sub_coupling (:763-797).  The fix-level sequencing is the shared
 * restatement in oracle_fix.inc.
 *
 * Built by oracle/Makefile into oracle/_ref/libcouplb_ref.so.
 */
#define ORC_FN(x) ref_##x
#include "couplb_oracle.h"

#include "couplb_lattice.h"
#include "couplb_collision.h"
#include "couplb_streaming.h"
#include "couplb_boundary.h"
#include "couplb_ibm.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

using namespace LAMMPS_NS::CoupLB;

namespace {

struct RefGridBase {
  virtual ~RefGridBase() {}
  virtual long ntotal() = 0;
  virtual void init_eq(double, double, double, double) = 0;
  virtual void set_f(const double*) = 0;
  virtual void get_f(double*) = 0;
  virtual void get_macro(double*, double*, double*, double*) = 0;
  virtual void set_force(const double*, const double*, const double*) = 0;
  virtual void get_force(double*, double*, double*) = 0;
  virtual void lbm_step(const double*) = 0;
  virtual void macro(int) = 0;
  virtual void exch_vel() = 0;
  virtual void fold() = 0;
  virtual void diag(double*, int*) = 0;
  virtual int ibm(const couplb_ibm_params*, int, const double*, const double*,
                  const double*, const int*, double*, int, int) = 0;
};

template <class L>
struct RefGrid : RefGridBase {
  Grid<L> g;
  BGK<L> b;
  Streaming<L> s;

  RefGrid(int nx, int ny, int nz, double tau, double rho0, const int wall[6],
          const double wv[3]) {
    g.allocate(nx, ny, (L::D == 3) ? nz : 1, 1.0, 0, 0, 0, nx, ny, nz);
    g.init_equilibrium(rho0, 0, 0, 0);
    b.set_tau(tau);
    int pn[3][2] = {{0, 0}, {0, 0}, {0, 0}};     /* one rank: self */
    s.set_comm(MPI_COMM_WORLD);
    s.set_neighbors(pn);
    s.set_periodic(true, true, L::D == 3);
    s.set_nprocs(1, 1, 1);
    s.allocate_buffers(g, rho0);
    if (wall[0] || wall[1]) Boundary<L>::set_walls_x(g, wall[0] > 0, wall[1] > 0, wall[0], wall[1]);
    if (wall[2] || wall[3]) Boundary<L>::set_walls_y(g, wall[2] > 0, wall[3] > 0, wall[2], wall[3]);
    if (L::D == 3 && (wall[4] || wall[5]))
      Boundary<L>::set_walls_z(g, wall[4] > 0, wall[5] > 0, wall[4], wall[5]);
    Boundary<L>::set_wall_velocity(g, 2, wv[0], wv[1], (L::D == 3) ? wv[2] : 0.0);
    s.precompute_wall_flags(g);
  }

  long ntotal() override { return g.ntotal; }
  void init_eq(double r, double a, double bb, double c) override { g.init_equilibrium(r, a, bb, c); }
  void set_f(const double* f) override {
    std::memcpy(g.f.data(), f, sizeof(double) * g.f.size());
    g.f_buf = g.f;                  /* couplb_io.h:814 */
    g.compute_macroscopic(false);   /* couplb_io.h:817 */
  }
  void get_f(double* f) override { std::memcpy(f, g.f.data(), sizeof(double) * g.f.size()); }
  void get_macro(double* r, double* a, double* bb, double* c) override {
    const size_t by = sizeof(double) * g.ntotal;
    if (r) std::memcpy(r, g.rho.data(), by);
    if (a) std::memcpy(a, g.ux.data(), by);
    if (bb) std::memcpy(bb, g.uy.data(), by);
    if (c) std::memcpy(c, g.uz.data(), by);
  }
  void set_force(const double* a, const double* bb, const double* c) override {
    const size_t by = sizeof(double) * g.ntotal;
    std::memcpy(g.fx.data(), a, by); std::memcpy(g.fy.data(), bb, by); std::memcpy(g.fz.data(), c, by);
  }
  void get_force(double* a, double* bb, double* c) override {
    const size_t by = sizeof(double) * g.ntotal;
    std::memcpy(a, g.fx.data(), by); std::memcpy(bb, g.fy.data(), by); std::memcpy(c, g.fz.data(), by);
  }
  /* FixCoupLB::do_lbm_step (fix_couplb.cpp:659-669) */
  void lbm_step(const double* gl) override {
    if (gl && !(std::fabs(gl[0]) < Constants::ZERO_TOL && std::fabs(gl[1]) < Constants::ZERO_TOL &&
                std::fabs(gl[2]) < Constants::ZERO_TOL)) {
      const int klo = (L::D == 3) ? 1 : 0, khi = (L::D == 3) ? (g.gz - 2) : 0;
      for (int k = klo; k <= khi; k++)
        for (int j = 1; j <= g.gy - 2; j++)
          for (int i = 1; i <= g.gx - 2; i++) {
            const int n = g.idx(i, j, k);
            if (g.type[n] != 0) continue;
            g.fx[n] += gl[0] * g.rho[n]; g.fy[n] += gl[1] * g.rho[n]; g.fz[n] += gl[2] * g.rho[n];
          }
    }
    g.compute_macroscopic(true);
    b.collide(g);
    s.exchange(g);
    s.stream(g);
    for (int n = 0; n < g.ntotal; n++) {       /* fix_couplb.cpp:800-809 */
      if (g.type[n] == 1) { g.rho[n] = 1.0; g.ux[n] = g.uy[n] = g.uz[n] = 0; }
      else if (g.type[n] == 2) { g.rho[n] = 1.0; g.ux[n] = g.bc_ux[n]; g.uy[n] = g.bc_uy[n]; g.uz[n] = g.bc_uz[n]; }
      else if (g.type[n] == 3) { g.rho[n] = 1.0; g.ux[n] = g.uy[n] = g.uz[n] = 0; }
    }
    g.clear_forces();
  }
  void macro(int guo) override { g.compute_macroscopic(guo != 0); }
  void exch_vel() override { s.exchange_velocity(g); }
  void fold() override { s.exchange_forces(g); }
  void diag(double* out, int* clamps) override {
    out[0] = g.max_velocity();
    g.compute_diagnostics(out[1], out[2], out[3], out[4]);
    if (clamps) *clamps = g.rho_clamp_count;
  }
  /* atom loop of FixCoupLB::do_ibm_sub_coupling (fix_couplb.cpp:755-797) */
  int ibm(const couplb_ibm_params* ip, int n, const double* x, const double* v,
          const double* mass, const int* active, double* f_add, int refresh,
          int fold_now) override {
    if (refresh) { g.compute_macroscopic(false); s.exchange_velocity(g); }
    const DeltaKernel kern = ip->delta == COUPLB_DELTA_ROMA ? DeltaKernel::ROMA : DeltaKernel::PESKIN4;
    const double inv_dx = 1.0 / ip->dx;
    const double xi_over_dtLBM = ip->xi_ibm / ip->dt_lbm;
    const double inv_N = 1.0 / static_cast<double>(ip->md_per_lb);
    const double dv = (L::D == 3) ? (ip->dx * ip->dx * ip->dx) : (ip->dx * ip->dx);
    int nc = 0;
    for (int a = 0; a < n; a++) {
      if (active && !active[a]) continue;
      nc++;
      auto uf = IBM<L>::interpolate(g, x[3*a], x[3*a+1], x[3*a+2], ip->domain_lo, inv_dx, kern);
      const double m = mass[a];
      const double fxi = m * xi_over_dtLBM * (uf[0]*ip->vel_scale - v[3*a]);
      const double fyi = m * xi_over_dtLBM * (uf[1]*ip->vel_scale - v[3*a+1]);
      const double fzi = m * xi_over_dtLBM * (uf[2]*ip->vel_scale - v[3*a+2]);
      f_add[3*a] += fxi; f_add[3*a+1] += fyi; f_add[3*a+2] += fzi;
      IBM<L>::spread(g, x[3*a], x[3*a+1], x[3*a+2],
                     -fxi * inv_N / ip->force_scale, -fyi * inv_N / ip->force_scale,
                     -fzi * inv_N / ip->force_scale, dv, ip->domain_lo, inv_dx, ip->dx, kern);
    }
    if (fold_now) s.exchange_forces(g);
    return nc;
  }
};

inline RefGridBase* G(void* p) { return static_cast<RefGridBase*>(p); }

}  // namespace

extern "C" {

void* ref_grid_create(int dim, int nx, int ny, int nz, double tau, double rho0,
                      const int wall[6], const double wall_vel[3]) {
  if (dim == 3) return static_cast<RefGridBase*>(new RefGrid<D3Q19>(nx, ny, nz, tau, rho0, wall, wall_vel));
  return static_cast<RefGridBase*>(new RefGrid<D2Q9>(nx, ny, 1, tau, rho0, wall, wall_vel));
}
void ref_grid_destroy(void* g) { delete G(g); }
long ref_grid_ntotal(void* g) { return G(g)->ntotal(); }
void ref_grid_init_equilibrium(void* g, double r, double a, double b, double c) { G(g)->init_eq(r, a, b, c); }
void ref_grid_set_f(void* g, const double* f) { G(g)->set_f(f); }
void ref_grid_get_f(void* g, double* f) { G(g)->get_f(f); }
void ref_grid_get_macro(void* g, double* r, double* a, double* b, double* c) { G(g)->get_macro(r, a, b, c); }
void ref_grid_set_force(void* g, const double* a, const double* b, const double* c) { G(g)->set_force(a, b, c); }
void ref_grid_get_force(void* g, double* a, double* b, double* c) { G(g)->get_force(a, b, c); }
void ref_grid_lbm_step(void* g, const double* gl) { G(g)->lbm_step(gl); }
void ref_grid_macroscopic(void* g, int guo) { G(g)->macro(guo); }
void ref_grid_exchange_velocity(void* g) { G(g)->exch_vel(); }
void ref_grid_fold_forces(void* g) { G(g)->fold(); }
void ref_grid_diagnostics(void* g, double out[5], int* clamps) { G(g)->diag(out, clamps); }
int ref_grid_ibm_substep(void* g, const couplb_ibm_params* ip, int n, const double* x,
                         const double* v, const double* mass, const int* active,
                         double* f_add, int refresh, int fold) {
  return G(g)->ibm(ip, n, x, v, mass, active, f_add, refresh, fold);
}

}  // extern "C"

#include "oracle_fix.inc"
