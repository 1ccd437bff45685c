/*
 * couplb_oracle.c -- plain-C restatement of CoupLB's per-timestep LBM + IBM
 * path, used ONLY as the checker of the CUDA implementation (tests/,
 * __graft_entry__.smoke(), bench.py's CPU-baseline leg).  It is never linked
 * into or called by the product library.
 *
 * Each function names the reference code it follows (paths relative to the
 * CoupLB source tree).  Arithmetic is kept in the reference's operation order
 * so that, compiled without FMA contraction, it reproduces the reference
 * bit for bit; tests/test_oracle_pin.py checks this against the reference's
 * own headers (oracle/_ref) and against committed golden vectors.
 *
 * One subdomain = the whole box (one MPI rank in the reference).  With one
 * rank every non-wall face exchanges with itself, so the MPI ghost exchange
 * (couplb_streaming.h:136-245) becomes the face copies below.
 */
#include "couplb_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- constants (couplb_lattice.h:13-20) ----------------------------- */
#define RHO_MIN        1e-10
#define DELTA_TOL      1e-12
#define ZERO_TOL       1e-15
#define RHO_CLAMP_FRAC 0.1
#define MA_WARN        0.3
#define MA_ERROR       0.5

/* ---- lattice descriptors (couplb_lattice.h:24-75) ------------------- */
static const int E9[9][3] = {{0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},
                             {1,1,0},{-1,-1,0},{1,-1,0},{-1,1,0}};
static const double W9[9] = {4.0/9.0, 1.0/9.0, 1.0/9.0, 1.0/9.0, 1.0/9.0,
                             1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0};
static const int OPP9[9] = {0,2,1,4,3,6,5,8,7};
static const int REFL9[3][9] = {{0,2,1,3,4,8,7,6,5},
                                {0,1,2,4,3,7,8,5,6},
                                {0,1,2,3,4,5,6,7,8}};
static const int E19[19][3] = {{0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},
                               {0,0,1},{0,0,-1},{1,1,0},{-1,-1,0},{1,-1,0},
                               {-1,1,0},{1,0,1},{-1,0,-1},{1,0,-1},{-1,0,1},
                               {0,1,1},{0,-1,-1},{0,1,-1},{0,-1,1}};
static const double W19[19] = {1.0/3.0, 1.0/18.0, 1.0/18.0, 1.0/18.0,
                               1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/36.0,
                               1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0,
                               1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0,
                               1.0/36.0, 1.0/36.0, 1.0/36.0};
static const int OPP19[19] = {0,2,1,4,3,6,5,8,7,10,9,12,11,14,13,16,15,18,17};
static const int REFL19[3][19] = {
  {0,2,1,3,4,5,6,10,9,8,7,14,13,12,11,15,16,17,18},
  {0,1,2,4,3,5,6,9,10,7,8,11,12,13,14,18,17,16,15},
  {0,1,2,3,4,6,5,7,8,9,10,13,14,11,12,17,18,15,16}};
static const double CS2 = 1.0 / 3.0;

typedef struct orc_grid {
  int D, Q;
  const int (*e)[3];
  const double* w;
  const int* opp;
  const int* refl;      /* refl[d*Q + q] */
  int nx, ny, nz, gx, gy, gz, ntotal;
  double *f, *f_buf, *rho, *ux, *uy, *uz, *fx, *fy, *fz;
  double *bc_ux, *bc_uy, *bc_uz;
  int *type, *wall_dim;
  int rho_clamp_count;
  double tau, omega, rho0;
  int wall_face[3][2];
  int ibm_wrap;         /* bit d: IBM window wrapped periodically along axis d */
} orc_grid;

static inline int gidx(const orc_grid* g, int i, int j, int k) {
  return i + g->gx * (j + g->gy * k);
}
#define FI(g, q, n)   ((g)->f[(size_t)(q) * (g)->ntotal + (n)])
#define FB(g, q, n)   ((g)->f_buf[(size_t)(q) * (g)->ntotal + (n)])

/* Grid::feq (couplb_lattice.h:137-144) */
static double feq(const orc_grid* g, int q, double r, double u0, double u1,
                  double u2) {
  const double eu = g->e[q][0]*u0 + g->e[q][1]*u1 + g->e[q][2]*u2;
  const double uu = u0*u0 + u1*u1 + u2*u2;
  const double cs4 = CS2 * CS2;
  return g->w[q] * r * (1.0 + eu/CS2 + 0.5*eu*eu/cs4 - 0.5*uu/CS2);
}

/* Grid::init_equilibrium (couplb_lattice.h:145-154) */
void ORC_FN(grid_init_equilibrium)(void* gp, double r0, double ux0, double uy0,
                                   double uz0) {
  orc_grid* g = (orc_grid*)gp;
  for (int n = 0; n < g->ntotal; n++) {
    g->rho[n] = r0;
    g->ux[n] = ux0; g->uy[n] = uy0; g->uz[n] = uz0;
    g->fx[n] = g->fy[n] = g->fz[n] = 0.0;
    for (int q = 0; q < g->Q; q++) FI(g, q, n) = feq(g, q, r0, ux0, uy0, uz0);
  }
  memcpy(g->f_buf, g->f, sizeof(double) * (size_t)g->Q * g->ntotal);
}

/* Boundary::set_walls_x/y/z (couplb_boundary.h:12-35) */
static void set_walls(orc_grid* g, int d, int lo, int hi, int tlo, int thi) {
  const int ext[3] = {g->gx, g->gy, g->gz};
  for (int side = 0; side < 2; side++) {
    if (!(side ? hi : lo)) continue;
    const int pos = side ? ext[d] - 1 : 0;
    for (int k = 0; k < g->gz; k++)
      for (int j = 0; j < g->gy; j++)
        for (int i = 0; i < g->gx; i++) {
          const int c[3] = {i, j, k};
          if (c[d] != pos) continue;
          const int n = gidx(g, i, j, k);
          g->type[n] = side ? thi : tlo;
          g->wall_dim[n] = d;
        }
  }
}

/* Streaming::has_wall_on_face (couplb_streaming.h:163-169) */
static int has_wall_on_face(const orc_grid* g, int d, int pos) {
  for (int k = 0; k < g->gz; k++)
    for (int j = 0; j < g->gy; j++)
      for (int i = 0; i < g->gx; i++) {
        const int c[3] = {i, j, k};
        if (c[d] != pos) continue;
        if (g->type[gidx(g, i, j, k)] == 0) return 0;
      }
  return 1;
}

/* Grid::allocate + init_equilibrium(rho0) + BGK::set_tau + setup_boundaries
 * + precompute_wall_flags (couplb_lattice.h:105-123, fix_couplb.cpp:501-539,
 * couplb_streaming.h:74-80).  In 2D only x and y walls are applied
 * (fix_couplb.cpp:533-537). */
void* ORC_FN(grid_create)(int dim, int nx, int ny, int nz, double tau,
                          double rho0, const int wall[6],
                          const double wall_vel[3]) {
  orc_grid* g = (orc_grid*)calloc(1, sizeof(orc_grid));
  g->D = dim;
  if (dim == 3) { g->Q = 19; g->e = E19; g->w = W19; g->opp = OPP19; g->refl = &REFL19[0][0]; }
  else          { g->Q = 9;  g->e = E9;  g->w = W9;  g->opp = OPP9;  g->refl = &REFL9[0][0]; }
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->gx = nx + 2; g->gy = ny + 2; g->gz = (dim == 3) ? nz + 2 : 1;
  g->ntotal = g->gx * g->gy * g->gz;
  const size_t G = (size_t)g->ntotal, QG = (size_t)g->Q * G;
  g->f = (double*)calloc(QG, sizeof(double));
  g->f_buf = (double*)calloc(QG, sizeof(double));
  g->rho = (double*)calloc(G, sizeof(double));
  g->ux = (double*)calloc(G, sizeof(double));
  g->uy = (double*)calloc(G, sizeof(double));
  g->uz = (double*)calloc(G, sizeof(double));
  g->fx = (double*)calloc(G, sizeof(double));
  g->fy = (double*)calloc(G, sizeof(double));
  g->fz = (double*)calloc(G, sizeof(double));
  g->bc_ux = (double*)calloc(G, sizeof(double));
  g->bc_uy = (double*)calloc(G, sizeof(double));
  g->bc_uz = (double*)calloc(G, sizeof(double));
  g->type = (int*)calloc(G, sizeof(int));
  g->wall_dim = (int*)malloc(G * sizeof(int));
  for (size_t n = 0; n < G; n++) { g->rho[n] = 1.0; g->wall_dim[n] = -1; }
  g->rho0 = rho0;
  ORC_FN(grid_init_equilibrium)(g, rho0, 0, 0, 0);
  g->tau = tau; g->omega = 1.0 / tau;
  const int nd = (dim == 3) ? 3 : 2;
  for (int d = 0; d < nd; d++) {
    const int tlo = wall[2*d], thi = wall[2*d + 1];
    if (tlo || thi) set_walls(g, d, tlo > 0, thi > 0, tlo, thi);
  }
  const double wv[3] = {wall_vel[0], wall_vel[1], dim == 3 ? wall_vel[2] : 0.0};
  for (int n = 0; n < g->ntotal; n++)
    if (g->type[n] == 2) { g->bc_ux[n] = wv[0]; g->bc_uy[n] = wv[1]; g->bc_uz[n] = wv[2]; }
  for (int d = 0; d < 3; d++) g->wall_face[d][0] = g->wall_face[d][1] = 0;
  for (int d = 0; d < nd; d++) {
    const int ext = d == 0 ? g->gx : d == 1 ? g->gy : g->gz;
    g->wall_face[d][0] = has_wall_on_face(g, d, 0);
    g->wall_face[d][1] = has_wall_on_face(g, d, ext - 1);
  }
  return g;
}

void ORC_FN(grid_destroy)(void* gp) {
  orc_grid* g = (orc_grid*)gp;
  if (!g) return;
  free(g->f); free(g->f_buf); free(g->rho); free(g->ux); free(g->uy); free(g->uz);
  free(g->fx); free(g->fy); free(g->fz); free(g->bc_ux); free(g->bc_uy);
  free(g->bc_uz); free(g->type); free(g->wall_dim); free(g);
}

long ORC_FN(grid_ntotal)(void* gp) { return ((orc_grid*)gp)->ntotal; }

/* Grid::compute_macroscopic (couplb_lattice.h:155-202) */
void ORC_FN(grid_macroscopic)(void* gp, int guo) {
  orc_grid* g = (orc_grid*)gp;
  const int klo = (g->D == 3) ? 1 : 0, khi = (g->D == 3) ? g->gz - 2 : 0;
  int clamps = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+:clamps)
  for (int k = klo; k <= khi; k++)
    for (int j = 1; j <= g->gy - 2; j++)
      for (int i = 1; i <= g->gx - 2; i++) {
        const int n = gidx(g, i, j, k);
        if (g->type[n] != 0) continue;
        double r = 0.0, su = 0.0, sv = 0.0, sw = 0.0;
        for (int q = 0; q < g->Q; q++) {
          const double fv = FI(g, q, n);
          r  += fv;
          su += g->e[q][0] * fv;
          sv += g->e[q][1] * fv;
          sw += g->e[q][2] * fv;
        }
        if (r <= RHO_MIN) { r = RHO_MIN; clamps++; }
        if (!isfinite(r)) { r = RHO_MIN; clamps++; }
        g->rho[n] = r;
        const double inv_r = 1.0 / r;
        if (guo) {
          g->ux[n] = (su + 0.5 * g->fx[n]) * inv_r;
          g->uy[n] = (sv + 0.5 * g->fy[n]) * inv_r;
          g->uz[n] = (sw + 0.5 * g->fz[n]) * inv_r;
        } else {
          g->ux[n] = su * inv_r;
          g->uy[n] = sv * inv_r;
          g->uz[n] = sw * inv_r;
        }
      }
  g->rho_clamp_count = clamps;
}

/* BGK::collide (couplb_collision.h:18-62) */
static void collide(orc_grid* g) {
  const double cs4 = CS2 * CS2;
  const double om = g->omega, half_om = 1.0 - 0.5 * om;
  const int klo = (g->D == 3) ? 1 : 0, khi = (g->D == 3) ? g->gz - 2 : 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = klo; k <= khi; k++)
    for (int j = 1; j <= g->gy - 2; j++)
      for (int i = 1; i <= g->gx - 2; i++) {
        const int n = gidx(g, i, j, k);
        if (g->type[n] != 0) continue;
        const double r = g->rho[n];
        const double u0 = g->ux[n], u1 = g->uy[n], u2 = g->uz[n];
        const double f0 = g->fx[n], f1 = g->fy[n], f2 = g->fz[n];
        const double uu = u0*u0 + u1*u1 + u2*u2;
        const double uf = u0*f0 + u1*f1 + u2*f2;
        for (int q = 0; q < g->Q; q++) {
          const double cx = g->e[q][0], cy = g->e[q][1], cz = g->e[q][2];
          const double w = g->w[q];
          const double eu = cx*u0 + cy*u1 + cz*u2;
          const double ef = cx*f0 + cy*f1 + cz*f2;
          const double fe = w * r * (1.0 + eu/CS2 + 0.5*eu*eu/cs4 - 0.5*uu/CS2);
          const double Si = w * half_om * ((ef - uf)/CS2 + eu*ef/cs4);
          FI(g, q, n) += -om * (FI(g, q, n) - fe) + Si;
        }
      }
}

/* Face iteration over the full ghost-inclusive extent of the other dims
 * (couplb_streaming.h:281-293): calls fn(src, dst) for every node of plane
 * s -> plane t along dim d. */
#define FACE_LOOP(g, d, s, t, BODY)                                            \
  do {                                                                         \
    if ((d) == 0) { for (int k_ = 0; k_ < (g)->gz; k_++) for (int j_ = 0; j_ < (g)->gy; j_++) { \
        const int sn = gidx(g, s, j_, k_), dn = gidx(g, t, j_, k_); BODY; } } \
    else if ((d) == 1) { for (int k_ = 0; k_ < (g)->gz; k_++) for (int i_ = 0; i_ < (g)->gx; i_++) { \
        const int sn = gidx(g, i_, s, k_), dn = gidx(g, i_, t, k_); BODY; } } \
    else { for (int j_ = 0; j_ < (g)->gy; j_++) for (int i_ = 0; i_ < (g)->gx; i_++) { \
        const int sn = gidx(g, i_, j_, s), dn = gidx(g, i_, j_, t); BODY; } } \
  } while (0)

static int dim_ext(const orc_grid* g, int d) {
  return d == 0 ? g->gx : d == 1 ? g->gy : g->gz;
}

/* Streaming::exchange with one rank (couplb_streaming.h:136-139, 176-194):
 * ghost_lo <- interior hi face, ghost_hi <- interior lo face, unless the
 * ghost face is all wall. */
static void exchange_f(orc_grid* g) {
  const int nd = (g->D == 3) ? 3 : 2;
  for (int d = 0; d < nd; d++) {
    const int ds = dim_ext(g, d), lf = 1, hf = ds - 2, gl = 0, gh = ds - 1;
    if (!g->wall_face[d][0])
      FACE_LOOP(g, d, hf, gl, for (int q = 0; q < g->Q; q++) FI(g, q, dn) = FI(g, q, sn));
    if (!g->wall_face[d][1])
      FACE_LOOP(g, d, lf, gh, for (int q = 0; q < g->Q; q++) FI(g, q, dn) = FI(g, q, sn));
  }
}

/* Streaming::exchange_velocity with one rank (couplb_streaming.h:140-143,
 * 196-214). */
void ORC_FN(grid_exchange_velocity)(void* gp) {
  orc_grid* g = (orc_grid*)gp;
  const int nd = (g->D == 3) ? 3 : 2;
  for (int d = 0; d < nd; d++) {
    const int ds = dim_ext(g, d), lf = 1, hf = ds - 2, gl = 0, gh = ds - 1;
    if (!g->wall_face[d][0])
      FACE_LOOP(g, d, hf, gl, { g->rho[dn] = g->rho[sn]; g->ux[dn] = g->ux[sn];
                                g->uy[dn] = g->uy[sn]; g->uz[dn] = g->uz[sn]; });
    if (!g->wall_face[d][1])
      FACE_LOOP(g, d, lf, gh, { g->rho[dn] = g->rho[sn]; g->ux[dn] = g->ux[sn];
                                g->uy[dn] = g->uy[sn]; g->uz[dn] = g->uz[sn]; });
  }
}

/* Streaming::exchange_forces with one rank (couplb_streaming.h:155-158,
 * 217-245): ghost_lo forces are added onto the interior hi face and ghost_hi
 * onto the interior lo face, x then y then z. */
static void exchange_forces(orc_grid* g) {
  const int nd = (g->D == 3) ? 3 : 2;
  for (int d = 0; d < nd; d++) {
    const int ds = dim_ext(g, d), lf = 1, hf = ds - 2, gl = 0, gh = ds - 1;
    FACE_LOOP(g, d, gl, hf, { g->fx[dn] += g->fx[sn]; g->fy[dn] += g->fy[sn];
                              g->fz[dn] += g->fz[sn]; });
    FACE_LOOP(g, d, gh, lf, { g->fx[dn] += g->fx[sn]; g->fy[dn] += g->fy[sn];
                              g->fz[dn] += g->fz[sn]; });
  }
}

/* Streaming::stream (couplb_streaming.h:82-134): pull from x - e_q with the
 * rule of the source node's type, then swap f and f_buf. */
static void stream(orc_grid* g) {
  const double a = RHO_CLAMP_FRAC * g->rho0;
  const double rho_floor = (a < RHO_MIN) ? RHO_MIN : a;     /* std::max */
  const int klo = (g->D == 3) ? 1 : 0, khi = (g->D == 3) ? g->gz - 2 : 0;
  const int Q = g->Q;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = klo; k <= khi; k++)
    for (int j = 1; j <= g->gy - 2; j++)
      for (int i = 1; i <= g->gx - 2; i++) {
        const int n = gidx(g, i, j, k);
        if (g->type[n] != 0) continue;
        for (int q = 0; q < Q; q++) {
          const int si = i - g->e[q][0], sj = j - g->e[q][1], sk = k - g->e[q][2];
          if (si < 0 || si >= g->gx || sj < 0 || sj >= g->gy ||
              (g->D == 3 && (sk < 0 || sk >= g->gz))) {
            FB(g, q, n) = FI(g, q, n);
            continue;
          }
          const int sn = gidx(g, si, sj, sk);
          const int st = g->type[sn];
          if (st == 0) {
            FB(g, q, n) = FI(g, q, sn);
          } else if (st == 1) {
            FB(g, q, n) = FI(g, g->opp[q], n);
          } else if (st == 2) {
            const int qo = g->opp[q];
            const double eu = g->e[q][0]*g->bc_ux[sn] + g->e[q][1]*g->bc_uy[sn]
                            + g->e[q][2]*g->bc_uz[sn];
            const double rn = g->rho[n];
            const double rw = (rn < rho_floor) ? rho_floor : rn;   /* std::max */
            FB(g, q, n) = FI(g, qo, n) + 2.0*g->w[qo]*rw*eu/CS2;
          } else if (st == 3) {
            FB(g, q, n) = FI(g, g->refl[g->wall_dim[sn] * Q + q], n);
          } else if (st == 4) {
            FB(g, q, n) = FI(g, q, n);
          }
        }
      }
  double* t = g->f; g->f = g->f_buf; g->f_buf = t;
}

/* FixCoupLB::enforce_wall_ghost_fields (fix_couplb.cpp:800-809), rho_lb = 1 */
static void enforce_wall_ghost_fields(orc_grid* g) {
  for (int n = 0; n < g->ntotal; n++) {
    if (g->type[n] == 1) { g->rho[n] = 1.0; g->ux[n] = g->uy[n] = g->uz[n] = 0; }
    else if (g->type[n] == 2) { g->rho[n] = 1.0; g->ux[n] = g->bc_ux[n];
                                g->uy[n] = g->bc_uy[n]; g->uz[n] = g->bc_uz[n]; }
    else if (g->type[n] == 3) { g->rho[n] = 1.0; g->ux[n] = g->uy[n] = g->uz[n] = 0; }
  }
}

/* Grid::clear_forces (couplb_lattice.h:243-247) */
static void clear_forces(orc_grid* g) {
  memset(g->fx, 0, sizeof(double) * g->ntotal);
  memset(g->fy, 0, sizeof(double) * g->ntotal);
  memset(g->fz, 0, sizeof(double) * g->ntotal);
}

/* The grid part of FixCoupLB::apply_external_force (fix_couplb.cpp:693-707):
 * g_lb already in lattice units; skipped when every |g| < ZERO_TOL.  It reads
 * rho[] as left by the last compute_macroscopic. */
static void apply_external_force(orc_grid* g, const double* gl) {
  if (!gl) return;
  if (fabs(gl[0]) < ZERO_TOL && fabs(gl[1]) < ZERO_TOL && fabs(gl[2]) < ZERO_TOL)
    return;
  const int klo = (g->D == 3) ? 1 : 0, khi = (g->D == 3) ? g->gz - 2 : 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = klo; k <= khi; k++)
    for (int j = 1; j <= g->gy - 2; j++)
      for (int i = 1; i <= g->gx - 2; i++) {
        const int n = gidx(g, i, j, k);
        if (g->type[n] != 0) continue;
        g->fx[n] += gl[0] * g->rho[n];
        g->fy[n] += gl[1] * g->rho[n];
        g->fz[n] += gl[2] * g->rho[n];
      }
}

/* FixCoupLB::do_lbm_step (fix_couplb.cpp:659-669) */
void ORC_FN(grid_lbm_step)(void* gp, const double* g_lb) {
  orc_grid* g = (orc_grid*)gp;
  apply_external_force(g, g_lb);
  ORC_FN(grid_macroscopic)(g, 1);
  collide(g);
  exchange_f(g);
  stream(g);
  enforce_wall_ghost_fields(g);
  clear_forces(g);
}

void ORC_FN(grid_set_f)(void* gp, const double* f) {
  orc_grid* g = (orc_grid*)gp;
  const size_t QG = (size_t)g->Q * g->ntotal;
  memcpy(g->f, f, QG * sizeof(double));
  memcpy(g->f_buf, f, QG * sizeof(double));      /* couplb_io.h:814 */
  ORC_FN(grid_macroscopic)(g, 0);                /* couplb_io.h:817 */
}

void ORC_FN(grid_get_f)(void* gp, double* f) {
  orc_grid* g = (orc_grid*)gp;
  memcpy(f, g->f, sizeof(double) * (size_t)g->Q * g->ntotal);
}

void ORC_FN(grid_get_macro)(void* gp, double* rho, double* ux, double* uy,
                            double* uz) {
  orc_grid* g = (orc_grid*)gp;
  const size_t b = sizeof(double) * g->ntotal;
  if (rho) memcpy(rho, g->rho, b);
  if (ux) memcpy(ux, g->ux, b);
  if (uy) memcpy(uy, g->uy, b);
  if (uz) memcpy(uz, g->uz, b);
}

void ORC_FN(grid_set_force)(void* gp, const double* fx, const double* fy,
                            const double* fz) {
  orc_grid* g = (orc_grid*)gp;
  const size_t b = sizeof(double) * g->ntotal;
  memcpy(g->fx, fx, b); memcpy(g->fy, fy, b); memcpy(g->fz, fz, b);
}

void ORC_FN(grid_get_force)(void* gp, double* fx, double* fy, double* fz) {
  orc_grid* g = (orc_grid*)gp;
  const size_t b = sizeof(double) * g->ntotal;
  memcpy(fx, g->fx, b); memcpy(fy, g->fy, b); memcpy(fz, g->fz, b);
}

/* Grid::max_velocity + compute_diagnostics + rho_clamp_count
 * (couplb_lattice.h:203-242, 100) */
void ORC_FN(grid_diagnostics)(void* gp, double out[5], int* clamps) {
  orc_grid* g = (orc_grid*)gp;
  const int klo = (g->D == 3) ? 1 : 0, khi = (g->D == 3) ? g->gz - 2 : 0;
  double umax2 = 0.0, mass = 0.0, px = 0.0, py = 0.0, pz = 0.0;
  for (int k = klo; k <= khi; k++)
    for (int j = 1; j <= g->gy - 2; j++)
      for (int i = 1; i <= g->gx - 2; i++) {
        const int n = gidx(g, i, j, k);
        if (g->type[n] != 0) continue;
        const double u2 = g->ux[n]*g->ux[n] + g->uy[n]*g->uy[n] + g->uz[n]*g->uz[n];
        if (u2 > umax2) umax2 = u2;
        mass += g->rho[n];
        px += g->rho[n] * g->ux[n];
        py += g->rho[n] * g->uy[n];
        pz += g->rho[n] * g->uz[n];
      }
  out[0] = sqrt(umax2); out[1] = mass; out[2] = px; out[3] = py; out[4] = pz;
  if (clamps) *clamps = g->rho_clamp_count;
}

/* ---- IBM (couplb_ibm.h) --------------------------------------------- */

/* delta_roma (couplb_ibm.h:11-22) */
static double delta_roma(double r) {
  const double ar = fabs(r);
  if (ar <= 0.5) {
    const double a = 1.0 - 3.0*r*r;
    return (1.0 + sqrt(a > 0.0 ? a : 0.0)) / 3.0;
  }
  if (ar <= 1.5) {
    const double a = -2.0 + 6.0*ar - 3.0*r*r;
    return (5.0 - 3.0*ar - sqrt(a > 0.0 ? a : 0.0)) / 6.0;
  }
  return 0.0;
}

/* delta_peskin4 (couplb_ibm.h:24-35) */
static double delta_peskin4(double r) {
  const double ar = fabs(r);
  if (ar <= 1.0) {
    const double a = 1.0 + 4.0*ar - 4.0*ar*ar;
    return (3.0 - 2.0*ar + sqrt(a > 0.0 ? a : 0.0)) / 8.0;
  }
  if (ar <= 2.0) {
    const double a = -7.0 + 12.0*ar - 4.0*ar*ar;
    return (5.0 - 2.0*ar - sqrt(a > 0.0 ? a : 0.0)) / 8.0;
  }
  return 0.0;
}

/* IBM::delta_product (couplb_ibm.h:42-45) */
static double delta_product(const orc_grid* g, int kern, double rx, double ry,
                            double rz) {
  double (*d)(double) = (kern == COUPLB_DELTA_ROMA) ? delta_roma : delta_peskin4;
  return d(rx) * d(ry) * ((g->D == 3) ? d(rz) : 1.0);
}

/* IBM::phys_to_local (couplb_ibm.h:49-55) */
static void phys_to_local(const orc_grid* g, const couplb_ibm_params* ip,
                          double inv_dx, double xp, double yp, double zp,
                          double* lx, double* ly, double* lz) {
  *lx = (xp - ip->domain_lo[0]) * inv_dx - ip->offset[0] + 1.0;
  *ly = (yp - ip->domain_lo[1]) * inv_dx - ip->offset[1] + 1.0;
  *lz = (g->D == 3) ? ((zp - ip->domain_lo[2]) * inv_dx - ip->offset[2] + 1.0) : 0.0;
}

/* Window index i along an axis of g ghost-inclusive nodes (n interior):
 * the reference clips the window to [0, g) (couplb_ibm.h:64-73, 110-115);
 * with the wrap option (no reference counterpart) an axis whose faces are
 * both periodic maps i to the interior image 1 + (i - 1 mod n).  Returns 0
 * when the node is outside. */
static int window_index(int wrap, int i, int g, int n, int* out) {
  if (wrap) {
    int m = (i - 1) % n;
    if (m < 0) m += n;
    *out = m + 1;
    return 1;
  }
  *out = i;
  return i >= 0 && i < g;
}

void ORC_FN(grid_set_ibm_wrap)(void* gp, int mask) { ((orc_grid*)gp)->ibm_wrap = mask; }

/* IBM::interpolate (couplb_ibm.h:57-90) */
static void interpolate(const orc_grid* g, const couplb_ibm_params* ip,
                        double inv_dx, double xp, double yp, double zp,
                        double out[3]) {
  double lx, ly, lz;
  phys_to_local(g, ip, inv_dx, xp, yp, zp, &lx, &ly, &lz);
  const int i0 = (int)floor(lx), j0 = (int)floor(ly);
  const int k0 = (g->D == 3) ? (int)floor(lz) : 0;
  double ui = 0, vi = 0, wi = 0, ws = 0;
  for (int k = (g->D == 3 ? k0 - 1 : 0); k <= (g->D == 3 ? k0 + 2 : 0); k++) {
    int kw = k;
    if (g->D == 3 && !window_index(g->ibm_wrap & 4, k, g->gz, g->nz, &kw)) continue;
    for (int j = j0 - 1; j <= j0 + 2; j++) {
      int jw;
      if (!window_index(g->ibm_wrap & 2, j, g->gy, g->ny, &jw)) continue;
      for (int i = i0 - 1; i <= i0 + 2; i++) {
        int iw;
        if (!window_index(g->ibm_wrap & 1, i, g->gx, g->nx, &iw)) continue;
        const int n = gidx(g, iw, jw, kw);
        const int nt = g->type[n];
        const double d = delta_product(g, ip->delta, lx - i, ly - j, lz - k);
        if (nt == 0) { ui += g->ux[n]*d; vi += g->uy[n]*d; wi += g->uz[n]*d; ws += d; }
        else if (nt == 1) { ws += d; }
        else if (nt == 2) { ui += g->bc_ux[n]*d; vi += g->bc_uy[n]*d; wi += g->bc_uz[n]*d; ws += d; }
        else if (nt == 3) { ws += d; }
      }
    }
  }
  if (ws > DELTA_TOL) {
    const double iw = 1.0 / ws;
    out[0] = ui*iw; out[1] = vi*iw; out[2] = wi*iw;
  } else {
    out[0] = out[1] = out[2] = 0.0;
  }
}

/* IBM::spread (couplb_ibm.h:92-133) */
static void spread(orc_grid* g, const couplb_ibm_params* ip, double inv_dx,
                   double xp, double yp, double zp, double fxl, double fyl,
                   double fzl, double dvl) {
  double lx, ly, lz;
  phys_to_local(g, ip, inv_dx, xp, yp, zp, &lx, &ly, &lz);
  const int i0 = (int)floor(lx), j0 = (int)floor(ly);
  const int k0 = (g->D == 3) ? (int)floor(lz) : 0;
  const double dxp = ip->dx;
  const double cell_vol = dxp * dxp * ((g->D == 3) ? dxp : 1.0);
  const double dvr = dvl / cell_vol;
  double ws = 0.0, dcache[64];
  int ncache[64], nc = 0;
  for (int k = (g->D == 3 ? k0 - 1 : 0); k <= (g->D == 3 ? k0 + 2 : 0); k++) {
    int kw = k;
    if (g->D == 3 && !window_index(g->ibm_wrap & 4, k, g->gz, g->nz, &kw)) continue;
    for (int j = j0 - 1; j <= j0 + 2; j++) {
      int jw;
      if (!window_index(g->ibm_wrap & 2, j, g->gy, g->ny, &jw)) continue;
      for (int i = i0 - 1; i <= i0 + 2; i++) {
        int iw;
        if (!window_index(g->ibm_wrap & 1, i, g->gx, g->nx, &iw)) continue;
        const int n = gidx(g, iw, jw, kw);
        if (g->type[n] != 0) continue;
        const double d = delta_product(g, ip->delta, lx - i, ly - j, lz - k);
        dcache[nc] = d; ncache[nc] = n; nc++;
        ws += d;
      }
    }
  }
  if (ws < DELTA_TOL) return;
  const double sc = dvr / ws;
  for (int c = 0; c < nc; c++) {
    const double w = dcache[c] * sc;
    g->fx[ncache[c]] += fxl * w;
    g->fy[ncache[c]] += fyl * w;
    g->fz[ncache[c]] += fzl * w;
  }
}

/* The per-atom part of FixCoupLB::do_ibm_sub_coupling (fix_couplb.cpp:
 * 755-797).  refresh: macroscopic(false) + exchange_velocity (:757-760);
 * fold: exchange_forces (:795-797).  Returns the number of coupled atoms. */
int ORC_FN(grid_ibm_substep)(void* gp, const couplb_ibm_params* ip, int n,
                             const double* x, const double* v,
                             const double* mass, const int* active,
                             double* f_add, int refresh, int fold) {
  orc_grid* g = (orc_grid*)gp;
  if (refresh) {
    ORC_FN(grid_macroscopic)(g, 0);
    ORC_FN(grid_exchange_velocity)(g);
  }
  const double inv_dx = 1.0 / ip->dx;
  const double xi_over_dtLBM = ip->xi_ibm / ip->dt_lbm;
  const double inv_N = 1.0 / (double)ip->md_per_lb;
  const double dv = (g->D == 3) ? (ip->dx * ip->dx * ip->dx) : (ip->dx * ip->dx);
  const double vs = ip->vel_scale, fs = ip->force_scale;
  int nc = 0;
  for (int a = 0; a < n; a++) {
    if (active && !active[a]) continue;
    nc++;
    double uf[3];
    interpolate(g, ip, inv_dx, x[3*a], x[3*a+1], x[3*a+2], uf);
    const double m = mass[a];
    const double fxi = m * xi_over_dtLBM * (uf[0]*vs - v[3*a]);
    const double fyi = m * xi_over_dtLBM * (uf[1]*vs - v[3*a+1]);
    const double fzi = m * xi_over_dtLBM * (uf[2]*vs - v[3*a+2]);
    f_add[3*a] += fxi; f_add[3*a+1] += fyi; f_add[3*a+2] += fzi;
    spread(g, ip, inv_dx, x[3*a], x[3*a+1], x[3*a+2],
           -fxi * inv_N / fs, -fyi * inv_N / fs, -fzi * inv_N / fs, dv);
  }
  if (fold) exchange_forces(g);
  return nc;
}

/* Streaming::exchange_forces as an entry point for the fix layer. */
void ORC_FN(grid_fold_forces)(void* gp) { exchange_forces((orc_grid*)gp); }

/* the port also restates the IBM forcing methods at the fix level */
#define ORC_METHODS 1
#define MLP_NPARAM_FIX 9795
int ORC_FN(grid_ibm_substep_method)(void* gp, const couplb_ibm_params* ip, int n,
                                    const double* x, const double* v, const double* mass,
                                    const int* active, double* f_add, int refresh, int fold,
                                    int method, int passes, double slip_tol,
                                    const double* mlp_w, double s_in, double s_out,
                                    const double g_lb[3], double* stats, double* rows);
#include "oracle_fix.inc"

/* ---- IBM forcing methods and the correction network ------------------
 * No counterpart in the reference: the reference applies the single penalty
 * pass above.  These restate the project's own definitions (multi-direct
 * forcing after Wang, Fan & Luo, J. Comput. Phys. 227 (2008), written with the
 * reference's penalty law; and the 84-64-64-3 correction network), so that the
 * CUDA forms have a CPU checker.  Definitions:
 *   u_corr(x) = u0(x) + (G(x)/rho(x) + g_lb)/2  at fluid nodes, u0 and rho from
 *               the refresh, G the IBM force field so far, g_lb the body force;
 *   U_i       = the reference's interpolation of u_corr at marker i;
 *   dF_i      = m xi/dt (U_i vs - v_i), added to the atom and spread as
 *               -dF_i/(N fs) (Jacobi: all dF_i of a pass before any spread);
 *   slip_i    = |U_i vs - v_i| after the last pass.
 * Network: x = (u0 at the 27 Roma nodes round(l)-1..round(l)+1, node-major
 * dz,dy,dx, then v/vs), all lattice velocities; h1 = relu(W1 s_in x + b1),
 * h2 = relu(W2 h1 + b2), y = W3 h2 + b3; correction dF = m xi/dt vs y/s_out. */

#define MLP_IN 84
#define MLP_HID 64
#define MLP_OUT 3
#define MLP_ROW 88
#define MLP_NPARAM (MLP_HID * MLP_IN + MLP_HID + MLP_HID * MLP_HID + MLP_HID + MLP_OUT * MLP_HID + MLP_OUT)

void ORC_FN(mlp_forward)(const double* w, double s_in, double s_out, int n,
                         const double* rows, int stride, double* y) {
  const double *W1 = w, *b1 = W1 + MLP_HID * MLP_IN, *W2 = b1 + MLP_HID;
  const double *b2 = W2 + MLP_HID * MLP_HID, *W3 = b2 + MLP_HID, *b3 = W3 + MLP_OUT * MLP_HID;
  for (int s = 0; s < n; s++) {
    const double* x = rows + (size_t)s * stride;
    double h1[MLP_HID], h2[MLP_HID];
    for (int j = 0; j < MLP_HID; j++) {
      double a = b1[j];
      for (int k = 0; k < MLP_IN; k++) a += W1[j * MLP_IN + k] * (x[k] * s_in);
      h1[j] = a > 0.0 ? a : 0.0;
    }
    for (int j = 0; j < MLP_HID; j++) {
      double a = b2[j];
      for (int k = 0; k < MLP_HID; k++) a += W2[j * MLP_HID + k] * h1[k];
      h2[j] = a > 0.0 ? a : 0.0;
    }
    for (int c = 0; c < MLP_OUT; c++) {
      double a = b3[c];
      for (int k = 0; k < MLP_HID; k++) a += W3[c * MLP_HID + k] * h2[k];
      y[(size_t)s * MLP_OUT + c] = a / s_out;
    }
  }
}

/* Loss L = sum over rows and outputs of (y_norm - s_out t)^2 / (3 n) with
 * t = rows[84..86]; returns L and writes dL/dw (MLP_NPARAM) to grad. */
double ORC_FN(mlp_loss_grad)(const double* w, double s_in, double s_out, int n,
                             const double* rows, double* grad) {
  const double *W1 = w, *b1 = W1 + MLP_HID * MLP_IN, *W2 = b1 + MLP_HID;
  const double *b2 = W2 + MLP_HID * MLP_HID, *W3 = b2 + MLP_HID, *b3 = W3 + MLP_OUT * MLP_HID;
  double *gW1 = grad, *gb1 = gW1 + MLP_HID * MLP_IN, *gW2 = gb1 + MLP_HID;
  double *gb2 = gW2 + MLP_HID * MLP_HID, *gW3 = gb2 + MLP_HID, *gb3 = gW3 + MLP_OUT * MLP_HID;
  memset(grad, 0, sizeof(double) * MLP_NPARAM);
  double loss = 0.0;
  const double inv = 1.0 / (3.0 * (double)n);
  for (int s = 0; s < n; s++) {
    const double* r = rows + (size_t)s * MLP_ROW;
    double x[MLP_IN], h1[MLP_HID], h2[MLP_HID], d2[MLP_HID], d1[MLP_HID], dy[MLP_OUT];
    for (int k = 0; k < MLP_IN; k++) x[k] = r[k] * s_in;
    for (int j = 0; j < MLP_HID; j++) {
      double a = b1[j];
      for (int k = 0; k < MLP_IN; k++) a += W1[j * MLP_IN + k] * x[k];
      h1[j] = a > 0.0 ? a : 0.0;
    }
    for (int j = 0; j < MLP_HID; j++) {
      double a = b2[j];
      for (int k = 0; k < MLP_HID; k++) a += W2[j * MLP_HID + k] * h1[k];
      h2[j] = a > 0.0 ? a : 0.0;
    }
    for (int c = 0; c < MLP_OUT; c++) {
      double a = b3[c];
      for (int k = 0; k < MLP_HID; k++) a += W3[c * MLP_HID + k] * h2[k];
      const double e = a - s_out * r[MLP_IN + c];
      loss += e * e * inv;
      dy[c] = 2.0 * e * inv;
    }
    for (int c = 0; c < MLP_OUT; c++) {
      gb3[c] += dy[c];
      for (int k = 0; k < MLP_HID; k++) gW3[c * MLP_HID + k] += dy[c] * h2[k];
    }
    for (int k = 0; k < MLP_HID; k++) {
      double a = 0.0;
      for (int c = 0; c < MLP_OUT; c++) a += W3[c * MLP_HID + k] * dy[c];
      d2[k] = h2[k] > 0.0 ? a : 0.0;
    }
    for (int j = 0; j < MLP_HID; j++) {
      gb2[j] += d2[j];
      for (int k = 0; k < MLP_HID; k++) gW2[j * MLP_HID + k] += d2[j] * h1[k];
    }
    for (int k = 0; k < MLP_HID; k++) {
      double a = 0.0;
      for (int j = 0; j < MLP_HID; j++) a += W2[j * MLP_HID + k] * d2[j];
      d1[k] = h1[k] > 0.0 ? a : 0.0;
    }
    for (int j = 0; j < MLP_HID; j++) {
      gb1[j] += d1[j];
      for (int k = 0; k < MLP_IN; k++) gW1[j * MLP_IN + k] += d1[j] * x[k];
    }
  }
  return loss;
}

/* Sum of the force field over all ghost-inclusive aliases of a fluid node
 * (spreads that landed on periodic ghosts are not folded until the last
 * sub-step). */
static void force_over_aliases(const orc_grid* g, int i, int j, int k, double out[3]) {
  const int nn[3] = {g->nx, g->ny, g->nz};
  const int c[3] = {i, j, k};
  int al[3][3], na[3];
  const int nd = (g->D == 3) ? 3 : 2;
  for (int d = 0; d < 3; d++) {
    if (d >= nd) { al[d][0] = c[d]; na[d] = 1; continue; }
    int ii = c[d];
    if (ii < 1) ii += nn[d];
    else if (ii > nn[d]) ii -= nn[d];
    na[d] = 0;
    al[d][na[d]++] = ii;
    if (ii == nn[d] && !g->wall_face[d][0]) al[d][na[d]++] = 0;
    if (ii == 1 && !g->wall_face[d][1]) al[d][na[d]++] = nn[d] + 1;
  }
  out[0] = out[1] = out[2] = 0.0;
  for (int a = 0; a < na[2]; a++)
    for (int b = 0; b < na[1]; b++)
      for (int e = 0; e < na[0]; e++) {
        const int n = gidx(g, al[0][e], al[1][b], al[2][a]);
        out[0] += g->fx[n]; out[1] += g->fy[n]; out[2] += g->fz[n];
      }
}

/* The reference's interpolation (couplb_ibm.h:57-90) of u_corr. */
static void interpolate_corr(const orc_grid* g, const couplb_ibm_params* ip, double inv_dx,
                             const double* xp, const double g_lb[3], double out[3]) {
  double lx, ly, lz;
  phys_to_local(g, ip, inv_dx, xp[0], xp[1], xp[2], &lx, &ly, &lz);
  const int i0 = (int)floor(lx), j0 = (int)floor(ly);
  const int k0 = (g->D == 3) ? (int)floor(lz) : 0;
  double ui = 0, vi = 0, wi = 0, ws = 0;
  for (int k = (g->D == 3 ? k0 - 1 : 0); k <= (g->D == 3 ? k0 + 2 : 0); k++) {
    if (g->D == 3 && (k < 0 || k >= g->gz)) continue;
    for (int j = j0 - 1; j <= j0 + 2; j++) {
      if (j < 0 || j >= g->gy) continue;
      for (int i = i0 - 1; i <= i0 + 2; i++) {
        if (i < 0 || i >= g->gx) continue;
        const int n = gidx(g, i, j, k);
        const int nt = g->type[n];
        const double d = delta_product(g, ip->delta, lx - i, ly - j, lz - k);
        if (nt == 0) {
          double G[3];
          force_over_aliases(g, i, j, k, G);
          const double ir = 1.0 / g->rho[n];
          const double c0 = g->ux[n] + 0.5 * (G[0] * ir + g_lb[0]);
          const double c1 = g->uy[n] + 0.5 * (G[1] * ir + g_lb[1]);
          const double c2 = g->uz[n] + 0.5 * (G[2] * ir + (g->D == 3 ? g_lb[2] : 0.0));
          ui += c0 * d; vi += c1 * d; wi += c2 * d; ws += d;
        } else if (nt == 1 || nt == 3) {
          ws += d;
        } else if (nt == 2) {
          ui += g->bc_ux[n] * d; vi += g->bc_uy[n] * d; wi += g->bc_uz[n] * d; ws += d;
        }
      }
    }
  }
  if (ws > DELTA_TOL) {
    const double iw = 1.0 / ws;
    out[0] = ui * iw; out[1] = vi * iw; out[2] = wi * iw;
  } else {
    out[0] = out[1] = out[2] = 0.0;
  }
}

/* Network input of one marker: u0 at the 27 Roma nodes and v / vs. */
static void mlp_input(const orc_grid* g, const couplb_ibm_params* ip, double inv_dx,
                      const double* xp, const double* vp, double* x) {
  double l[3];
  phys_to_local(g, ip, inv_dx, xp[0], xp[1], xp[2], &l[0], &l[1], &l[2]);
  int s[3];
  for (int d = 0; d < 3; d++) {
    const int f = (int)floor(l[d]);
    s[d] = f - 1 + ((l[d] - f) >= 0.5 ? 1 : 0);
  }
  for (int p = 0; p < 27; p++) {
    const int i = s[0] + p % 3, j = s[1] + (p / 3) % 3, k = s[2] + p / 9;
    double u[3] = {0.0, 0.0, 0.0};
    if (i >= 0 && i < g->gx && j >= 0 && j < g->gy && k >= 0 && k < g->gz) {
      const int n = gidx(g, i, j, k);
      if (g->type[n] == 0) { u[0] = g->ux[n]; u[1] = g->uy[n]; u[2] = g->uz[n]; }
      else if (g->type[n] == 2) { u[0] = g->bc_ux[n]; u[1] = g->bc_uy[n]; u[2] = g->bc_uz[n]; }
    }
    x[3 * p] = u[0]; x[3 * p + 1] = u[1]; x[3 * p + 2] = u[2];
  }
  for (int c = 0; c < 3; c++) x[81 + c] = vp[c] / ip->vel_scale;
}

static void slip_stats(const orc_grid* g, const couplb_ibm_params* ip, double inv_dx, int n,
                       const double* x, const double* v, const int* active,
                       const double g_lb[3], int nc, double* rms, double* mx) {
  double s2 = 0.0, m = 0.0;
  for (int a = 0; a < n; a++) {
    if (active && !active[a]) continue;
    double U[3];
    interpolate_corr(g, ip, inv_dx, x + 3*a, g_lb, U);
    double e2 = 0.0;
    for (int c = 0; c < 3; c++) { const double e = U[c] * ip->vel_scale - v[3*a+c]; e2 += e * e; }
    s2 += e2;
    if (sqrt(e2) > m) m = sqrt(e2);
  }
  *rms = nc ? sqrt(s2 / nc) : 0.0;
  *mx = m;
}

/* One sub-step with a forcing method.  method 1: iterative with `passes`
 * passes (1 = the reference pass plus a slip measurement); method 2: the
 * reference pass plus the network correction (mlp_w, bf16-valued weights),
 * then the slip check; above slip_tol the passes-1 iterative corrections run.
 * stats: [rms slip of the method-2 check, its max, rms slip at the end, its
 * max, 1 if the fallback ran, coupled markers].  rows (n x 88, may be NULL):
 * network input, total correction beyond the reference pass / (m xi vs / dt)
 * in lattice velocity units, 0. */
int ORC_FN(grid_ibm_substep_method)(void* gp, const couplb_ibm_params* ip, int n,
                                    const double* x, const double* v, const double* mass,
                                    const int* active, double* f_add, int refresh, int fold,
                                    int method, int passes, double slip_tol,
                                    const double* mlp_w, double s_in, double s_out,
                                    const double g_lb[3], double* stats, double* rows) {
  orc_grid* g = (orc_grid*)gp;
  if (refresh) {
    ORC_FN(grid_macroscopic)(g, 0);
    ORC_FN(grid_exchange_velocity)(g);
  }
  const double inv_dx = 1.0 / ip->dx;
  const double xo = ip->xi_ibm / ip->dt_lbm;
  const double inv_N = 1.0 / (double)ip->md_per_lb;
  const double dv = (g->D == 3) ? (ip->dx * ip->dx * ip->dx) : (ip->dx * ip->dx);
  const double vs = ip->vel_scale, fs = ip->force_scale;
  double* dF = (double*)calloc((size_t)3 * (n > 0 ? n : 1), sizeof(double));
  double* corr = (double*)calloc((size_t)3 * (n > 0 ? n : 1), sizeof(double));
  int nc = 0;
  /* pass 0: the reference pass (+ the network correction) */
  for (int a = 0; a < n; a++) {
    if (active && !active[a]) continue;
    nc++;
    double uf[3];
    interpolate(g, ip, inv_dx, x[3*a], x[3*a+1], x[3*a+2], uf);
    const double m = mass[a];
    double F[3];
    for (int c = 0; c < 3; c++) F[c] = m * xo * (uf[c] * vs - v[3*a+c]);
    if (method == 2) {
      double in[MLP_IN], y[3];
      mlp_input(g, ip, inv_dx, x + 3*a, v + 3*a, in);
      ORC_FN(mlp_forward)(mlp_w, s_in, s_out, 1, in, MLP_IN, y);
      for (int c = 0; c < 3; c++) { corr[3*a+c] = m * xo * vs * y[c]; F[c] += corr[3*a+c]; }
    }
    for (int c = 0; c < 3; c++) f_add[3*a+c] += F[c];
    spread(g, ip, inv_dx, x[3*a], x[3*a+1], x[3*a+2],
           -F[0] * inv_N / fs, -F[1] * inv_N / fs, -F[2] * inv_N / fs, dv);
  }
  double rms0 = 0.0, max0 = 0.0, rms1 = 0.0, max1 = 0.0;
  int fallback = 0, run = 1;
  if (method == 2) {
    slip_stats(g, ip, inv_dx, n, x, v, active, g_lb, nc, &rms0, &max0);
    run = rms0 > slip_tol;
    fallback = run;
    if (!run) { rms1 = rms0; max1 = max0; }
  }
  if (run) {
    for (int it = 0; it < passes - 1; it++) {
      for (int a = 0; a < n; a++) {
        if (active && !active[a]) continue;
        double U[3];
        interpolate_corr(g, ip, inv_dx, x + 3*a, g_lb, U);
        for (int c = 0; c < 3; c++) dF[3*a+c] = mass[a] * xo * (U[c] * vs - v[3*a+c]);
      }
      for (int a = 0; a < n; a++) {
        if (active && !active[a]) continue;
        for (int c = 0; c < 3; c++) { f_add[3*a+c] += dF[3*a+c]; corr[3*a+c] += dF[3*a+c]; }
        spread(g, ip, inv_dx, x[3*a], x[3*a+1], x[3*a+2],
               -dF[3*a] * inv_N / fs, -dF[3*a+1] * inv_N / fs, -dF[3*a+2] * inv_N / fs, dv);
      }
    }
    slip_stats(g, ip, inv_dx, n, x, v, active, g_lb, nc, &rms1, &max1);
  }
  if (stats) {
    stats[0] = rms0; stats[1] = max0; stats[2] = rms1; stats[3] = max1;
    stats[4] = fallback; stats[5] = nc;
  }
  if (rows) {
    for (int a = 0; a < n; a++) {
      double* r = rows + (size_t)a * MLP_ROW;
      if (active && !active[a]) { memset(r, 0, sizeof(double) * MLP_ROW); continue; }
      mlp_input(g, ip, inv_dx, x + 3*a, v + 3*a, r);
      for (int c = 0; c < 3; c++) r[MLP_IN + c] = corr[3*a+c] / (mass[a] * xo * vs);
      r[MLP_ROW - 1] = 0.0;
    }
  }
  free(dF);
  free(corr);
  if (fold) exchange_forces(g);
  return nc;
}
