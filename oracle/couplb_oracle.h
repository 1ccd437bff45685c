/*
 * couplb_oracle.h -- CPU oracle API (TEST INFRASTRUCTURE ONLY).
 *
 * Two libraries implement this API with the same signatures:
 *   - libcouplb_oracle.so : couplb_oracle.c, a plain-C restatement of the
 *                           reference algorithm (function prefix orc_);
 *   - _ref/libcouplb_ref.so: ref_harness.cpp, the reference's own headers
 *                           (CoupLB/couplb_*.h, compiled unmodified) driven
 *                           by a restatement of FixCoupLB's sequencing
 *                           (function prefix ref_).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use them, as
 * the checker of the CUDA path; the product never links or calls them.
 *
 * Grid arrays use the reference layout: ghost-inclusive G = gx*gy*gz nodes,
 * n = i + gx*(j + gy*k), populations f[q*G + n] (couplb_lattice.h:82-129).
 */
#ifndef COUPLB_ORACLE_H
#define COUPLB_ORACLE_H

#include "../include/couplb_b200.h"

#ifndef ORC_FN
#define ORC_FN(x) orc_##x
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* grid layer (CoupLB::Grid/BGK/Streaming/Boundary/IBM) */
void*  ORC_FN(grid_create)(int dim, int nx, int ny, int nz, double tau,
                           double rho0, const int wall[6],
                           const double wall_vel[3]);
void   ORC_FN(grid_destroy)(void* g);
long   ORC_FN(grid_ntotal)(void* g);
void   ORC_FN(grid_init_equilibrium)(void* g, double rho, double ux, double uy,
                                     double uz);
void   ORC_FN(grid_set_f)(void* g, const double* f);
void   ORC_FN(grid_get_f)(void* g, double* f);
void   ORC_FN(grid_get_macro)(void* g, double* rho, double* ux, double* uy,
                              double* uz);
void   ORC_FN(grid_set_force)(void* g, const double* fx, const double* fy,
                              const double* fz);
void   ORC_FN(grid_get_force)(void* g, double* fx, double* fy, double* fz);
void   ORC_FN(grid_lbm_step)(void* g, const double* g_lb);
void   ORC_FN(grid_macroscopic)(void* g, int guo);
void   ORC_FN(grid_exchange_velocity)(void* g);
void   ORC_FN(grid_diagnostics)(void* g, double out[5], int* clamps);
void   ORC_FN(grid_fold_forces)(void* g);
int    ORC_FN(grid_ibm_substep)(void* g, const couplb_ibm_params* ip, int n,
                                const double* x, const double* v,
                                const double* mass, const int* active,
                                double* f_add, int refresh, int fold);

/* IBM forcing methods and the correction network (project definitions, no
 * reference counterpart; port library only) */
/* Periodic wrap of the single-pass IBM window (bit d: axis d); 0 = the
 * reference's clipping. */
void   ORC_FN(grid_set_ibm_wrap)(void* g, int mask);
int    ORC_FN(grid_ibm_substep_method)(void* g, const couplb_ibm_params* ip, int n,
                                       const double* x, const double* v,
                                       const double* mass, const int* active,
                                       double* f_add, int refresh, int fold,
                                       int method, int passes, double slip_tol,
                                       const double* mlp_w, double s_in, double s_out,
                                       const double g_lb[3], double* stats,
                                       double* rows);
void   ORC_FN(mlp_forward)(const double* w, double s_in, double s_out, int n,
                           const double* rows, int stride, double* y);
double ORC_FN(mlp_loss_grad)(const double* w, double s_in, double s_out, int n,
                             const double* rows, double* grad);

/* fix layer (FixCoupLB hooks) */
void*  ORC_FN(fix_create)(const couplb_fix_config* cfg, const couplb_domain* dom,
                          char* err, int errlen);
void   ORC_FN(fix_destroy)(void* fx);
int    ORC_FN(fix_setup)(void* fx, const couplb_atoms* at, long long step);
int    ORC_FN(fix_post_force)(void* fx, const couplb_atoms* at, long long step);
int    ORC_FN(fix_end_of_step)(void* fx, long long step);
void   ORC_FN(fix_set_gravity)(void* fx, const double g[3]);
void*  ORC_FN(fix_grid)(void* fx);
void   ORC_FN(fix_last_diag)(void* fx, double out[5], int* clamps);
void   ORC_FN(fix_scales)(void* fx, double out[6]);
const char* ORC_FN(fix_last_error)(void* fx);

#ifdef __cplusplus
}
#endif
#endif
