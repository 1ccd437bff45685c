/*
 * couplb_b200.h -- C ABI of the B200 (sm_100a) CoupLB hot path.
 *
 * Two layers, both plain C (no CUDA or torch types in any signature):
 *
 *   1. The lattice engine (couplb_*): one handle owns the device state of one
 *      LBM subdomain (populations, force field, moments) and runs the
 *      per-step kernels on one CUDA stream.  It replaces the member calls that
 *      FixCoupLB makes on CoupLB::Grid / BGK / Streaming / IBM.
 *
 *   2. The fix core (couplb_fix_*): the `fix couplb` keyword parser, unit
 *      conversion and the init / setup / post_force / end_of_step sequencing of
 *      FixCoupLB, written against plain atom arrays so that a LAMMPS FixCoupLB
 *      (or any MD code) forwards its hooks here.
 *
 * Every function returns an int status: COUPLB_OK (0) on success, a negative
 * COUPLB_ERR_* code on failure.  Nothing aborts the process; the message of the
 * last failure is available from couplb_last_error / couplb_fix_last_error.
 * A handle is used from one host thread at a time.
 *
 * Reference interfaces each entry point replaces are cited as
 * <file>:<line> relative to the CoupLB source tree.
 */
#ifndef COUPLB_B200_H
#define COUPLB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COUPLB_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------- */
#define COUPLB_OK               0
#define COUPLB_ERR_ARG         -1  /* invalid argument / size                */
#define COUPLB_ERR_CUDA        -2  /* a CUDA runtime call failed              */
#define COUPLB_ERR_STATE       -3  /* call out of order / handle not ready    */
#define COUPLB_ERR_NUMERIC     -4  /* non-finite density or Mach > 0.5        */
#define COUPLB_ERR_IO          -5  /* checkpoint / profile file error         */
#define COUPLB_ERR_PARSE       -6  /* `fix couplb` argument error             */
#define COUPLB_ERR_UNSUPPORTED -7  /* feature outside this build              */
#define COUPLB_ERR_TOO_LARGE   -8  /* input above a fixed capacity            */

/* ---- enumerations ---------------------------------------------------- */
/* storage / arithmetic precision of the populations */
#define COUPLB_FP64          0  /* plain f in FP64, FP64 arithmetic            */
#define COUPLB_FP32_SHIFTED  1  /* h = f - w*rho0 stored and computed in FP32  */
#define COUPLB_FP16_SHIFTED  2  /* h stored as scaled IEEE half, FP32 compute  */

/* IBM delta kernel (couplb_ibm.h:37) */
#define COUPLB_DELTA_ROMA    0
#define COUPLB_DELTA_PESKIN4 1

/* wall types (fix_couplb.cpp:56-58) */
#define COUPLB_WALL_PERIODIC 0
#define COUPLB_WALL_NOSLIP   1
#define COUPLB_WALL_MOVING   2
#define COUPLB_WALL_FREESLIP 3
#define COUPLB_WALL_OPEN     4

/* gravity component styles (fix_couplb.h:172) */
#define COUPLB_G_NONE     0
#define COUPLB_G_CONSTANT 1
#define COUPLB_G_EQUAL    2

/* ======================================================================
 * Layer 1: lattice engine
 * ==================================================================== */

/* Lattice of one subdomain, in lattice units (dx = dt = 1). */
typedef struct couplb_lattice_params {
  int    dim;          /* 2 -> D2Q9, 3 -> D3Q19                               */
  int    nx, ny, nz;   /* interior nodes; nz must be 1 when dim == 2          */
  double tau;          /* BGK relaxation time, > 0.5                          */
  double rho0;         /* lattice reference density (FixCoupLB uses 1.0)      */
  int    wall[6];      /* xlo xhi ylo yhi zlo zhi wall types, 0..4            */
  double wall_vel[3];  /* velocity of type-2 walls, lattice units             */
  int    body_force;   /* 1 if a gravity style is set: keeps the density field
                          that apply_external_force reads (fix_couplb.cpp:706) */
  int    precision;    /* COUPLB_FP64 / COUPLB_FP32_SHIFTED / COUPLB_FP16_SHIFTED */
  int    device;       /* CUDA device ordinal                                 */
} couplb_lattice_params;

/* IBM coupling constants (fix_couplb.cpp:286-317, 763-769). */
typedef struct couplb_ibm_params {
  int    delta;          /* COUPLB_DELTA_ROMA / COUPLB_DELTA_PESKIN4          */
  int    md_per_lb;      /* MD sub-steps per LB step, >= 1                    */
  double xi_ibm;         /* penalty relaxation factor, 0 < xi <= 1            */
  double dt_lbm;         /* LB time step, MD units                           */
  double dx;             /* lattice spacing, MD units                         */
  double vel_scale;      /* dx / dt_lbm                                       */
  double force_scale;    /* rho * dx^(D+1) / dt_lbm^2                         */
  double domain_lo[3];   /* box lower corner, MD units                        */
  int    offset[3];      /* global index of this subdomain's first node       */
} couplb_ibm_params;

/* Reductions of a20 (couplb_lattice.h:203-242, fix_couplb.cpp:818-844). */
typedef struct couplb_diag {
  double umax;       /* max |u| over fluid nodes, lattice units               */
  double mass;       /* sum rho over fluid nodes (FP64 on the device)         */
  double mom[3];     /* sum rho*u over fluid nodes (FP64 on the device)       */
  int    clamps;     /* density clamps of the last moment pass                */
  int    nonfinite;  /* non-finite densities seen by any kernel since reset   */
} couplb_diag;

typedef struct couplb_handle couplb_handle;

/* Create / destroy.  Replaces Grid::allocate + init_equilibrium(rho0,0,0,0)
 * (couplb_lattice.h:105-154), BGK::set_tau (couplb_collision.h:15),
 * Boundary::set_walls_x/y/z + set_wall_velocity (couplb_boundary.h:12-38) and
 * Streaming::precompute_wall_flags (couplb_streaming.h:74-80), as called from
 * FixCoupLB::setup_grid / setup_boundaries (fix_couplb.cpp:484-539). */
int  couplb_create(const couplb_lattice_params* p, couplb_handle** out);
int  couplb_destroy(couplb_handle* h);
const char* couplb_last_error(const couplb_handle* h);  /* h may be NULL */
int  couplb_version(void);
/* sizeof of the ABI structs, for bindings to check their layouts:
 * 0 lattice_params, 1 ibm_params, 2 diag, 3 fix_config, 4 domain, 5 atoms,
 * 6 ibm_method, 7 mlp_train_params.
 * No counterpart in the reference (binding support only). */
size_t couplb_struct_size(int which);

/* Run on a caller-owned stream (a cudaStream_t passed as void*). */
int  couplb_set_stream(couplb_handle* h, void* cuda_stream);
int  couplb_synchronize(couplb_handle* h);

/* Grid::init_equilibrium (couplb_lattice.h:145-154). */
int  couplb_init_equilibrium(couplb_handle* h, double rho, double ux,
                             double uy, double uz);

/* Populations in the reference layout: double f[q*G + n], G = gx*gy*gz
 * ghost-inclusive nodes, n = i + gx*(j + gy*k) (couplb_lattice.h:82-129).
 * set: like IO::read_checkpoint (couplb_io.h:802-817) -- f and f_buf take the
 * values, then the moments are recomputed without the Guo term.  Only interior
 * values are used.  get: interior values are the post-stream state; ghost
 * values are the periodic images (non-wall faces) or w_q*rho0 (wall faces). */
int  couplb_set_populations(couplb_handle* h, const double* f_host);
int  couplb_get_populations(couplb_handle* h, double* f_host);
size_t couplb_ghost_nodes(const couplb_handle* h);   /* G */

/* One LB step: FixCoupLB::do_lbm_step (fix_couplb.cpp:659-669) =
 * apply_external_force (:680-708) + compute_macroscopic(true) + collide +
 * exchange + stream + enforce_wall_ghost_fields + clear_forces, fused.
 * g_lb: body-force acceleration in lattice units, or NULL when no gravity
 * style is set (fix_couplb.cpp:686). */
int  couplb_lbm_step(couplb_handle* h, const double* g_lb);

/* Slab decomposition along z (the populations part of
 * Streaming::exchange_dim, couplb_streaming.h:176-194, for d = z): a lattice
 * that is one z slab of a larger one, with a neighbour subdomain across one
 * or both z faces.  couplb_halo_attach binds to face `side` (0: z low,
 * 1: z high; the face must be periodic, COUPLB_WALL_PERIODIC) a device
 * buffer of couplb_halo_bytes that holds, before every LB step, the
 * populations that cross that face from the neighbour: the buffer
 * couplb_halo_pack(neighbour, 1 - side, buf) wrote after the neighbour's last
 * LB step (5 planes of nx * ny values in the storage format).  The pull of a
 * source beyond an attached face reads that buffer instead of wrapping onto
 * this lattice's other face, so the slabs step exactly like the whole
 * lattice.  NULL detaches.  The caller moves the buffers between slabs (a
 * device copy, a peer copy or an NCCL send / receive) between LB steps.  The
 * first LB step after couplb_set_populations or couplb_init_equilibrium reads
 * the post-stream state in place and needs no halo; pack needs the
 * post-collision state of an LB step.  Ghost values of attached faces in
 * couplb_get_populations are not the neighbour's.  IBM sub-steps on a lattice
 * with an attached face need the IBM halos below on that face. */
int  couplb_halo_attach(couplb_handle* h, int side, const void* d_recv);
size_t couplb_halo_bytes(const couplb_handle* h);
int  couplb_halo_pack(couplb_handle* h, int side, void* d_send);

/* IBM across z slabs (the velocity exchange and the reverse force exchange
 * of Streaming::exchange_velocity / exchange_forces, couplb_streaming.h:
 * 196-245, for d = z).  A marker window [k0-1, k0+2] reaches one plane below
 * a slab's low face and two above its high face; the reference's ghost layer
 * is one plane wide, so its multi-rank windows lose the second plane above
 * each internal face.  Here the halo holds what the whole lattice would use:
 * planes = 1 below; above, 2 at an internal face, and 1 at the face that
 * wraps the global periodic box in the clipped window mode (ibm_window 0,
 * where the whole lattice clips the plane beyond its ghost layer), so slab
 * sub-steps give the forces of the undecomposed lattice.
 * couplb_ibm_halo_attach binds to z face `side` (which carries a population
 * halo) d_vel, the neighbour's {ux, uy, uz, rho} of those planes, and
 * d_force, where sub-steps add the forces spread onto them; both hold
 * couplb_ibm_halo_bytes(h, planes) in the auxiliary type (4 values per node,
 * plane-major).  d_vel NULL detaches.  Per LB cycle, after the LB step and the
 * population exchange: couplb_ibm_halo_moments(neighbour, 1 - side, planes,
 * buf) writes what this lattice's d_vel of `side` must hold (side 0 of the
 * neighbour above: its planes 0..planes-1; side 1 of the neighbour below: its
 * top plane); after the last sub-step of the cycle, before the next LB step,
 * the caller hands each d_force to the neighbour across that face, which adds
 * it with couplb_ibm_halo_fold(neighbour, 1 - side, planes, buf), and zeroes
 * d_force.  Single-pass sub-steps only (the ITERATIVE and LEARNED methods
 * return COUPLB_ERR_UNSUPPORTED on a slab). */
size_t couplb_ibm_halo_bytes(const couplb_handle* h, int planes);
int  couplb_ibm_halo_attach(couplb_handle* h, int side, int planes, const void* d_vel, void* d_force);
int  couplb_ibm_halo_moments(couplb_handle* h, int side, int planes, void* d_out);
int  couplb_ibm_halo_fold(couplb_handle* h, int side, int planes, const void* d_in);

/* Grid::compute_macroscopic(false) (couplb_lattice.h:155-202) followed by
 * Streaming::exchange_velocity (couplb_streaming.h:140-143). */
int  couplb_macroscopic(couplb_handle* h);

/* Ghost-inclusive (G-node) copies of rho, u after the last couplb_macroscopic;
 * wall ghost nodes carry the values of enforce_wall_ghost_fields
 * (fix_couplb.cpp:800-809).  Any pointer may be NULL. */
int  couplb_get_macroscopic(couplb_handle* h, double* rho, double* ux,
                            double* uy, double* uz);

/* The Eulerian force field (Grid::fx/fy/fz), G-node layout; ghost values 0.
 * set is for tests and restarts: the values act as already folded forces. */
int  couplb_get_force_field(couplb_handle* h, double* fx, double* fy, double* fz);
int  couplb_set_force_field(couplb_handle* h, const double* fx,
                            const double* fy, const double* fz);

/* Grid::max_velocity + compute_diagnostics + rho_clamp_count over the moments
 * of the last couplb_macroscopic (couplb_lattice.h:203-242). */
int  couplb_diagnostics(couplb_handle* h, couplb_diag* out);

/* couplb_diagnostics_noalloc -- the reductions of couplb_diagnostics (max |u|,
 * total mass, total momentum) for callers that cannot let a library allocate
 * device memory: an MD code that owns all device memory through its own pool
 * (a foreign cudaMalloc fragments the pool, and cudaFree synchronises the
 * whole device) or a time loop that must not stall on such a synchronisation.
 * No counterpart in the reference; nothing here calls cudaMalloc or cudaFree.
 *   d_rho, d_ux, d_uy, d_uz: caller-owned device arrays of n moments --
 *       double for COUPLB_FP64 (rho absolute), float for the shifted formats
 *       (rho stored as its deviation from rho0, like the lattice's moments);
 *   d_out: caller-owned device array of 5 doubles receiving
 *       {max |u|, sum rho, sum rho*ux, sum rho*uy, sum rho*uz};
 *   stream: cudaStream_t (as void*) the two kernels are queued on; no sync.
 * Scratch lives in a fixed array of COUPLB_NOALLOC_MAX_PARTIALS * 5 doubles
 * (1.25 MiB) in device global memory that every GPU loading this library keeps
 * until exit; n above COUPLB_NOALLOC_MAX_NODES returns COUPLB_ERR_TOO_LARGE.
 * The first call on a device looks up that array's device address (with the
 * device current), so make that first call before any stream capture.  All
 * calls share the array and it keeps the last call's contents; nothing in it
 * needs to start at zero, but calls whose kernels overlap on the GPU race on
 * it and must be serialised by the caller.  max |u| is NaN when any node's
 * velocity is NaN (couplb_diagnostics follows the reference, whose maximum
 * skips NaN, and reports non-finite densities in its own count). */
#define COUPLB_NOALLOC_CHUNK        2048        /* nodes reduced per block      */
#define COUPLB_NOALLOC_MAX_PARTIALS 32768       /* scratch slots                */
#define COUPLB_NOALLOC_MAX_NODES    (COUPLB_NOALLOC_CHUNK * (long long)COUPLB_NOALLOC_MAX_PARTIALS)
int  couplb_diagnostics_noalloc(const void* d_rho, const void* d_ux,
                                const void* d_uy, const void* d_uz, long long n,
                                int precision, double rho0, double* d_out,
                                void* stream);

/* Per-j sums over i and k of ux, uy and rho after the last couplb_macroscopic
 * (each output holds ny doubles): the local sums of FixCoupLB::write_profile
 * (fix_couplb.cpp:906-910). */
int  couplb_y_profile(couplb_handle* h, double* ux_sum, double* uy_sum,
                      double* rho_sum);

/* IBM: constants, then one MD sub-step of FixCoupLB::do_ibm_sub_coupling
 * (fix_couplb.cpp:730-798): interpolate (couplb_ibm.h:57-90), penalty force
 * (fix_couplb.cpp:777-785), spread (couplb_ibm.h:92-133) and the reverse
 * force fold (couplb_streaming.h:155-158).
 *   host arrays:   x, v: n*3 doubles (MD units), mass: n doubles,
 *                  active: n ints (nonzero = atom is in the fix group) or NULL,
 *                  f_add: n*3 doubles; the IBM force is ADDED to it.
 *   refresh:       nonzero on the first sub-step of an LB cycle (or when atoms
 *                  reappear): recompute the fluid velocity (fix_couplb.cpp:757).
 * Returns the number of coupled atoms through *ncoupled (may be NULL). */
int  couplb_set_ibm_params(couplb_handle* h, const couplb_ibm_params* ip);
int  couplb_ibm_substep(couplb_handle* h, int n, const double* x,
                        const double* v, const double* mass, const int* active,
                        double* f_add, int refresh, int* ncoupled);
/* Same with device-resident atom arrays (device pointers, same shapes). */
int  couplb_ibm_substep_device(couplb_handle* h, int n, const double* d_x,
                               const double* d_v, const double* d_mass,
                               const int* d_active, double* d_f_add,
                               int refresh);

/* One LB step and the first IBM sub-step of its cycle in one call: the
 * sequence FixCoupLB::post_force runs on the first MD sub-step of an LB cycle
 * (fix_couplb.cpp:640-651: do_lbm_step, :659-669, then do_ibm_sub_coupling
 * with the refresh, :730-798), i.e. couplb_lbm_step(h, g_lb) followed by
 * couplb_ibm_substep(h, n, ..., refresh = 1, ncoupled), with the same
 * results.  The host->device copies of the atom arrays run on a copy stream
 * while the LB kernel runs. */
int  couplb_lbm_step_ibm(couplb_handle* h, const double* g_lb, int n, const double* x,
                         const double* v, const double* mass, const int* active,
                         double* f_add, int* ncoupled);
/* Same with device-resident atom arrays: couplb_lbm_step followed by
 * couplb_ibm_substep_device(..., refresh = 1). */
int  couplb_lbm_step_ibm_device(couplb_handle* h, const double* g_lb, int n,
                                const double* d_x, const double* d_v,
                                const double* d_mass, const int* d_active,
                                double* d_f_add);

/* FP64 sum over all spread markers of the force given to the grid (lattice
 * units), accumulated on the device since the last reset: the fluid side of the
 * momentum balance of docs/theory.md (sub-stepped coupling).  No counterpart
 * function in the reference, which conserves this sum implicitly. */
int  couplb_ibm_total_force(couplb_handle* h, double out[3], int reset);

/* ---- IBM forcing methods and the no-slip correction network ----------
 * No counterpart in the reference, which applies one penalty pass per
 * sub-step (fix_couplb.cpp:777-792); these entry points are additions.
 *
 * u_corr(x) = u0(x) + (G(x)/rho(x) + g_lb)/2 is the fluid velocity the next
 * collision sees (u0, rho of the refresh, G the IBM force so far, g_lb the body
 * force of the last LB step).  A correction pass interpolates u_corr at every
 * marker, adds dF = m xi/dt (U vs - v) to the atom and spreads -dF/(N fs) with
 * the reference's weights; the slip of a marker is |U vs - v| (MD velocity
 * units).  Exact for md_per_lb = 1; with sub-steps G holds those so far. */
#define COUPLB_IBM_SINGLE    0  /* the reference's single pass (default)          */
#define COUPLB_IBM_ITERATIVE 1  /* passes-1 correction passes, then the slip      */
#define COUPLB_IBM_LEARNED   2  /* single pass + network correction (D3Q19);
                                   slip check, and the passes-1 corrections run
                                   when the RMS slip exceeds slip_tol; with
                                   slip_tol >= 1e300 (or +inf) there is no
                                   fallback and so no check                     */

typedef struct couplb_mlp couplb_mlp;   /* 84-64-64-3 network, BF16 weights */

typedef struct couplb_ibm_method {
  int    method;          /* COUPLB_IBM_*                                     */
  int    passes;          /* total passes of the iterative method, >= 1       */
  double slip_tol;        /* LEARNED: RMS slip above which the fallback runs  */
  const couplb_mlp* model;/* LEARNED: the network (same device)               */
} couplb_ibm_method;

int  couplb_set_ibm_method(couplb_handle* h, const couplb_ibm_method* m);
/* Slip of the last sub-step that measured it (synchronises):
 * out[0] RMS slip after the last pass, out[1] its max, out[2] RMS slip of the
 * learned check (0 if none), out[3] its max, out[4] markers, out[5] 1 if the
 * last sub-step fell back, out[6] slip checks and out[7] fallbacks since
 * the last reset (reset != 0 clears both counters). */
int  couplb_ibm_slip(couplb_handle* h, double out[8], int reset);
/* Training-sample capture: every later ITERATIVE or LEARNED sub-step appends
 * one row of COUPLB_MLP_ROW floats per marker to d_rows (device memory of
 * capacity rows) -- the network input (u0 at the 27 nodes round(l)-1..
 * round(l)+1, node-major z,y,x; then v / vel_scale), the correction beyond the
 * penalty pass over (m xi vel_scale / dt), lattice velocity units, and a 0.
 * Needs all atoms coupled (no group mask).  d_rows NULL stops the capture.
 * A sub-step that would overflow the capacity records nothing. */
#define COUPLB_MLP_IN  84
#define COUPLB_MLP_HID 64
#define COUPLB_MLP_OUT 3
#define COUPLB_MLP_ROW 88
#define COUPLB_MLP_NPARAM 9795   /* W1[64][84] b1 W2[64][64] b2 W3[3][64] b3 */
int  couplb_ibm_record(couplb_handle* h, float* d_rows, long long capacity);
int  couplb_ibm_record_count(couplb_handle* h, long long* rows);

/* Network y = (W3 relu(W2 relu(W1 s_in x + b1) + b2) + b3) / s_out, FP32
 * arithmetic with weights rounded to BF16.  Parameters flat as in
 * COUPLB_MLP_NPARAM (FP32 master copy).  Training minimises the mean of
 * (y s_out - t s_out)^2 over the three outputs with Adam. */
typedef struct couplb_mlp_train_params {
  int    epochs;          /* passes over the training rows                    */
  int    batch;           /* rows per Adam step (multiple of 64)              */
  double lr, lr_final;    /* cosine schedule from lr to lr_final              */
  double beta1, beta2, eps;
  unsigned long long seed;/* minibatch sampling                               */
  long long n_val;        /* the last n_val rows are held out for validation  */
} couplb_mlp_train_params;

int  couplb_mlp_create(int device, unsigned long long seed, couplb_mlp** out);
int  couplb_mlp_destroy(couplb_mlp* m);
const char* couplb_mlp_last_error(const couplb_mlp* m);
int  couplb_mlp_set_stream(couplb_mlp* m, void* cuda_stream);
int  couplb_mlp_set_weights(couplb_mlp* m, const float* w, double s_in, double s_out);
int  couplb_mlp_get_weights(couplb_mlp* m, float* w, double* s_in, double* s_out);
/* s_in = 1 / RMS of the inputs, s_out = 1 / RMS of the targets of n rows. */
int  couplb_mlp_fit_scales(couplb_mlp* m, const float* d_rows, long long n);
/* Outputs (n x 3 floats, device) of n rows (device, COUPLB_MLP_ROW floats). */
int  couplb_mlp_forward(couplb_mlp* m, const float* d_rows, long long n, float* d_out);
/* Loss and its gradient (host, COUPLB_MLP_NPARAM floats) over n rows. */
int  couplb_mlp_loss_grad(couplb_mlp* m, const float* d_rows, long long n, double* loss,
                          float* grad);
int  couplb_mlp_train(couplb_mlp* m, const float* d_rows, long long n,
                      const couplb_mlp_train_params* tp, double* train_loss,
                      double* val_loss);
/* File: "CLBMLP01", s_in, s_out (double), COUPLB_MLP_NPARAM floats. */
int  couplb_mlp_save(couplb_mlp* m, const char* path);
int  couplb_mlp_load(couplb_mlp* m, const char* path);

/* Device status word: counts of density clamps / non-finite densities seen by
 * the stepping kernels since the last reset.  Reading synchronises. */
int  couplb_read_status(couplb_handle* h, int* clamps, int* nonfinite, int reset);
/* Pipelined form of the same read (no counterpart in the reference): post
 * enqueues a copy of the status word on the handle's stream; last returns the
 * counts of the post before the latest one, waiting only for that copy, so a
 * per-step failure check keeps the next step queued on the device.  With a
 * single post, last waits for it.  Both return zeros before any post. */
int  couplb_status_post(couplb_handle* h);
int  couplb_status_last(couplb_handle* h, int* clamps, int* nonfinite);

/* Runtime options of a handle (no counterpart in the reference):
 *   "kernel"      variant of the fused LB kernel: -1 auto (default: packed for
 *                 the shifted formats, plain for FP64), 0 plain (one node per
 *                 thread), 2 packed (two nodes per thread in paired FP32
 *                 arithmetic; shifted formats, even nx).  A variant that does
 *                 not apply falls back to plain.
 *   "last_kernel" read-only: the variant the last LB step ran.
 *   "ibm_resident" 1 (default): ITERATIVE / LEARNED sub-steps of a 3D lattice
 *                 whose markers each fit a warp of one cooperative launch keep
 *                 each marker's stencil in registers across passes; 0 always
 *                 uses the general form (same results).
 *   "ibm_window"  0 (default): the IBM window of the reference, [i0-1, i0+2]
 *                 per axis clipped to the ghost-inclusive box
 *                 (couplb_ibm.h:64-73, 110-115), so a marker within a cell of a
 *                 high periodic face loses the plane beyond the ghost layer;
 *                 1: an axis whose two faces are periodic is wrapped instead
 *                 (every window node is used, through its interior image) --
 *                 for physics runs; results then differ from the reference's
 *                 near those faces.
 *   "ibm_group"   lanes per marker of the SINGLE-pass sub-step of a 3D lattice:
 *                 8 (default; four markers per warp, for markers whose window
 *                 lies inside the interior and whose stencil is cached, the
 *                 rest one warp each) or 32 (one warp per marker).  The two
 *                 differ only in the order of the interpolation sums.
 *   "ibm_sort"    refreshes between re-sorts of the order in which the
 *                 single-pass refresh visits the markers: by bands of 8 z
 *                 planes of their cell (y rows in 2D), so that markers whose
 *                 windows share population lines meet them in L2; when most
 *                 markers lie within 2 cells of their successor (chain or
 *                 spatially sorted arrays) the index order is kept.  A
 *                 sort waits for the lattice's stream once to read that
 *                 choice back.  Default 16; 0 always visits them in index
 *                 order.  Results do not depend on it.
 *   "ibm_block"   threads per block of the grouped (ibm_group 8) sub-step: 64,
 *                 128 (default) or 256; a launch shape, results unchanged up
 *                 to the order of the FP64 total-force sums.
 *   "ibm_slip"    1 (default): ITERATIVE / LEARNED sub-steps measure the slip
 *                 after their last pass (couplb_ibm_slip); 0: they do not, which
 *                 saves an interpolation pass and, for a learned sub-step
 *                 without fallback, the only grid-wide barrier of the launch.
 *   "barrier_spin" poll limit of each grid-wide barrier of the ITERATIVE /
 *                 LEARNED sub-step kernels (default 2^21 polls of ~100 ns).
 *                 A block whose barrier runs out counts a timeout and returns;
 *                 the sub-step's results are then invalid, the next launch
 *                 starts clean.  0 gives up at the first failed poll (tests).
 *   "timeouts"    read-only: bounded device waits that gave up (synchronises). */
int  couplb_set_option(couplb_handle* h, const char* name, long long value);
int  couplb_get_option(couplb_handle* h, const char* name, long long* value);

/* Bytes of device memory held by the handle. */
size_t couplb_device_bytes(const couplb_handle* h);

/* ======================================================================
 * Layer 2: fix core (`fix ID group couplb Nx Ny Nz nu rho [keywords]`)
 * ==================================================================== */

#define COUPLB_PATH_MAX 256

#define COUPLB_VTK_MAX_ATTR 32

/* Parsed arguments of `fix couplb` (fix_couplb.cpp:71-238). */
typedef struct couplb_fix_config {
  int    Nx, Ny, Nz;
  double nu, rho;
  int    md_per_lb;
  double xi_ibm;
  int    gstyle[3];                 /* COUPLB_G_*                          */
  double gconst[3];                 /* constant components, MD units       */
  char   gvar[3][64];               /* variable names of v_ components     */
  int    wall[6];
  double wall_vel[3];
  int    output_every;
  char   output_file[COUPLB_PATH_MAX];
  int    check_every;
  int    delta;                     /* COUPLB_DELTA_*                      */
  int    vtk_every;
  char   vtk_prefix[COUPLB_PATH_MAX];
  int    has_vtk_region;
  int    vtk_region_n;              /* 4 or 6 values given                 */
  double vtk_rlo[3], vtk_rhi[3];
  int    vtk_solid_nattr;           /* 0 = off                             */
  int    checkpoint_every;
  char   checkpoint_prefix[COUPLB_PATH_MAX];
  int    do_restart;
  char   restart_prefix[COUPLB_PATH_MAX];
  int    precision;                 /* `precision fp64|fp32|fp16`, default fp64 */
  int    dimension;                 /* domain->dimension                   */
  /* IBM forcing method (keywords of this implementation, no reference
   * counterpart): `ibm_method single|iterative|learned`, `ibm_passes N`
   * (default 5), `slip_tol V` (MD velocity units; learned method: RMS slip
   * above which the iterative passes run; 0 = never), `mlp_model FILE`
   * (network file of couplb_mlp_save; required by `learned`). */
  int    ibm_method;                /* COUPLB_IBM_*                        */
  int    ibm_passes;
  double slip_tol;
  char   mlp_model[COUPLB_PATH_MAX];
  char   vtk_solid_attr[COUPLB_VTK_MAX_ATTR][16];  /* vtk_solid attribute names */
  /* `ibm_window clip|wrap` (no reference counterpart): clip (default) is the
   * reference's IBM window, clipped to the ghost-inclusive box; wrap wraps it
   * across periodic axes (handle option "ibm_window"). */
  int    ibm_window;
} couplb_fix_config;

/* The MD side of one subdomain (LAMMPS: domain, update). */
typedef struct couplb_domain {
  int       dimension;
  double    boxlo[3], boxhi[3];
  double    sublo[3], subhi[3];   /* = box for one rank                     */
  int       periodicity[3];
  double    dt;                   /* MD time step                           */
  long long ntimestep;
} couplb_domain;

/* Atom arrays of one subdomain (LAMMPS: atom->x[0], v[0], f[0], ...). */
typedef struct couplb_atoms {
  int           nlocal;
  const double* x;           /* nlocal*3                                     */
  const double* v;           /* nlocal*3                                     */
  double*       f;           /* nlocal*3, IBM force added                    */
  const int*    mask;        /* nlocal, or NULL = every atom in the group    */
  int           groupbit;
  const double* rmass;       /* nlocal per-atom masses, or NULL              */
  const double* mass;        /* per-type masses indexed by type, if !rmass   */
  const int*    type;        /* nlocal, used with mass                       */
  /* optional arrays, read only by the vtk_solid output (NULL when absent) */
  const long long* tag;      /* nlocal atom IDs                              */
  const long long* molecule; /* nlocal molecule IDs                          */
  const double* radius;      /* nlocal                                       */
  const double* mu;          /* nlocal*4 dipole x, y, z, |mu|                */
  const double* omega;       /* nlocal*3                                     */
  const double* torque;      /* nlocal*3                                     */
} couplb_atoms;

typedef struct couplb_fix couplb_fix;

/* Gravity callback for v_ components: fills *value (MD units) for component
 * comp (0..2); called once per LB step, like update_gravity_variables
 * (fix_couplb.cpp:671-678).  Return 0 on success. */
typedef int  (*couplb_gravity_fn)(void* ctx, int comp, double* value);
/* Screen/log sink for rank-0 messages (fix_couplb.cpp:452-481). */
typedef void (*couplb_log_fn)(void* ctx, const char* line);

/* FixCoupLB::FixCoupLB argument parsing (fix_couplb.cpp:71-238); arg[0..2] are
 * ID, group, "couplb" as in LAMMPS.  On failure err holds the reference's
 * message. */
int  couplb_fix_parse(int narg, const char* const* arg, int dimension,
                      couplb_fix_config* cfg, char* err, int errlen);
int  couplb_fix_create(const couplb_fix_config* cfg, couplb_fix** out);
int  couplb_fix_destroy(couplb_fix* fx);
const char* couplb_fix_last_error(const couplb_fix* fx);
int  couplb_fix_set_gravity_callback(couplb_fix* fx, couplb_gravity_fn fn, void* ctx);
int  couplb_fix_set_log_callback(couplb_fix* fx, couplb_log_fn fn, void* ctx);
/* Values for v_ gravity components when no callback is set (MD units). */
int  couplb_fix_set_gravity_values(couplb_fix* fx, const double g[3]);
int  couplb_fix_set_device(couplb_fix* fx, int device);

/* Several ranks, the MD domain split along z only (every sub-box spans the
 * box in x and y, and its z range is whole lattice planes, at least 2): the
 * fix runs this rank's slab of the lattice and moves the slab halos through
 * the host code's communicator (the exchanges of Streaming::exchange_dim /
 * exchange_velocity / exchange_forces for d = z, couplb_streaming.h:176-245,
 * with the windows of the undecomposed lattice, see couplb_ibm_halo_attach).
 *   sendrecv: send send_bytes of device memory d_send to the rank across z
 *     face `side` of this sub-box (0 low, 1 high) and receive recv_bytes into
 *     d_recv from the rank across the other face (MPI_Sendrecv with
 *     procneigh[2]); a pointer is NULL where that neighbour does not exist
 *     (MPI_PROC_NULL).  The fix synchronises its stream first; every rank
 *     makes the same calls in the same order.
 *   allreduce: n doubles in place over all ranks, op 0 sum, op 1 max.
 * Both return 0 on success.  Diagnostics and the profile are reduced over
 * the ranks (rank 0 writes), checkpoints are one file per rank; VTK output is
 * refused.  Call before couplb_fix_init; nprocs 1 is the one-rank run. */
typedef struct couplb_fix_comm {
  int   nprocs;
  int   rank;
  int (*sendrecv)(void* ctx, int side, const void* d_send, size_t send_bytes, void* d_recv,
                  size_t recv_bytes);
  int (*allreduce)(void* ctx, double* buf, int n, int op);
  void* ctx;
} couplb_fix_comm;
int  couplb_fix_set_comm(couplb_fix* fx, const couplb_fix_comm* comm);

/* FixCoupLB::setmask: POST_FORCE | END_OF_STEP (fix_couplb.cpp:248-254). */
#define COUPLB_MASK_POST_FORCE  1
#define COUPLB_MASK_END_OF_STEP 2
int  couplb_fix_setmask(void);

/* Hooks (fix_couplb.h:26-30). */
int  couplb_fix_init(couplb_fix* fx, const couplb_domain* dom);       /* :256-482 */
int  couplb_fix_setup(couplb_fix* fx, const couplb_atoms* at,
                      long long ntimestep);                           /* :551-638 */
int  couplb_fix_post_force(couplb_fix* fx, const couplb_atoms* at,
                           long long ntimestep);                      /* :640-651 */
int  couplb_fix_end_of_step(couplb_fix* fx, long long ntimestep);     /* :846-901 */
/* The solid part of end_of_step's VTK output (IO::write_solid_vtk,
 * couplb_io.h:309-614, and the solid .pvd): the atoms are not an argument of
 * end_of_step, so a driver calls this right after it with the same step.  It
 * writes <prefix>_solid_<step>.vtp and <prefix>_solid.pvd when that
 * end_of_step wrote field output and vtk_solid is set; otherwise it returns
 * COUPLB_OK doing nothing.  Files are VTK XML with binary appended data (the
 * reference writes ASCII) and the same names and layout. */
int  couplb_fix_write_solid(couplb_fix* fx, const couplb_atoms* at,
                            long long ntimestep);

/* Accessors for drivers and tests. */
couplb_handle* couplb_fix_handle(couplb_fix* fx);
int  couplb_fix_scales(const couplb_fix* fx, double out[6]);  /* dx dt_LBM vel_scale force_scale nu_lb tau */
int  couplb_fix_last_diag(const couplb_fix* fx, couplb_diag* out);
long long couplb_fix_lbm_steps(const couplb_fix* fx);

#ifdef __cplusplus
}
#endif
#endif /* COUPLB_B200_H */
