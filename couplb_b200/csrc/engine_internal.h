// engine_internal.h -- the lattice handle, shared by engine.cu and the fix
// core.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/couplb_b200.h"

namespace couplb {
struct StencilKey;
}

struct couplb_handle {
  couplb_lattice_params p{};
  int Q = 0;
  size_t N = 0;    // interior nodes
  size_t qs = 0;   // q-plane stride (elements)
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  void* f[2] = {nullptr, nullptr};   // population buffers (A-B)
  int cur = 0;                       // buffer holding the current state
  int poststream = 1;                // 1: f[cur] is post-stream S, 0: post-collision P
  void* F = nullptr;                 // Eulerian force field {fx, fy, fz, 0} per node
  int force_dirty = 0;               // F holds nonzero values
  int force_rows_all = 0;            // F was set from outside: the segment flags do not cover it
  unsigned char* seg_force = nullptr;   // per 8 consecutive nodes: IBM force spread there
  unsigned cur_epoch = 0;            // epoch of the current population state
  void* sbuf = nullptr;              // IBM stencil velocity records (64 x 3 per marker slot)
  couplb::StencilKey* skey = nullptr;   // their keys
  int stencil_cap = 0;
  void* rho_field = nullptr;         // density of the last fused launch (body force, moving walls)
  bool moving_walls = false;         // a face of type 2
  bool idx32 = true;                 // Q * qs fits 32-bit element indices
  int kernel = -1;                   // fused-kernel choice (couplb::KernelKind), -1 auto
  int last_kernel = 0;               // the variant the last LB step ran
  int rho_state = 0;                 // couplb::RhoMode: what the next LB step reads
  void* macro[4] = {nullptr, nullptr, nullptr, nullptr};   // rho(dev), ux, uy, uz
  int macro_valid = 0;               // macro[] are the moments of the current state
  long long lbm_steps = 0;

  int* d_status = nullptr;           // clamp / non-finite counters
  double* d_ftot = nullptr;          // FP64 sum of the spread IBM force
  void* h_small = nullptr;           // pinned host scratch for small read-backs
  int* h_status_ring = nullptr;      // pinned, mapped: two posted copies of the status word
  int* d_status_ring = nullptr;      // the same memory as seen by kernels
  cudaEvent_t status_ev[2] = {nullptr, nullptr};
  long long status_posts = 0;
  void* d_staging = nullptr;         // import / export staging
  size_t staging_bytes = 0;
  void* d_scratch = nullptr;         // reduction partials
  int scratch_blocks = 0;

  couplb_ibm_params ip{};
  int ip_set = 0;
  void* d_x = nullptr;
  void* d_v = nullptr;
  void* d_m = nullptr;
  void* d_fout = nullptr;
  void* d_active = nullptr;
  double* h_fout = nullptr;
  double* h_mass = nullptr;          // pinned host staging of the per-atom masses
  int* h_active = nullptr;           // pinned host staging of the group flags
  int atom_cap = 0;
  // staging hint of the fix core (engine_atom_host_hint): for the next
  // host-array sub-step of hint_n atoms from h_mass / h_active, their group
  // count and whether they are unchanged since their last device copy
  int hint_n = -1, hint_count = 0, hint_unchanged = 0;
  int statics_n = -1;                // d_m / d_active hold the pinned buffers' n atoms

  // IBM forcing method (couplb_set_ibm_method)
  int ibm_method = 0;                // COUPLB_IBM_*
  int ibm_passes = 1;
  double slip_tol = 0.0;
  const couplb_mlp* mlp = nullptr;
  double* d_corr = nullptr;          // per marker: correction beyond the penalty pass
  double* d_dF = nullptr;            // per marker: increment of the current pass
  int method_cap = 0;
  void* d_pass = nullptr;            // two couplb::PassState, alternating per sub-step
  int pass_cur = 0;                  // the one of the last sub-step
  int ibm_resident = 1;              // option: register-resident form when markers fit
  int ibm_window = 0;                // option: 0 clip the IBM window like the reference, 1 wrap
  int ibm_slip = 1;                  // option: ITERATIVE / LEARNED measure the slip after the last pass
  int ibm_group = 8;                 // option: lanes per marker of the single-pass 3D sub-step (8, 32)
  int ibm_block = 128;               // option: threads per block of the grouped sub-step (64, 128, 256)
  int ibm_sort = 16;                 // option: refreshes between re-sorts of the marker order (0: off)
  int* d_order = nullptr;            // marker processing order (k_order_*), its ranks and buckets
  int* d_order_rank = nullptr;
  int* d_order_count = nullptr;
  int order_cap = 0, order_nb = 0;   // capacity of the two per-marker arrays, buckets
  int order_n = -1, order_age = 0;   // markers the order is for, refreshes since it was made
  int* h_order_near = nullptr;       // pinned copy of the near-successor count of the last sort
  int order_identity = -1;           // the last sort kept the index order: 1, else 0
  const void* halo[2] = {nullptr, nullptr};   // z-face halos of a slab decomposition
  const void* ih_vel[2] = {nullptr, nullptr};  // IBM halos of those faces: neighbour moments,
  void* ih_force[2] = {nullptr, nullptr};      // forces spread beyond the face,
  int ih_planes[2] = {0, 0};                   // planes of each
  long long barrier_spin = 1LL << 21;   // option: grid-barrier poll limit of the method kernels
  cudaStream_t copy_stream = nullptr;   // host->device atom copies of couplb_lbm_step_ibm
  cudaEvent_t copy_ev[2] = {nullptr, nullptr};   // main stream reached / copies done
  cudaEvent_t fout_ev[4] = {nullptr, nullptr, nullptr, nullptr};   // force chunks back on the host
  int staged_n = -1;                    // atoms whose x, v engine_host_begin queued
  int coop_blocks[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // resident blocks of k_ibm_method (Roma,
                                                   // Peskin4, learned Roma, learned Peskin4),
                                                   // then of its register-resident form
  double g_lb[3] = {0.0, 0.0, 0.0};  // body force of the last LB step
  float* rec_rows = nullptr;         // training-sample capture
  long long rec_cap = 0, rec_count = 0;

  size_t device_bytes = 0;
  std::string err;
};

namespace couplb {
int engine_macro(couplb_handle* h);
// One LB step (couplb_lbm_step).
int engine_lbm_step(couplb_handle* h, const double* g_lb);
// Pinned host buffers of n masses and n group flags owned by the handle (valid
// until the next call with a larger n), for host drivers that assemble those
// arrays before couplb_ibm_substep, so that every host->device copy of a
// sub-step starts from pinned memory.
int engine_atom_host_buffers(couplb_handle* h, int n, double** mass, int** active);
// After filling those buffers: the group count and whether the values are
// the ones of the previous fill, so the next sub-step neither recounts nor
// copies them again.
void engine_atom_host_hint(couplb_handle* h, int n, int count, int unchanged);
// A refresh sub-step with no coupled atoms on this lattice (other slabs have
// some): only its effect on the density the next LB step reads.
void engine_note_refresh(couplb_handle* h);
// A sub-step of host atom arrays in two calls, so that the caller can fill
// the masses and group flags while the positions travel (and the LB kernel
// runs): engine_host_begin queues the x, v copies on the copy stream and, with
// lbm, the LB step on the lattice's stream; engine_host_finish copies the
// masses and flags unless the hint says they are unchanged, runs the
// sub-step (the refresh one with lbm) and adds the forces to f_add.
int engine_host_begin(couplb_handle* h, bool lbm, const double* g_lb, int n, const double* x, const double* v);
int engine_host_finish(couplb_handle* h, bool lbm, int n, const double* mass, const int* active, double* f_add,
                       int refresh, int* ncoupled);
int engine_ibm(couplb_handle* h, int n, const double* d_x, const double* d_v, const double* d_m,
               const int* d_active, double* d_fout, int accumulate, int refresh);
}  // namespace couplb
