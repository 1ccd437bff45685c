// fix_core.cpp -- layer 2 of the C ABI: the `fix couplb` front end.
//
// Keyword parsing, unit conversion and the init / setup / post_force /
// end_of_step sequencing of FixCoupLB (fix_couplb.cpp), written against plain
// atom arrays so that a LAMMPS fix (or any MD driver) forwards its hooks
// here.  The lattice work goes to the layer-1 engine on the GPU; this file does
// host bookkeeping only.  Error messages are the reference's.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/couplb_b200.h"
#include "engine_internal.h"
#include "vtk_io.h"

using couplb::VtkArray;
using couplb::write_pvd;
using couplb::write_vti;
using couplb::write_vtp;

namespace {

constexpr double kRhoLb = 1.0;   // FixCoupLB::rho_lb (fix_couplb.h:180)
constexpr double kZeroTol = 1e-15, kMaWarn = 0.3, kMaError = 0.5;
constexpr uint32_t kCkptMagic = 0x434C424B;   // "CLBK" (couplb_io.h:21)
constexpr int32_t kCkptVersion = 1;

const char* const kKeywords[] = {"md_per_lb", "xi_ibm",      "gravity", "wall_x",     "wall_y",
                                 "wall_z",    "wall_vel",    "output",  "check_every", "kernel",
                                 "vtk",       "vtk_region",  "vtk_solid", "checkpoint", "restart",
                                 "precision", "ibm_method", "ibm_passes", "slip_tol", "mlp_model",
                                 "ibm_window", nullptr};

// is_couplb_keyword (fix_couplb.cpp:22-36), plus the keywords of this
// implementation (precision, IBM forcing method).
bool is_keyword(const char* s) {
  for (int i = 0; kKeywords[i]; i++)
    if (std::strcmp(s, kKeywords[i]) == 0) return true;
  return false;
}

struct ParseError {
  std::string msg;
};

[[noreturn]] void perr(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw ParseError{buf};
}

// std::stoi / std::stod semantics: leading number parsed, error when none.
int to_int(const char* s) {
  errno = 0;
  char* end = nullptr;
  const long v = std::strtol(s, &end, 10);
  if (end == s) perr("fix couplb: expected an integer, got '%s'", s);
  if (errno == ERANGE || v > INT32_MAX || v < INT32_MIN) perr("fix couplb: integer out of range: '%s'", s);
  return (int)v;
}

double to_double(const char* s) {
  errno = 0;
  char* end = nullptr;
  const double v = std::strtod(s, &end);
  if (end == s) perr("fix couplb: expected a number, got '%s'", s);
  return v;
}

void copy_str(char* dst, const char* src) {
  std::strncpy(dst, src, COUPLB_PATH_MAX - 1);
  dst[COUPLB_PATH_MAX - 1] = 0;
}

}  // namespace

struct couplb_fix {
  couplb_fix_config cfg{};
  couplb_handle* h = nullptr;
  couplb_mlp* mlp = nullptr;          // network of ibm_method learned
  int device = 0;
  int rank = 0;
  bool inited = false;
  bool is3d = true;
  double dx = 0, inv_dx = 0, dt = 0, dt_LBM = 0, vel_scale = 0, nu_lb = 0, tau = 0,
         force_scale = 0;
  double domain_lo[3] = {0, 0, 0}, domain_hi[3] = {0, 0, 0};
  int nl[3] = {0, 0, 0}, off[3] = {0, 0, 0};
  int md_sub_count = 0;
  bool ibm_has_particles = false;
  long long next_output = 0, next_check = -1, next_vtk = -1, next_checkpoint = -1;
  long long lbm_step_count = 0;
  double gvals[3] = {0, 0, 0};
  couplb_gravity_fn gcb = nullptr;
  void* gctx = nullptr;
  couplb_log_fn logcb = nullptr;
  void* logctx = nullptr;
  couplb_diag last_diag{};
  std::string err;
  int vtk_region[6] = {0, 0, 0, 0, 0, 0};
  double vtk_rlo[3] = {0, 0, 0}, vtk_rhi[3] = {0, 0, 0};   // clamped region, MD units
  std::vector<long long> vtk_steps;   // steps with field output (the .pvd series)
  long long vtk_last = -1;            // step of the last field output
  // several ranks along z (couplb_fix_set_comm): this rank's slab and its halos
  couplb_fix_comm comm{};
  bool decomposed = false;
  int nbr[2] = {0, 0};                // a neighbour across z face side
  int ih_own[2] = {0, 0};             // IBM halo planes beyond each face of this slab
  int ih_nbr[2] = {0, 0};             // planes of the neighbours' halos that face this slab
  void* pop_send[2] = {nullptr, nullptr};
  void* pop_recv[2] = {nullptr, nullptr};
  void* vel[2] = {nullptr, nullptr};  // neighbour moments beyond each face
  void* frc[2] = {nullptr, nullptr};  // forces spread beyond each face
  void* msend[2] = {nullptr, nullptr};   // this slab's moments for the neighbours
  void* frecv[2] = {nullptr, nullptr};   // the neighbours' forces on this slab
  bool fold_pending = false;

  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  int engine_fail(int rc) {
    err = couplb_last_error(h);
    return rc;
  }
  void log(const char* fmt, ...) {
    if (!logcb || rank != 0) return;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    logcb(logctx, buf);
  }
};

namespace {

// ---- several ranks along z: the slab halos through the host communicator --
void free_slab_buffers(couplb_fix* F) {
  void** bufs[] = {F->pop_send, F->pop_recv, F->vel, F->frc, F->msend, F->frecv};
  for (void** b : bufs)
    for (int s = 0; s < 2; s++)
      if (b[s]) { cudaFree(b[s]); b[s] = nullptr; }
}

int slab_alloc(couplb_fix* F, void** p, size_t bytes) {
  if (!bytes) return COUPLB_OK;
  if (cudaSetDevice(F->device) != cudaSuccess || cudaMalloc(p, bytes) != cudaSuccess ||
      cudaMemsetAsync(*p, 0, bytes, F->h->stream) != cudaSuccess)
    return F->fail(COUPLB_ERR_CUDA, "fix couplb: cannot allocate %zu bytes of slab halo", bytes);
  return COUPLB_OK;
}

// One sendrecv of the communicator after the lattice's stream has finished
// what the buffers depend on.
int slab_sendrecv(couplb_fix* F, int side, const void* send, size_t sb, void* recv, size_t rb) {
  int rc = couplb_synchronize(F->h);
  if (rc) return F->engine_fail(rc);
  if (F->comm.sendrecv(F->comm.ctx, side, send, send ? sb : 0, recv, recv ? rb : 0) != 0)
    return F->fail(COUPLB_ERR_CUDA, "fix couplb: halo exchange across z face %d failed", side);
  return COUPLB_OK;
}

int slab_allreduce(couplb_fix* F, double* buf, int n, int op) {
  if (!F->decomposed) return COUPLB_OK;
  if (F->comm.allreduce(F->comm.ctx, buf, n, op) != 0)
    return F->fail(COUPLB_ERR_CUDA, "fix couplb: allreduce over the ranks failed");
  return COUPLB_OK;
}

// After an LB step: the populations that cross each bound face (5 planes),
// then the moments of the planes the neighbours' marker windows reach.
int slab_exchange_state(couplb_fix* F, bool populations) {
  if (!F->decomposed) return COUPLB_OK;
  int rc;
  if (populations) {
    const size_t pb = couplb_halo_bytes(F->h);
    for (int s = 0; s < 2; s++)
      if (F->nbr[s] && (rc = couplb_halo_pack(F->h, s, F->pop_send[s]))) return F->engine_fail(rc);
    // up: my top planes into the slab above, the slab below's into my low halo
    if ((rc = slab_sendrecv(F, 1, F->nbr[1] ? F->pop_send[1] : nullptr, pb, F->nbr[0] ? F->pop_recv[0] : nullptr,
                            pb)))
      return rc;
    if ((rc = slab_sendrecv(F, 0, F->nbr[0] ? F->pop_send[0] : nullptr, pb, F->nbr[1] ? F->pop_recv[1] : nullptr,
                            pb)))
      return rc;
  }
  for (int s = 0; s < 2; s++)
    if (F->nbr[s] && (rc = couplb_ibm_halo_moments(F->h, s, F->ih_nbr[s], F->msend[s]))) return F->engine_fail(rc);
  const size_t m1 = couplb_ibm_halo_bytes(F->h, F->ih_nbr[1]), v0 = couplb_ibm_halo_bytes(F->h, F->ih_own[0]);
  const size_t m0 = couplb_ibm_halo_bytes(F->h, F->ih_nbr[0]), v1 = couplb_ibm_halo_bytes(F->h, F->ih_own[1]);
  if ((rc = slab_sendrecv(F, 1, F->nbr[1] ? F->msend[1] : nullptr, m1, F->nbr[0] ? F->vel[0] : nullptr, v0)))
    return rc;
  return slab_sendrecv(F, 0, F->nbr[0] ? F->msend[0] : nullptr, m0, F->nbr[1] ? F->vel[1] : nullptr, v1);
}

// Before an LB step: the forces this slab spread beyond its faces go to the
// neighbours, theirs on this slab are added to its field.
int slab_fold(couplb_fix* F) {
  if (!F->decomposed) return COUPLB_OK;   // a collective: every rank, every LB step
  const size_t f0 = couplb_ibm_halo_bytes(F->h, F->ih_own[0]), r1 = couplb_ibm_halo_bytes(F->h, F->ih_nbr[1]);
  const size_t f1 = couplb_ibm_halo_bytes(F->h, F->ih_own[1]), r0 = couplb_ibm_halo_bytes(F->h, F->ih_nbr[0]);
  int rc;
  if ((rc = slab_sendrecv(F, 0, F->nbr[0] ? F->frc[0] : nullptr, f0, F->nbr[1] ? F->frecv[1] : nullptr, r1)))
    return rc;
  if ((rc = slab_sendrecv(F, 1, F->nbr[1] ? F->frc[1] : nullptr, f1, F->nbr[0] ? F->frecv[0] : nullptr, r0)))
    return rc;
  for (int s = 0; s < 2; s++) {
    if (!F->nbr[s]) continue;
    if ((rc = couplb_ibm_halo_fold(F->h, s, F->ih_nbr[s], F->frecv[s]))) return F->engine_fail(rc);
    if (cudaMemsetAsync(F->frc[s], 0, couplb_ibm_halo_bytes(F->h, F->ih_own[s]), F->h->stream) != cudaSuccess)
      return F->fail(COUPLB_ERR_CUDA, "fix couplb: cannot clear a force halo");
  }
  F->fold_pending = false;
  return COUPLB_OK;
}

// FixCoupLB::write_profile (fix_couplb.cpp:903-979) for one rank.
int write_profile(couplb_fix* F, long long step) {
  const int ny = F->nl[1];
  std::vector<double> su(ny), sv(ny), sr(ny);
  int rc = couplb_y_profile(F->h, su.data(), sv.data(), sr.data());
  if (rc) return F->engine_fail(rc);
  // sums over the ranks' slabs (fix_couplb.cpp:955-958)
  if ((rc = slab_allreduce(F, su.data(), ny, 0)) || (rc = slab_allreduce(F, sv.data(), ny, 0)) ||
      (rc = slab_allreduce(F, sr.data(), ny, 0)))
    return rc;
  if (F->rank != 0) return COUPLB_OK;
  const int Ny = F->cfg.Ny;
  const int cxz = F->nl[0] * (F->is3d ? (F->decomposed ? F->cfg.Nz : F->nl[2]) : 1);
  std::vector<double> ux(Ny, 0.0), uy(Ny, 0.0), rr(Ny, 0.0);
  std::vector<int> cnt(Ny, 0);
  for (int j = 0; j < ny; j++) {
    const int gy = F->off[1] + j;
    if (gy < 0 || gy >= Ny) continue;
    ux[gy] = su[j]; uy[gy] = sv[j]; rr[gy] = sr[j]; cnt[gy] = cxz;
  }
  FILE* fp = std::fopen(F->cfg.output_file, "a");
  if (!fp) {
    F->log("CoupLB WARNING: cannot open %s\n", F->cfg.output_file);
    return COUPLB_OK;
  }
  std::fprintf(fp, "# step = %lld\n", step);
  for (int j = 0; j < Ny; j++) {
    const double inv = (cnt[j] > 0) ? 1.0 / cnt[j] : 0.0;
    std::fprintf(fp, "%lld %d %.6f %.8f %.10e %.10e\n", step, j, F->domain_lo[1] + (double)j * F->dx,
                 F->cfg.rho * (rr[j] * inv), F->vel_scale * (ux[j] * inv), F->vel_scale * (uy[j] * inv));
  }
  std::fprintf(fp, "\n");
  std::fclose(fp);
  return COUPLB_OK;
}

// IO::write_vtk (couplb_io.h:42-281) + IO::write_pvd (:284-295): the cells of
// the region (default: the whole grid) with rho * rho_phys, velocity *
// vel_scale, the node type (0: interior) and the force field * force_scale,
// as <prefix>_<step>.vti; the series is rewritten as <prefix>.pvd.
int write_field_vtk(couplb_fix* F, long long step) {
  const couplb_fix_config& c = F->cfg;
  const int Nz = F->is3d ? c.Nz : 1;
  const int r0[6] = {0, c.Nx, 0, c.Ny, 0, Nz};
  const int* r = c.has_vtk_region ? F->vtk_region : r0;
  const int ext[3] = {r[1] - r[0], r[3] - r[2], r[5] - r[4]};
  const size_t ncell = (size_t)ext[0] * ext[1] * ext[2];
  const size_t G = couplb_ghost_nodes(F->h);
  std::vector<double> rho(G), ux(G), uy(G), uz(G), fx(G), fy(G), fz(G);
  int rc = couplb_get_macroscopic(F->h, rho.data(), ux.data(), uy.data(), uz.data());
  if (!rc) rc = couplb_get_force_field(F->h, fx.data(), fy.data(), fz.data());
  if (rc) return F->engine_fail(rc);
  const size_t gx = (size_t)F->nl[0] + 2, gy = (size_t)F->nl[1] + 2;
  std::vector<VtkArray> a(4);
  a[0].name = "rho";
  a[1].name = "velocity_phys"; a[1].ncomp = 3;
  a[2].name = "type"; a[2].is_int = true;
  a[3].name = "force_phys"; a[3].ncomp = 3;
  a[0].f.resize(ncell); a[1].f.resize(3 * ncell); a[2].i.assign(ncell, 0); a[3].f.resize(3 * ncell);
  size_t c_ = 0;
  for (int k = r[4]; k < r[5]; k++)
    for (int j = r[2]; j < r[3]; j++)
      for (int i = r[0]; i < r[1]; i++, c_++) {
        const size_t n = (size_t)(i + 1) + gx * ((size_t)(j + 1) + gy * (size_t)(F->is3d ? k + 1 : 0));
        a[0].f[c_] = rho[n] * c.rho;
        a[1].f[3 * c_] = ux[n] * F->vel_scale;
        a[1].f[3 * c_ + 1] = uy[n] * F->vel_scale;
        a[1].f[3 * c_ + 2] = uz[n] * F->vel_scale;
        a[3].f[3 * c_] = fx[n] * F->force_scale;
        a[3].f[3 * c_ + 1] = fy[n] * F->force_scale;
        a[3].f[3 * c_ + 2] = fz[n] * F->force_scale;
      }
  if (F->rank != 0) return COUPLB_OK;
  char fname[COUPLB_PATH_MAX + 32];
  std::snprintf(fname, sizeof fname, "%s_%06lld.vti", c.vtk_prefix, step);
  const double origin[3] = {F->domain_lo[0] + r[0] * F->dx, F->domain_lo[1] + r[2] * F->dx,
                            F->domain_lo[2] + r[4] * F->dx};
  if (!write_vti(fname, ext, origin, F->dx, a)) {
    F->log("CoupLB IO: cannot open %s\n", fname);
    return COUPLB_OK;
  }
  F->log("CoupLB: VTK written at step %lld -> %s (%dx%dx%d region)\n", step, fname, ext[0], ext[1], ext[2]);
  F->vtk_steps.push_back(step);
  F->vtk_last = step;
  write_pvd(std::string(c.vtk_prefix) + ".pvd", c.vtk_prefix, F->vtk_steps, F->dt, "vti");
  return COUPLB_OK;
}

// Attributes of vtk_solid (couplb_io.h:366-411): scalars, and the vector
// groups that are written as one 3-component array when all three
// components are asked for.
struct SolidAttr {
  const char* name;
  const char* group;   // vector group or nullptr
  int comp;
};
const SolidAttr kSolidAttrs[] = {
    {"id", nullptr, 0},         {"type", nullptr, 0},       {"mol", nullptr, 0},
    {"mass", nullptr, 0},       {"diameter", nullptr, 0},   {"x", "position", 0},
    {"y", "position", 1},       {"z", "position", 2},       {"vx", "velocity", 0},
    {"vy", "velocity", 1},      {"vz", "velocity", 2},      {"fx", "force", 0},
    {"fy", "force", 1},         {"fz", "force", 2},         {"mux", "dipole", 0},
    {"muy", "dipole", 1},       {"muz", "dipole", 2},       {"omegax", "omega", 0},
    {"omegay", "omega", 1},     {"omegaz", "omega", 2},     {"tqx", "torque", 0},
    {"tqy", "torque", 1},       {"tqz", "torque", 2}};

const SolidAttr* find_attr(const char* a) {
  for (const SolidAttr& s : kSolidAttrs)
    if (!std::strcmp(s.name, a)) return &s;
  return nullptr;
}

bool solid_attr_known(const char* a) { return find_attr(a) != nullptr; }

// Per-atom value of an attribute; false if the array is not available.
bool attr_value(const couplb_atoms* at, const char* name, int i, double* v) {
  const std::string a(name);
  if (a == "id") { if (!at->tag) return false; *v = (double)at->tag[i]; }
  else if (a == "type") { if (!at->type) return false; *v = at->type[i]; }
  else if (a == "mol") { if (!at->molecule) return false; *v = (double)at->molecule[i]; }
  else if (a == "mass") {
    if (at->rmass) *v = at->rmass[i];
    else if (at->mass && at->type) *v = at->mass[at->type[i]];
    else return false;
  } else if (a == "diameter") { if (!at->radius) return false; *v = 2.0 * at->radius[i]; }
  else if (a == "x" || a == "y" || a == "z") *v = at->x[3 * i + (a[0] - 'x')];
  else if (a == "vx" || a == "vy" || a == "vz") *v = at->v[3 * i + (a[1] - 'x')];
  else if (a == "fx" || a == "fy" || a == "fz") *v = at->f[3 * i + (a[1] - 'x')];
  else if (a.rfind("mu", 0) == 0) { if (!at->mu) return false; *v = at->mu[4 * i + (a[2] - 'x')]; }
  else if (a.rfind("omega", 0) == 0) { if (!at->omega) return false; *v = at->omega[3 * i + (a[5] - 'x')]; }
  else if (a.rfind("tq", 0) == 0) { if (!at->torque) return false; *v = at->torque[3 * i + (a[2] - 'x')]; }
  else return false;
  return true;
}

// IO::write_solid_vtk (couplb_io.h:309-614) + IO::write_pvd_vtp: the group's
// atoms inside the clamped VTK region as PolyData vertices.
int write_solid_vtk(couplb_fix* F, const couplb_atoms* at, long long step) {
  const couplb_fix_config& c = F->cfg;
  const int na = c.vtk_solid_nattr;
  // output fields: a vector group once when all three components are asked
  struct Out { std::string name; const char* comp[3]; int ncomp; };
  std::vector<Out> outs;
  std::vector<std::string> done;
  for (int k = 0; k < na; k++) {
    const SolidAttr* s = find_attr(c.vtk_solid_attr[k]);
    if (!s) return F->fail(COUPLB_ERR_ARG, "fix couplb vtk_solid: unknown attribute '%s'", c.vtk_solid_attr[k]);
    if (s->group) {
      bool seen = false;
      for (const std::string& d : done) seen |= (d == s->group);
      if (seen) continue;
      const char* comp[3] = {nullptr, nullptr, nullptr};
      for (int m = 0; m < na; m++) {
        const SolidAttr* q = find_attr(c.vtk_solid_attr[m]);
        if (q && q->group && !std::strcmp(q->group, s->group)) comp[q->comp] = q->name;
      }
      if (comp[0] && comp[1] && comp[2]) {
        outs.push_back({s->group, {comp[0], comp[1], comp[2]}, 3});
        done.push_back(s->group);
        continue;
      }
    }
    outs.push_back({s->name, {s->name, nullptr, nullptr}, 1});
  }
  std::vector<double> pts;
  std::vector<VtkArray> fields(outs.size());
  for (size_t o = 0; o < outs.size(); o++) { fields[o].name = outs[o].name; fields[o].ncomp = outs[o].ncomp; }
  for (int i = 0; i < at->nlocal; i++) {
    if (at->mask && !(at->mask[i] & at->groupbit)) continue;
    if (c.has_vtk_region) {
      bool in = true;
      for (int d = 0; d < 3; d++) in &= at->x[3 * i + d] >= F->vtk_rlo[d] && at->x[3 * i + d] < F->vtk_rhi[d];
      if (!in) continue;
    }
    for (int d = 0; d < 3; d++) pts.push_back(at->x[3 * i + d]);
    for (size_t o = 0; o < outs.size(); o++)
      for (int d = 0; d < outs[o].ncomp; d++) {
        double v = 0.0;
        if (!attr_value(at, outs[o].comp[d], i, &v))
          return F->fail(COUPLB_ERR_ARG, "fix couplb vtk_solid: attribute '%s' is not available for these atoms",
                         outs[o].comp[d]);
        fields[o].f.push_back(v);
      }
  }
  if (F->rank != 0) return COUPLB_OK;
  char fname[COUPLB_PATH_MAX + 40];
  std::snprintf(fname, sizeof fname, "%s_solid_%06lld.vtp", c.vtk_prefix, step);
  if (!write_vtp(fname, pts, fields)) return F->fail(COUPLB_ERR_IO, "CoupLB IO: cannot open %s", fname);
  F->log("CoupLB: solid VTK written at step %lld -> %s (%d atoms, %d fields)\n", step, fname,
         (int)(pts.size() / 3), (int)fields.size());
  write_pvd(std::string(c.vtk_prefix) + "_solid.pvd", std::string(c.vtk_prefix) + "_solid", F->vtk_steps,
            F->dt, "vtp");
  return COUPLB_OK;
}

// IO::write_checkpoint (couplb_io.h:669-719): prefix.<rank>.clbk, header then
// Q x G doubles of f including ghost nodes.
int write_checkpoint(couplb_fix* F, long long step) {
  char fname[COUPLB_PATH_MAX + 32];
  std::snprintf(fname, sizeof(fname), "%s.%d.clbk", F->cfg.checkpoint_prefix, F->rank);
  const int Q = F->is3d ? 19 : 9;
  const size_t G = couplb_ghost_nodes(F->h);
  std::vector<double> f((size_t)Q * G);
  int rc = couplb_get_populations(F->h, f.data());
  if (rc) return F->engine_fail(rc);
  FILE* fp = std::fopen(fname, "wb");
  if (!fp) return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d cannot open %s for writing", F->rank, fname);
  const uint32_t magic = kCkptMagic;
  const int32_t version = kCkptVersion;
  const int64_t s64 = step;
  const int32_t D = F->is3d ? 3 : 2, Qi = Q;
  const int32_t dims[3] = {F->nl[0], F->nl[1], F->is3d ? F->nl[2] : 1};
  const int32_t offs[3] = {F->off[0], F->off[1], F->is3d ? F->off[2] : 0};
  const int32_t glob[3] = {F->cfg.Nx, F->cfg.Ny, F->is3d ? F->cfg.Nz : 1};
  bool ok = std::fwrite(&magic, 4, 1, fp) == 1 && std::fwrite(&version, 4, 1, fp) == 1 &&
            std::fwrite(&s64, 8, 1, fp) == 1 && std::fwrite(&D, 4, 1, fp) == 1 &&
            std::fwrite(&Qi, 4, 1, fp) == 1 && std::fwrite(dims, 4, 3, fp) == 3 &&
            std::fwrite(offs, 4, 3, fp) == 3 && std::fwrite(glob, 4, 3, fp) == 3 &&
            std::fwrite(f.data(), sizeof(double), f.size(), fp) == f.size();
  std::fclose(fp);
  if (!ok) return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d write error in %s", F->rank, fname);
  F->log("CoupLB: checkpoint written at step %lld -> %s.*.clbk\n", step, F->cfg.checkpoint_prefix);
  return COUPLB_OK;
}

// IO::read_checkpoint (couplb_io.h:721-829): every header field validated.
int read_checkpoint(couplb_fix* F, long long* step_out) {
  char fname[COUPLB_PATH_MAX + 32];
  std::snprintf(fname, sizeof(fname), "%s.%d.clbk", F->cfg.restart_prefix, F->rank);
  FILE* fp = std::fopen(fname, "rb");
  if (!fp) return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d cannot open %s for reading", F->rank, fname);
  struct Closer { FILE* f; ~Closer() { std::fclose(f); } } closer{fp};
  uint32_t magic = 0;
  if (std::fread(&magic, 4, 1, fp) != 1 || magic != kCkptMagic)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d bad magic in %s", F->rank, fname);
  int32_t version = 0;
  if (std::fread(&version, 4, 1, fp) != 1 || version != kCkptVersion)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d unsupported version %d in %s", F->rank, version, fname);
  int64_t s64 = 0;
  if (std::fread(&s64, 8, 1, fp) != 1)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d truncated header (step) in %s", F->rank, fname);
  int32_t D = 0, Q = 0;
  if (std::fread(&D, 4, 1, fp) != 1 || std::fread(&Q, 4, 1, fp) != 1)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d truncated header (D/Q) in %s", F->rank, fname);
  const int eD = F->is3d ? 3 : 2, eQ = F->is3d ? 19 : 9;
  if (D != eD || Q != eQ)
    return F->fail(COUPLB_ERR_IO,
                   "CoupLB IO: rank %d D/Q mismatch in %s (file: D=%d Q=%d, expected: D=%d Q=%d)",
                   F->rank, fname, D, Q, eD, eQ);
  int32_t dims[3], offs[3], glob[3];
  if (std::fread(dims, 4, 3, fp) != 3 || std::fread(offs, 4, 3, fp) != 3 || std::fread(glob, 4, 3, fp) != 3)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d truncated header (dims) in %s", F->rank, fname);
  const int nz = F->is3d ? F->nl[2] : 1;
  if (dims[0] != F->nl[0] || dims[1] != F->nl[1] || dims[2] != nz)
    return F->fail(COUPLB_ERR_IO,
                   "CoupLB IO: rank %d local grid mismatch in %s (file: %dx%dx%d, current: %dx%dx%d)",
                   F->rank, fname, dims[0], dims[1], dims[2], F->nl[0], F->nl[1], nz);
  const int oz = F->is3d ? F->off[2] : 0;
  if (offs[0] != F->off[0] || offs[1] != F->off[1] || offs[2] != oz)
    return F->fail(COUPLB_ERR_IO,
                   "CoupLB IO: rank %d offset mismatch in %s (file: %d,%d,%d, current: %d,%d,%d)",
                   F->rank, fname, offs[0], offs[1], offs[2], F->off[0], F->off[1], oz);
  const int gz = F->is3d ? F->cfg.Nz : 1;
  if (glob[0] != F->cfg.Nx || glob[1] != F->cfg.Ny || glob[2] != gz)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d global grid mismatch in %s", F->rank, fname);
  const size_t nf = (size_t)Q * couplb_ghost_nodes(F->h);
  std::vector<double> f(nf);
  const size_t nread = std::fread(f.data(), sizeof(double), nf, fp);
  if (nread != nf)
    return F->fail(COUPLB_ERR_IO, "CoupLB IO: rank %d short read in %s (%zu/%zu doubles)", F->rank,
                   fname, nread, nf);
  int rc = couplb_set_populations(F->h, f.data());
  if (rc) return F->engine_fail(rc);
  *step_out = s64;
  F->log("CoupLB: checkpoint loaded from step %lld <- %s.*.clbk\n", (long long)s64, F->cfg.restart_prefix);
  F->log("CoupLB WARNING: LAMMPS timestep is NOT updated by checkpoint.\n"
         "  Use 'reset_timestep %lld' in your input script if needed.\n", (long long)s64);
  return COUPLB_OK;
}

// FixCoupLB::do_ibm_sub_coupling (fix_couplb.cpp:730-798).  With lbm, the
// LB step of the cycle (do_lbm_step with body force g_lb, or none when
// g_lb is null) is queued first, the position copies beside it, and the host
// loop over the atoms runs while both are in flight.
int ibm_sub_coupling(couplb_fix* F, const couplb_atoms* at, bool lbm = false,
                     const double* g_lb = nullptr) {
  const bool first = (F->md_sub_count == 0);
  const int nl = at ? at->nlocal : 0;
  // the position copies (and the cycle's LB step) start before the loop over
  // the atoms below
  int rc0 = couplb::engine_host_begin(F->h, lbm, g_lb, nl, nl ? at->x : nullptr, nl ? at->v : nullptr);
  if (rc0) return F->engine_fail(rc0);
  // masses and group flags go to pinned buffers of the lattice handle, so the
  // engine's host->device copies of a sub-step start from pinned memory
  double* mass_buf = nullptr;
  int* active_buf = nullptr;
  if ((rc0 = couplb::engine_atom_host_buffers(F->h, nl, &mass_buf, &active_buf))) return F->engine_fail(rc0);
  int ng = 0;
  int changed = 0;
  // every value is written and compared without a branch (m != old is also
  // true for NaN), so the loop vectorises
  auto fill = [&](auto mass_of) {
    const int* mask = at->mask;
    const int gb = at->groupbit;
    for (int i = 0; i < nl; i++) {
      const int act = mask ? ((mask[i] & gb) != 0) : 1;
      const double m = mass_of(i);
      changed |= (active_buf[i] != act) | (mass_buf[i] != m);
      active_buf[i] = act;
      mass_buf[i] = m;
      ng += act;
    }
  };
  if (nl > 0) {
    if (at->rmass) fill([r = at->rmass](int i) { return r[i]; });
    else if (at->mass) fill([m = at->mass, t = at->type](int i) { return m[t[i]]; });
    else fill([](int) { return 1.0; });
  }
  couplb::engine_atom_host_hint(F->h, nl, ng, changed ? 0 : 1);
  // the group count is global (fix_couplb.cpp:743-747)
  double ng_all = ng;
  if (F->decomposed) {
    int rca = slab_allreduce(F, &ng_all, 1, 0);
    if (rca) return rca;
  }
  if (ng_all == 0) {
    // the cycle's LB step is queued already
    F->ibm_has_particles = false;
    return COUPLB_OK;
  }
  const int refresh = (first || !F->ibm_has_particles) ? 1 : 0;
  F->ibm_has_particles = true;
  if (ng == 0) {
    // a slab without coupled atoms while other slabs have some: the refresh
    // still happens here (its density state), nothing is spread
    if (refresh) couplb::engine_note_refresh(F->h);
    return COUPLB_OK;
  }
  int nc = 0;
  const int rc = couplb::engine_host_finish(F->h, lbm, nl, mass_buf, active_buf, at->f, refresh, &nc);
  if (rc) return F->engine_fail(rc);
  return COUPLB_OK;
}

}  // namespace

extern "C" {

int couplb_fix_setmask(void) { return COUPLB_MASK_POST_FORCE | COUPLB_MASK_END_OF_STEP; }

// FixCoupLB::FixCoupLB (fix_couplb.cpp:71-238)
int couplb_fix_parse(int narg, const char* const* arg, int dimension, couplb_fix_config* cfg,
                     char* err, int errlen) {
  if (!cfg || !arg) return COUPLB_ERR_ARG;
  couplb_fix_config c;
  std::memset(&c, 0, sizeof(c));
  try {
    if (narg < 8) perr("Illegal fix couplb command: need Nx Ny Nz nu rho");
    c.Nx = to_int(arg[3]); c.Ny = to_int(arg[4]); c.Nz = to_int(arg[5]);
    c.nu = to_double(arg[6]); c.rho = to_double(arg[7]);
    if (c.Nx <= 0 || c.Ny <= 0 || c.Nz <= 0) perr("fix couplb: Nx, Ny, and Nz must be positive");
    if (c.nu <= 0.0 || !std::isfinite(c.nu)) perr("fix couplb: viscosity must be positive and finite");
    if (c.rho <= 0.0 || !std::isfinite(c.rho)) perr("fix couplb: density must be positive and finite");
    c.md_per_lb = 1;
    c.xi_ibm = 1.0;
    copy_str(c.output_file, "couplb_profile.dat");
    copy_str(c.vtk_prefix, "couplb_vtk");
    copy_str(c.checkpoint_prefix, "couplb_ckpt");
    c.delta = COUPLB_DELTA_ROMA;
    c.precision = COUPLB_FP64;
    c.ibm_method = COUPLB_IBM_SINGLE;
    c.ibm_passes = 5;
    c.slip_tol = 0.0;
    int iarg = 8;
    while (iarg < narg) {
      const char* kw = arg[iarg];
      if (!is_keyword(kw)) perr("Unknown fix couplb keyword: %s", kw);
      if (!std::strcmp(kw, "md_per_lb")) {
        if (iarg + 2 > narg) perr("fix couplb md_per_lb: need 1 value");
        c.md_per_lb = to_int(arg[iarg + 1]);
        if (c.md_per_lb < 1) perr("fix couplb: md_per_lb must be >= 1");
        iarg += 2;
      } else if (!std::strcmp(kw, "xi_ibm")) {
        if (iarg + 2 > narg) perr("fix couplb xi_ibm: need 1 value");
        c.xi_ibm = to_double(arg[iarg + 1]);
        if (c.xi_ibm <= 0.0 || c.xi_ibm > 1.0 || !std::isfinite(c.xi_ibm))
          perr("fix couplb: xi_ibm must satisfy 0 < xi_ibm <= 1");
        iarg += 2;
      } else if (!std::strcmp(kw, "gravity")) {
        if (iarg + 4 > narg) perr("fix couplb gravity: need 3 values");
        for (int d = 0; d < 3; d++) {
          const char* a = arg[iarg + 1 + d];
          if (std::strstr(a, "v_") == a) {
            std::strncpy(c.gvar[d], a + 2, 63);
            c.gvar[d][63] = 0;
            c.gstyle[d] = COUPLB_G_EQUAL;
          } else {
            c.gconst[d] = to_double(a);
            c.gstyle[d] = COUPLB_G_CONSTANT;
          }
        }
        iarg += 4;
      } else if (!std::strcmp(kw, "wall_x") || !std::strcmp(kw, "wall_y") || !std::strcmp(kw, "wall_z")) {
        const int d = kw[5] - 'x';
        if (iarg + 3 > narg) perr("fix couplb %s: need 2 values", kw);
        const int lo = to_int(arg[iarg + 1]), hi = to_int(arg[iarg + 2]);
        c.wall[2 * d] = lo;
        c.wall[2 * d + 1] = hi;
        if (lo < 0 || lo > 4 || hi < 0 || hi > 4) perr("fix couplb: %s types must be in [0,4]", kw);
        iarg += 3;
      } else if (!std::strcmp(kw, "wall_vel")) {
        if (iarg + 4 > narg) perr("fix couplb wall_vel: need 3 values");
        for (int d = 0; d < 3; d++) c.wall_vel[d] = to_double(arg[iarg + 1 + d]);
        iarg += 4;
      } else if (!std::strcmp(kw, "output")) {
        if (iarg + 3 > narg) perr("fix couplb output: need 2 values");
        c.output_every = to_int(arg[iarg + 1]);
        copy_str(c.output_file, arg[iarg + 2]);
        if (c.output_every < 0) perr("fix couplb: output frequency cannot be negative");
        iarg += 3;
      } else if (!std::strcmp(kw, "check_every")) {
        if (iarg + 2 > narg) perr("fix couplb check_every: need 1 value");
        c.check_every = to_int(arg[iarg + 1]);
        if (c.check_every < 0) perr("fix couplb: check_every cannot be negative");
        iarg += 2;
      } else if (!std::strcmp(kw, "kernel")) {
        if (iarg + 2 > narg) perr("fix couplb kernel: need 1 value");
        if (!std::strcmp(arg[iarg + 1], "roma")) c.delta = COUPLB_DELTA_ROMA;
        else if (!std::strcmp(arg[iarg + 1], "peskin4")) c.delta = COUPLB_DELTA_PESKIN4;
        else perr("fix couplb kernel: use roma or peskin4");
        iarg += 2;
      } else if (!std::strcmp(kw, "vtk")) {
        if (iarg + 3 > narg) perr("fix couplb vtk: need N prefix");
        c.vtk_every = to_int(arg[iarg + 1]);
        copy_str(c.vtk_prefix, arg[iarg + 2]);
        if (c.vtk_every < 0) perr("fix couplb: vtk frequency cannot be negative");
        iarg += 3;
      } else if (!std::strcmp(kw, "vtk_region")) {
        iarg++;
        int nreg = 0;
        while (iarg + nreg < narg && !is_keyword(arg[iarg + nreg])) nreg++;
        if (nreg != 4 && nreg != 6)
          perr("fix couplb vtk_region: need 4 values (2D: xlo xhi ylo yhi) or 6 values (3D: xlo xhi ylo yhi zlo zhi)");
        c.vtk_rlo[0] = to_double(arg[iarg]); c.vtk_rhi[0] = to_double(arg[iarg + 1]);
        c.vtk_rlo[1] = to_double(arg[iarg + 2]); c.vtk_rhi[1] = to_double(arg[iarg + 3]);
        if (nreg == 6) { c.vtk_rlo[2] = to_double(arg[iarg + 4]); c.vtk_rhi[2] = to_double(arg[iarg + 5]); }
        else { c.vtk_rlo[2] = -1e30; c.vtk_rhi[2] = 1e30; }
        c.has_vtk_region = 1;
        c.vtk_region_n = nreg;
        iarg += nreg;
      } else if (!std::strcmp(kw, "vtk_solid")) {
        if (c.vtk_solid_nattr) perr("fix couplb vtk_solid: keyword specified more than once");
        iarg++;
        int na = 0;
        while (iarg < narg && !is_keyword(arg[iarg])) {
          if (na >= COUPLB_VTK_MAX_ATTR) perr("fix couplb vtk_solid: too many attributes");
          std::snprintf(c.vtk_solid_attr[na], sizeof(c.vtk_solid_attr[na]), "%s", arg[iarg]);
          na++;
          iarg++;
        }
        if (na == 0) perr("fix couplb vtk_solid: need at least one attribute");
        c.vtk_solid_nattr = na;
      } else if (!std::strcmp(kw, "checkpoint")) {
        if (iarg + 3 > narg) perr("fix couplb checkpoint: need N prefix");
        c.checkpoint_every = to_int(arg[iarg + 1]);
        copy_str(c.checkpoint_prefix, arg[iarg + 2]);
        if (c.checkpoint_every < 0) perr("fix couplb: checkpoint frequency cannot be negative");
        iarg += 3;
      } else if (!std::strcmp(kw, "restart")) {
        if (iarg + 2 > narg) perr("fix couplb restart: need prefix");
        copy_str(c.restart_prefix, arg[iarg + 1]);
        c.do_restart = 1;
        iarg += 2;
      } else if (!std::strcmp(kw, "precision")) {
        if (iarg + 2 > narg) perr("fix couplb precision: need 1 value");
        if (!std::strcmp(arg[iarg + 1], "fp64")) c.precision = COUPLB_FP64;
        else if (!std::strcmp(arg[iarg + 1], "fp32")) c.precision = COUPLB_FP32_SHIFTED;
        else if (!std::strcmp(arg[iarg + 1], "fp16")) c.precision = COUPLB_FP16_SHIFTED;
        else perr("fix couplb precision: use fp64, fp32 or fp16");
        iarg += 2;
      } else if (!std::strcmp(kw, "ibm_method")) {
        if (iarg + 2 > narg) perr("fix couplb ibm_method: need 1 value");
        if (!std::strcmp(arg[iarg + 1], "single")) c.ibm_method = COUPLB_IBM_SINGLE;
        else if (!std::strcmp(arg[iarg + 1], "iterative")) c.ibm_method = COUPLB_IBM_ITERATIVE;
        else if (!std::strcmp(arg[iarg + 1], "learned")) c.ibm_method = COUPLB_IBM_LEARNED;
        else perr("fix couplb ibm_method: use single, iterative or learned");
        iarg += 2;
      } else if (!std::strcmp(kw, "ibm_passes")) {
        if (iarg + 2 > narg) perr("fix couplb ibm_passes: need 1 value");
        c.ibm_passes = to_int(arg[iarg + 1]);
        if (c.ibm_passes < 1 || c.ibm_passes > 64) perr("fix couplb: ibm_passes must be 1..64");
        iarg += 2;
      } else if (!std::strcmp(kw, "slip_tol")) {
        if (iarg + 2 > narg) perr("fix couplb slip_tol: need 1 value");
        c.slip_tol = to_double(arg[iarg + 1]);
        if (c.slip_tol < 0.0 || !std::isfinite(c.slip_tol)) perr("fix couplb: slip_tol must be >= 0");
        iarg += 2;
      } else if (!std::strcmp(kw, "mlp_model")) {
        if (iarg + 2 > narg) perr("fix couplb mlp_model: need 1 value");
        copy_str(c.mlp_model, arg[iarg + 1]);
        iarg += 2;
      } else if (!std::strcmp(kw, "ibm_window")) {
        if (iarg + 2 > narg) perr("fix couplb ibm_window: need 1 value");
        if (!std::strcmp(arg[iarg + 1], "clip")) c.ibm_window = 0;
        else if (!std::strcmp(arg[iarg + 1], "wrap")) c.ibm_window = 1;
        else perr("fix couplb ibm_window: use clip or wrap");
        iarg += 2;
      }
    }
    c.dimension = dimension;
    if (dimension != 3 && c.Nz != 1) perr("fix couplb: Nz must be 1 for 2D");
  } catch (const ParseError& e) {
    if (err && errlen > 0) {
      std::strncpy(err, e.msg.c_str(), errlen - 1);
      err[errlen - 1] = 0;
    }
    return COUPLB_ERR_PARSE;
  }
  *cfg = c;
  return COUPLB_OK;
}

int couplb_fix_create(const couplb_fix_config* cfg, couplb_fix** out) {
  if (!cfg || !out) return COUPLB_ERR_ARG;
  couplb_fix* F = new couplb_fix();
  F->cfg = *cfg;
  *out = F;
  return COUPLB_OK;
}

int couplb_fix_destroy(couplb_fix* F) {
  if (!F) return COUPLB_OK;
  free_slab_buffers(F);
  if (F->h) couplb_destroy(F->h);
  if (F->mlp) couplb_mlp_destroy(F->mlp);
  delete F;
  return COUPLB_OK;
}

const char* couplb_fix_last_error(const couplb_fix* F) { return F ? F->err.c_str() : ""; }

int couplb_fix_set_gravity_callback(couplb_fix* F, couplb_gravity_fn fn, void* ctx) {
  if (!F) return COUPLB_ERR_ARG;
  F->gcb = fn;
  F->gctx = ctx;
  return COUPLB_OK;
}

int couplb_fix_set_log_callback(couplb_fix* F, couplb_log_fn fn, void* ctx) {
  if (!F) return COUPLB_ERR_ARG;
  F->logcb = fn;
  F->logctx = ctx;
  return COUPLB_OK;
}

int couplb_fix_set_gravity_values(couplb_fix* F, const double g[3]) {
  if (!F || !g) return COUPLB_ERR_ARG;
  for (int d = 0; d < 3; d++) F->gvals[d] = g[d];
  return COUPLB_OK;
}

int couplb_fix_set_device(couplb_fix* F, int device) {
  if (!F) return COUPLB_ERR_ARG;
  if (F->h) return F->fail(COUPLB_ERR_STATE, "couplb_fix_set_device must precede couplb_fix_init");
  F->device = device;
  return COUPLB_OK;
}

int couplb_fix_set_comm(couplb_fix* F, const couplb_fix_comm* comm) {
  if (!F || !comm) return COUPLB_ERR_ARG;
  if (F->h) return F->fail(COUPLB_ERR_STATE, "couplb_fix_set_comm must precede couplb_fix_init");
  if (comm->nprocs < 1 || comm->rank < 0 || comm->rank >= comm->nprocs)
    return F->fail(COUPLB_ERR_ARG, "fix couplb: bad communicator (rank %d of %d)", comm->rank, comm->nprocs);
  if (comm->nprocs > 1 && (!comm->sendrecv || !comm->allreduce))
    return F->fail(COUPLB_ERR_ARG, "fix couplb: a communicator of several ranks needs sendrecv and allreduce");
  F->comm = *comm;
  F->rank = comm->rank;
  return COUPLB_OK;
}

couplb_handle* couplb_fix_handle(couplb_fix* F) { return F ? F->h : nullptr; }

int couplb_fix_scales(const couplb_fix* F, double out[6]) {
  if (!F || !out) return COUPLB_ERR_ARG;
  out[0] = F->dx; out[1] = F->dt_LBM; out[2] = F->vel_scale;
  out[3] = F->force_scale; out[4] = F->nu_lb; out[5] = F->tau;
  return COUPLB_OK;
}

int couplb_fix_last_diag(const couplb_fix* F, couplb_diag* out) {
  if (!F || !out) return COUPLB_ERR_ARG;
  *out = F->last_diag;
  return COUPLB_OK;
}

long long couplb_fix_lbm_steps(const couplb_fix* F) { return F ? F->lbm_step_count : 0; }

// FixCoupLB::init (fix_couplb.cpp:256-482) for one rank.
int couplb_fix_init(couplb_fix* F, const couplb_domain* dom) {
  if (!F || !dom) return COUPLB_ERR_ARG;
  const couplb_fix_config& c = F->cfg;
  if (c.md_per_lb < 1) return F->fail(COUPLB_ERR_ARG, "fix couplb: md_per_lb must be >= 1");
  if (c.xi_ibm <= 0.0 || c.xi_ibm > 1.0 || !std::isfinite(c.xi_ibm))
    return F->fail(COUPLB_ERR_ARG, "fix couplb: xi_ibm must satisfy 0 < xi_ibm <= 1");
  F->is3d = (dom->dimension == 3);
  for (int d = 0; d < 3; d++) { F->domain_lo[d] = dom->boxlo[d]; F->domain_hi[d] = dom->boxhi[d]; }
  const double dx_x = (F->domain_hi[0] - F->domain_lo[0]) / c.Nx;
  const double dx_y = (F->domain_hi[1] - F->domain_lo[1]) / c.Ny;
  if (std::fabs(dx_x - dx_y) > 1e-10 * dx_x)
    return F->fail(COUPLB_ERR_ARG,
                   "fix couplb: non-cubic grid cells (Lx/Nx=%.6e != Ly/Ny=%.6e). Adjust Nx, Ny, or domain size.",
                   dx_x, dx_y);
  if (F->is3d) {
    const double dx_z = (F->domain_hi[2] - F->domain_lo[2]) / c.Nz;
    if (std::fabs(dx_x - dx_z) > 1e-10 * dx_x)
      return F->fail(COUPLB_ERR_ARG,
                     "fix couplb: non-cubic grid cells (Lx/Nx=%.6e != Lz/Nz=%.6e). Adjust Nx, Nz, or domain size.",
                     dx_x, dx_z);
  }
  F->dx = dx_x;
  F->inv_dx = 1.0 / F->dx;
  F->dt = dom->dt;
  F->dt_LBM = dom->dt * c.md_per_lb;
  F->vel_scale = F->dx / F->dt_LBM;
  F->nu_lb = c.nu * F->dt_LBM / (F->dx * F->dx);
  F->tau = F->nu_lb / (1.0 / 3.0) + 0.5;
  if (F->tau <= 0.5) return F->fail(COUPLB_ERR_ARG, "fix couplb: tau <= 0.5 (unstable)");
  if (F->tau < 0.505) F->log("WARNING: fix couplb: tau very close to 0.5\n");
  const int dim = F->is3d ? 3 : 2;
  double dp = 1.0;
  for (int d = 0; d < dim + 1; d++) dp *= F->dx;
  F->force_scale = c.rho * dp / (F->dt_LBM * F->dt_LBM);
  if (F->force_scale <= 0.0 || !std::isfinite(F->force_scale))
    return F->fail(COUPLB_ERR_ARG,
                   "fix couplb: force_scale is non-positive or non-finite (check rho, dx, dt_LBM)");
  const double inv_vel = 1.0 / F->vel_scale;
  const double wv_lb[3] = {c.wall_vel[0] * inv_vel, c.wall_vel[1] * inv_vel, c.wall_vel[2] * inv_vel};
  const double cs = std::sqrt(1.0 / 3.0);
  const double uw = std::sqrt(wv_lb[0] * wv_lb[0] + wv_lb[1] * wv_lb[1] + wv_lb[2] * wv_lb[2]);
  if (uw > kMaError * cs) return F->fail(COUPLB_ERR_ARG, "fix couplb: wall Ma > 0.5");
  if (uw > kMaWarn * cs) F->log("CoupLB WARNING: wall Ma=%.3f > 0.3\n", uw / cs);
  if (c.gstyle[0] == COUPLB_G_CONSTANT && c.gstyle[1] == COUPLB_G_CONSTANT &&
      c.gstyle[2] == COUPLB_G_CONSTANT) {
    const double ac = F->dt_LBM * F->dt_LBM / F->dx;
    const double gx = c.gconst[0] * ac, gy = c.gconst[1] * ac, gz = c.gconst[2] * ac;
    const double gm = std::sqrt(gx * gx + gy * gy + gz * gz);
    if (gm > kZeroTol) {
      const int H = (c.wall[2] > 0 && c.wall[3] > 0) ? c.Ny : (c.wall[4] > 0 && c.wall[5] > 0) ? c.Nz : 0;
      if (H > 0) {
        const double ue = gm * H * H / (8.0 * F->nu_lb);
        if (ue / cs > kMaError) return F->fail(COUPLB_ERR_ARG, "fix couplb: estimated Poiseuille Ma > 0.5");
        if (ue / cs > kMaWarn) F->log("CoupLB WARNING: estimated Poiseuille Ma=%.3f\n", ue / cs);
      }
    }
  }
  if (c.output_every > 0) F->next_output = dom->ntimestep + c.output_every;
  F->next_check = (c.check_every > 0) ? dom->ntimestep + c.check_every : -1;
  F->next_vtk = (c.vtk_every > 0) ? dom->ntimestep + c.vtk_every : -1;
  F->next_checkpoint = (c.checkpoint_every > 0) ? dom->ntimestep + c.checkpoint_every : -1;
  F->lbm_step_count = 0;
  F->md_sub_count = 0;

  // setup_grid (fix_couplb.cpp:484-520)
  const double eps = 1e-12;
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = (int)std::floor((dom->sublo[d] - F->domain_lo[d]) / F->dx + eps);
    hi[d] = (int)std::floor((dom->subhi[d] - F->domain_lo[d]) / F->dx + eps);
    F->nl[d] = hi[d] - lo[d];
    F->off[d] = lo[d];
  }
  if (!F->is3d) { F->nl[2] = 1; F->off[2] = 0; }
  if (F->nl[0] <= 0 || F->nl[1] <= 0 || (F->is3d && F->nl[2] <= 0))
    return F->fail(COUPLB_ERR_ARG, "fix couplb: local grid empty");
  // Without a communicator the fix runs one lattice: the kernels wrap every
  // non-wall face of the local grid onto itself (the self-exchange of a
  // one-rank run), so a sub-box that is only part of the box would silently
  // simulate a periodic piece of its own; that is refused.  With one
  // (couplb_fix_set_comm) the sub-boxes may split z: this rank runs its slab
  // and exchanges the halos (fix_couplb.cpp:494-500, couplb_streaming.h:176-245).
  F->decomposed = F->is3d && F->comm.nprocs > 1;
  {
    const int full[3] = {c.Nx, c.Ny, F->is3d ? c.Nz : 1};
    for (int d = 0; d < (F->is3d ? 3 : 2); d++)
      if ((F->off[d] != 0 || F->nl[d] != full[d]) && !(F->decomposed && d == 2))
        return F->fail(COUPLB_ERR_UNSUPPORTED,
                       "fix couplb: the MD sub-box covers nodes %d..%d of %d along %c, but this build "
                       "runs the whole lattice on one rank, or z slabs with a communicator "
                       "(couplb_fix_set_comm; sub-boxes split along z only)",
                       F->off[d], F->off[d] + F->nl[d] - 1, full[d], "xyz"[d]);
  }
  if (F->decomposed) {
    if (F->nl[2] < 2) return F->fail(COUPLB_ERR_UNSUPPORTED, "fix couplb: a z slab needs at least 2 planes");
    if (c.vtk_every > 0) return F->fail(COUPLB_ERR_UNSUPPORTED, "fix couplb: vtk output with several ranks");
    // every correction pass would need its own halo exchange
    if (c.ibm_method != COUPLB_IBM_SINGLE)
      return F->fail(COUPLB_ERR_UNSUPPORTED, "fix couplb: ibm_method %s with several ranks",
                     c.ibm_method == COUPLB_IBM_LEARNED ? "learned" : "iterative");
    const bool periodic = c.wall[4] == 0 && c.wall[5] == 0;
    const bool glo = F->off[2] == 0, ghi = F->off[2] + F->nl[2] == c.Nz;
    // a face is bound to a neighbour unless it is a wall of the box
    F->nbr[0] = !glo || periodic;
    F->nbr[1] = !ghi || periodic;
    // window planes beyond each face: 1 below, 2 above, 1 above the face
    // that wraps the periodic box with the clipped window (where the whole
    // lattice stops at its ghost layer); and those of the neighbours' halos
    // facing this slab
    const bool clip = c.ibm_window == 0;
    F->ih_own[0] = F->nbr[0] ? 1 : 0;
    F->ih_own[1] = F->nbr[1] ? ((ghi && periodic && clip) ? 1 : 2) : 0;
    F->ih_nbr[0] = F->nbr[0] ? ((glo && periodic && clip) ? 1 : 2) : 0;
    F->ih_nbr[1] = F->nbr[1] ? 1 : 0;
  }
  if (F->h) { couplb_destroy(F->h); F->h = nullptr; }
  couplb_lattice_params lp;
  std::memset(&lp, 0, sizeof(lp));
  lp.dim = dim;
  lp.nx = F->nl[0]; lp.ny = F->nl[1]; lp.nz = F->nl[2];
  lp.tau = F->tau;
  lp.rho0 = kRhoLb;
  // setup_boundaries (fix_couplb.cpp:522-539): in 2D only x and y walls; a
  // z face bound to a neighbour slab is an open (periodic-type) face
  for (int f = 0; f < (F->is3d ? 6 : 4); f++) lp.wall[f] = c.wall[f];
  if (F->decomposed)
    for (int s = 0; s < 2; s++)
      if (F->nbr[s]) lp.wall[4 + s] = COUPLB_WALL_PERIODIC;
  for (int d = 0; d < 3; d++) lp.wall_vel[d] = wv_lb[d];
  if (!F->is3d) lp.wall_vel[2] = 0.0;
  lp.body_force = (c.gstyle[0] != COUPLB_G_NONE || c.gstyle[1] != COUPLB_G_NONE ||
                   c.gstyle[2] != COUPLB_G_NONE);
  lp.precision = c.precision;
  lp.device = F->device;
  int rc = couplb_create(&lp, &F->h);
  if (rc) return F->fail(rc, "%s", couplb_last_error(nullptr));
  couplb_ibm_params ip;
  std::memset(&ip, 0, sizeof(ip));
  ip.delta = c.delta;
  ip.md_per_lb = c.md_per_lb;
  ip.xi_ibm = c.xi_ibm;
  ip.dt_lbm = F->dt_LBM;
  ip.dx = F->dx;
  ip.vel_scale = F->vel_scale;
  ip.force_scale = F->force_scale;
  for (int d = 0; d < 3; d++) { ip.domain_lo[d] = F->domain_lo[d]; ip.offset[d] = F->off[d]; }
  if ((rc = couplb_set_ibm_params(F->h, &ip))) return F->engine_fail(rc);
  if ((rc = couplb_set_option(F->h, "ibm_window", c.ibm_window))) return F->engine_fail(rc);
  if (F->decomposed) {
    free_slab_buffers(F);
    const size_t pb = couplb_halo_bytes(F->h);
    for (int s = 0; s < 2; s++) {
      if (!F->nbr[s]) continue;
      if ((rc = slab_alloc(F, &F->pop_send[s], pb)) || (rc = slab_alloc(F, &F->pop_recv[s], pb))) return rc;
      const size_t own = couplb_ibm_halo_bytes(F->h, F->ih_own[s]);
      const size_t nb = couplb_ibm_halo_bytes(F->h, F->ih_nbr[s]);
      if ((rc = slab_alloc(F, &F->vel[s], own)) || (rc = slab_alloc(F, &F->frc[s], own)) ||
          (rc = slab_alloc(F, &F->msend[s], nb)) || (rc = slab_alloc(F, &F->frecv[s], nb)))
        return rc;
      if ((rc = couplb_halo_attach(F->h, s, F->pop_recv[s]))) return F->engine_fail(rc);
      if ((rc = couplb_ibm_halo_attach(F->h, s, F->ih_own[s], F->vel[s], F->frc[s]))) return F->engine_fail(rc);
    }
    F->fold_pending = false;
  }
  if (c.ibm_method != COUPLB_IBM_SINGLE) {
    couplb_ibm_method m;
    std::memset(&m, 0, sizeof(m));
    m.method = c.ibm_method;
    m.passes = c.ibm_passes;
    m.slip_tol = c.slip_tol > 0.0 ? c.slip_tol : 1e300;
    if (c.ibm_method == COUPLB_IBM_LEARNED) {
      if (!c.mlp_model[0]) return F->fail(COUPLB_ERR_ARG, "fix couplb: ibm_method learned requires mlp_model");
      if (F->mlp) { couplb_mlp_destroy(F->mlp); F->mlp = nullptr; }
      if ((rc = couplb_mlp_create(F->device, 0, &F->mlp)))
        return F->fail(rc, "fix couplb: cannot create the correction network");
      if ((rc = couplb_mlp_load(F->mlp, c.mlp_model)))
        return F->fail(rc, "fix couplb: %s", couplb_mlp_last_error(F->mlp));
      m.model = F->mlp;
    }
    if ((rc = couplb_set_ibm_method(F->h, &m))) return F->engine_fail(rc);
  }

  if (c.do_restart) {
    long long ck = 0;
    if ((rc = read_checkpoint(F, &ck))) {
      const std::string why = F->err;
      return F->fail(rc, "fix couplb: failed to read checkpoint (%s)", why.c_str());
    }
    F->log("CoupLB: restarted from checkpoint step %lld\n", ck);
    F->cfg.do_restart = 0;
  }
  if (c.vtk_solid_nattr > 0) {
    if (c.vtk_every <= 0)
      return F->fail(COUPLB_ERR_ARG, "fix couplb vtk_solid requires vtk keyword to set output frequency");
    F->log("CoupLB: vtk_solid with %d attributes\n", c.vtk_solid_nattr);
  }
  if (c.has_vtk_region) {
    // clamp, convert to node indices and validate (fix_couplb.cpp:386-426)
    double rlo[3], rhi[3];
    for (int d = 0; d < 3; d++) {
      rlo[d] = std::max(c.vtk_rlo[d], F->domain_lo[d]);
      rhi[d] = std::min(c.vtk_rhi[d], F->domain_hi[d]);
    }
    for (int d = 0; d < 3; d++) { F->vtk_rlo[d] = rlo[d]; F->vtk_rhi[d] = rhi[d]; }
    int* r = F->vtk_region;
    r[0] = (int)std::floor((rlo[0] - F->domain_lo[0]) / F->dx);
    r[1] = (int)std::ceil((rhi[0] - F->domain_lo[0]) / F->dx);
    r[2] = (int)std::floor((rlo[1] - F->domain_lo[1]) / F->dx);
    r[3] = (int)std::ceil((rhi[1] - F->domain_lo[1]) / F->dx);
    if (F->is3d) {
      r[4] = (int)std::floor((rlo[2] - F->domain_lo[2]) / F->dx);
      r[5] = (int)std::ceil((rhi[2] - F->domain_lo[2]) / F->dx);
    } else { r[4] = 0; r[5] = 1; }
    const int Nn[3] = {c.Nx, c.Ny, c.Nz};
    for (int d = 0; d < (F->is3d ? 3 : 2); d++)
      for (int s = 0; s < 2; s++) r[2 * d + s] = std::max(0, std::min(r[2 * d + s], Nn[d]));
    if (r[1] <= r[0] || r[3] <= r[2] || r[5] <= r[4])
      return F->fail(COUPLB_ERR_ARG,
                     "fix couplb vtk_region: empty or inverted region ([%d,%d]x[%d,%d]x[%d,%d]). Check that xlo<xhi, ylo<yhi%s",
                     r[0], r[1], r[2], r[3], r[4], r[5], F->is3d ? ", zlo<zhi" : "");
  }
  for (int a = 0; a < c.vtk_solid_nattr; a++)
    if (!solid_attr_known(c.vtk_solid_attr[a]))
      return F->fail(COUPLB_ERR_ARG, "fix couplb vtk_solid: unknown attribute '%s'", c.vtk_solid_attr[a]);
  F->vtk_steps.clear();
  F->vtk_last = -1;
  F->log("CoupLB: %dD grid %dx%dx%d tau=%.6f nu=%.6f rho=%.4f\n", dim, c.Nx, c.Ny, c.Nz, F->tau, c.nu, c.rho);
  F->log("CoupLB: nu=%.4e -> nu_lb=%.6f\n", c.nu, F->nu_lb);
  F->log("CoupLB: dx=%.4e dt_LBM=%.4e vel_scale=%.4e force_scale=%.4e\n", F->dx, F->dt_LBM, F->vel_scale,
         F->force_scale);
  F->log("CoupLB: kernel=%s xi_ibm=%.4f\n", c.delta == COUPLB_DELTA_ROMA ? "roma" : "peskin4", c.xi_ibm);
  if (c.ibm_method != COUPLB_IBM_SINGLE)
    F->log("CoupLB: ibm_method=%s passes=%d\n", c.ibm_method == COUPLB_IBM_LEARNED ? "learned" : "iterative",
           c.ibm_passes);
  F->log("CoupLB: precision=%s device memory %.1f MB\n",
         c.precision == COUPLB_FP64 ? "fp64" : (c.precision == COUPLB_FP32_SHIFTED ? "fp32" : "fp16"),
         couplb_device_bytes(F->h) / 1048576.0);
  F->inited = true;
  return COUPLB_OK;
}

// FixCoupLB::setup (fix_couplb.cpp:551-638): spread the first forces without
// advancing the fluid, then the step-0 profile.
int couplb_fix_setup(couplb_fix* F, const couplb_atoms* at, long long ntimestep) {
  if (!F || !F->inited) return F ? F->fail(COUPLB_ERR_STATE, "couplb_fix_init not called") : COUPLB_ERR_ARG;
  F->md_sub_count = 0;
  int rc = slab_exchange_state(F, false);
  if (rc) return rc;
  if ((rc = ibm_sub_coupling(F, at))) return rc;
  F->md_sub_count = 0;
  const couplb_fix_config& c = F->cfg;
  const bool need_macro = (c.output_every > 0 || c.vtk_every > 0);
  if (need_macro && (rc = couplb_macroscopic(F->h))) return F->engine_fail(rc);
  if (c.output_every > 0) {
    if (F->rank == 0) {
      FILE* fp = std::fopen(c.output_file, ntimestep == 0 ? "w" : "a");
      if (fp) {
        if (ntimestep == 0) {
          std::fprintf(fp, "# H=Ny=%d tau=%.6f nu=%.4e nu_lb=%.6f rho=%.4f kernel=%s\n", c.Ny, F->tau, c.nu,
                       F->nu_lb, c.rho, c.delta == COUPLB_DELTA_ROMA ? "roma" : "peskin4");
          std::fprintf(fp, "# CoupLB velocity profile\n# Columns: step j y rho ux uy\n#\n");
        }
        std::fclose(fp);
      }
    }
    if ((rc = write_profile(F, ntimestep))) return rc;
  }
  return COUPLB_OK;
}

// FixCoupLB::post_force + lbm_step + apply_external_force's gravity
// (fix_couplb.cpp:640-651, 671-695).
int couplb_fix_post_force(couplb_fix* F, const couplb_atoms* at, long long ntimestep) {
  (void)ntimestep;
  if (!F || !F->inited) return F ? F->fail(COUPLB_ERR_STATE, "couplb_fix_init not called") : COUPLB_ERR_ARG;
  const couplb_fix_config& c = F->cfg;
  int rc;
  if (F->md_sub_count == 0) {
    // do_lbm_step (with the gravity of update_gravity_variables), then the
    // refresh sub-step, in one engine call
    const bool none = c.gstyle[0] == COUPLB_G_NONE && c.gstyle[1] == COUPLB_G_NONE &&
                      c.gstyle[2] == COUPLB_G_NONE;
    double gl[3] = {0.0, 0.0, 0.0};
    if (!none) {
      double gv[3];
      for (int d = 0; d < 3; d++) {
        if (c.gstyle[d] == COUPLB_G_EQUAL) {
          if (F->gcb) {
            if (F->gcb(F->gctx, d, &gv[d]) != 0)
              return F->fail(COUPLB_ERR_ARG, "Variable %s for gravity in fix couplb could not be evaluated",
                             c.gvar[d]);
          } else {
            gv[d] = F->gvals[d];
          }
        } else {
          gv[d] = c.gconst[d];
        }
      }
      const double ac = F->dt_LBM * F->dt_LBM / F->dx;
      for (int d = 0; d < 3; d++) gl[d] = gv[d] * ac;
    }
    if (F->decomposed) {
      // fold last cycle's halo forces, the LB step, the halos of the new
      // state, then the refresh sub-step
      if ((rc = slab_fold(F))) return rc;
      if ((rc = couplb_lbm_step(F->h, none ? nullptr : gl))) return F->engine_fail(rc);
      if ((rc = slab_exchange_state(F, true))) return rc;
      rc = ibm_sub_coupling(F, at);
    } else {
      rc = ibm_sub_coupling(F, at, true, none ? nullptr : gl);
    }
    if (rc) return rc;
    F->lbm_step_count++;
  } else {
    rc = ibm_sub_coupling(F, at);
    if (rc) return rc;
  }
  F->md_sub_count = (F->md_sub_count + 1) % c.md_per_lb;
  return COUPLB_OK;
}

// FixCoupLB::end_of_step (fix_couplb.cpp:846-901) with
// check_stability_precomputed (:818-844).
int couplb_fix_end_of_step(couplb_fix* F, long long step) {
  if (!F || !F->inited) return F ? F->fail(COUPLB_ERR_STATE, "couplb_fix_init not called") : COUPLB_ERR_ARG;
  const couplb_fix_config& c = F->cfg;
  bool chk = false, out = false, vtk = false, ckpt = false;
  if (c.check_every > 0 && step >= F->next_check) { chk = true; F->next_check = step + c.check_every; }
  if (c.output_every > 0 && step >= F->next_output) { out = true; chk = true; F->next_output += c.output_every; }
  if (c.vtk_every > 0 && step >= F->next_vtk) { vtk = true; F->next_vtk = step + c.vtk_every; }
  if (c.checkpoint_every > 0 && step >= F->next_checkpoint) { ckpt = true; F->next_checkpoint = step + c.checkpoint_every; }
  if (!chk && !out && !vtk && !ckpt) return COUPLB_OK;
  int rc;
  if (chk || out || vtk) {
    if ((rc = couplb_macroscopic(F->h))) return F->engine_fail(rc);
  }
  if (chk) {
    couplb_diag d;
    if ((rc = couplb_diagnostics(F->h, &d))) return F->engine_fail(rc);
    if (F->decomposed) {
      // check_stability_precomputed reduces over the ranks (fix_couplb.cpp:818-844)
      double sums[5] = {d.mass, d.mom[0], d.mom[1], d.mom[2], (double)d.clamps};
      double mx = d.umax;
      if ((rc = slab_allreduce(F, sums, 5, 0)) || (rc = slab_allreduce(F, &mx, 1, 1))) return rc;
      d.mass = sums[0]; d.mom[0] = sums[1]; d.mom[1] = sums[2]; d.mom[2] = sums[3];
      d.clamps = (int)sums[4];
      d.umax = mx;
    }
    F->last_diag = d;
    const double ma = d.umax / std::sqrt(1.0 / 3.0);
    if (ma > kMaError) return F->fail(COUPLB_ERR_NUMERIC, "fix couplb: Ma>0.5, simulation invalid");
    if (ma > kMaWarn) F->log("CoupLB WARNING: Ma=%.4f at step %lld\n", ma, step);
    F->log("CoupLB step %lld: Ma=%.4f mass=%.8e mom=(%.4e,%.4e,%.4e)\n", step, ma, d.mass, d.mom[0], d.mom[1],
           d.mom[2]);
    if (d.clamps > 0) F->log("CoupLB WARNING: %d nodes had density clamped at step %lld\n", d.clamps, step);
  }
  if (out && (rc = write_profile(F, step))) return rc;
  if (vtk && (rc = write_field_vtk(F, step))) return rc;
  if (ckpt && (rc = write_checkpoint(F, step))) return rc;
  return COUPLB_OK;
}

int couplb_fix_write_solid(couplb_fix* F, const couplb_atoms* at, long long step) {
  if (!F || !at) return COUPLB_ERR_ARG;
  if (F->cfg.vtk_solid_nattr <= 0 || F->vtk_last != step) return COUPLB_OK;
  return write_solid_vtk(F, at, step);
}

}  // extern "C"
