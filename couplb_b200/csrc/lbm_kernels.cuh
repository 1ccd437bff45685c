// lbm_kernels.cuh -- LBM kernels of one subdomain.
//
// Device layout (interior nodes only, no ghost layer):
//   node n = i + nx*(j + ny*k), 0 <= i < nx, 0 <= j < ny, 0 <= k < nz
//   population q of node n at f[q*qs + n], qs = N rounded up to 64 elements
//   (every q plane starts 256-byte aligned).
// Ghost planes of the reference (couplb_lattice.h:82-129) are not stored:
// a neighbour index that leaves the box selects the wall rule of that face,
// or wraps around on a periodic face -- the self-exchange of a one-rank
// decomposition (couplb_streaming.h:176-194) done as index arithmetic.
//
// Time stepping stores the POST-COLLISION populations P between launches and
// fuses "stream of step k-1" with "collide of step k" in one pass (pull):
//   S_{k-1}(n, q) = rule(P_{k-1} at n - e_q)      streaming, couplb_streaming.h:82-134
//   rho, u        = moments of S_{k-1} + Guo       couplb_lattice.h:155-202
//   P_k(n, q)     = BGK + Guo collision            couplb_collision.h:18-62
// A state that is post-stream (initial condition, restart, after a
// materialise pass) is read in place instead of pulled (Mode::Own).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.cuh"
#include "storage.cuh"

namespace couplb {

enum RhoMode : int { kRhoNone = 0, kRhoField = 1, kRhoCurrent = 2 };
enum StatusSlot : int { kStClamps = 0, kStNonfinite = 1, kStMacroClamps = 2 };

// Geometry + boundary description shared by all lattice kernels.
struct Geom {
  int nx, ny, nz;
  long long qs;      // q-plane stride in elements
  int face[6];       // wall type per face: xlo xhi ylo yhi zlo zhi
  double uw[3];      // type-2 wall velocity
  double rho0;       // shift / reference density
};

template <class S>
struct LBArgs {
  Geom g;
  const typename S::T* __restrict__ fin;
  typename S::T* __restrict__ fout;
  const typename S::A* __restrict__ Fx;   // IBM force field, or null
  const typename S::A* __restrict__ Fy;
  const typename S::A* __restrict__ Fz;
  typename S::A* __restrict__ rho_field;  // stale density (see RhoMode)
  int rho_mode;
  int write_rho;
  double grav[3];
  double omega;
  int* status;
};

// ---------------------------------------------------------------------------
// Density clamp of couplb_lattice.h:178-186: rho <= RHO_MIN or non-finite
// becomes RHO_MIN and is counted.
template <class Cf>
__device__ __forceinline__ Cf clamp_rho(Cf r, int* status, int slot) {
  if (r <= Cf(RHO_MIN)) {
    r = Cf(RHO_MIN);
    atomicAdd(status + slot, 1);
  }
  if (!isfinite(r)) {
    r = Cf(RHO_MIN);
    atomicAdd(status + slot, 1);
    atomicAdd(status + kStNonfinite, 1);
  }
  return r;
}

// Density of the receiving node that the moving-wall rule uses: in the
// reference it is rho[n] of the last compute_macroscopic(true), i.e. the
// density of the state this node collided from, which equals the sum of its
// post-collision populations (BGK + Guo conserve mass).
template <class L, class S>
__device__ __forceinline__ typename S::C moving_wall_rho(const typename S::T* fin, long long qs,
                                                         long long n, double rho0) {
  using C = typename S::C;
  C s = C(0);
#pragma unroll
  for (int q = 0; q < L::Q; q++) s += S::ld(fin + q * qs + n);
  C r = S::kShift ? C(rho0) + s : s;
  if (r <= C(RHO_MIN) || !isfinite(r)) r = C(RHO_MIN);
  const C fl = C(RHO_CLAMP_FRAC * rho0 < RHO_MIN ? RHO_MIN : RHO_CLAMP_FRAC * rho0);
  return (r < fl) ? fl : r;
}

// Pull of all Q populations of node (i,j,k) with the reference's boundary
// rules (couplb_streaming.h:99-129).  The source x - e_q of an interior node
// is either interior, or on one or more ghost planes; on a ghost node the wall
// set last (x, then y, then z: couplb_boundary.h, fix_couplb.cpp:529-531)
// decides the rule, and a ghost node without wall is a periodic image.
template <class L, class S>
__device__ __forceinline__ void pull_general(const Geom& g, const typename S::T* __restrict__ fin,
                                             int i, int j, int k, long long n,
                                             typename S::C (&f)[L::Q]) {
  using C = typename S::C;
  const long long sxy = (long long)g.nx * g.ny;
  bool near_moving = (g.face[0] == 2 && i == 0) || (g.face[1] == 2 && i == g.nx - 1) ||
                     (g.face[2] == 2 && j == 0) || (g.face[3] == 2 && j == g.ny - 1);
  if (L::D == 3) near_moving |= (g.face[4] == 2 && k == 0) || (g.face[5] == 2 && k == g.nz - 1);
  C rw = C(0);
  if (near_moving) rw = moving_wall_rho<L, S>(fin, g.qs, n, g.rho0);
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
    int si = i - ex, sj = j - ey, sk = k - ez;
    const bool ox = si < 0 || si >= g.nx;
    const bool oy = sj < 0 || sj >= g.ny;
    const bool oz = (L::D == 3) && (sk < 0 || sk >= g.nz);
    if (!(ox || oy || oz)) {
      f[q] = S::ld(fin + q * g.qs + (n - ex - (long long)ey * g.nx - (long long)ez * sxy));
      continue;
    }
    int t = 0, wd = 0;
    if (ox) { const int ft = si < 0 ? g.face[0] : g.face[1]; if (ft) { t = ft; wd = 0; } }
    if (oy) { const int ft = sj < 0 ? g.face[2] : g.face[3]; if (ft) { t = ft; wd = 1; } }
    if (oz) { const int ft = sk < 0 ? g.face[4] : g.face[5]; if (ft) { t = ft; wd = 2; } }
    if (t == 0) {
      si = si < 0 ? si + g.nx : (si >= g.nx ? si - g.nx : si);
      sj = sj < 0 ? sj + g.ny : (sj >= g.ny ? sj - g.ny : sj);
      if (L::D == 3) sk = sk < 0 ? sk + g.nz : (sk >= g.nz ? sk - g.nz : sk);
      f[q] = S::ld(fin + q * g.qs + (si + (long long)g.nx * sj + sxy * sk));
    } else if (t == 1) {
      f[q] = S::ld(fin + L::opp(q) * g.qs + n);
    } else if (t == 2) {
      const C eu = C(ex * g.uw[0] + ey * g.uw[1] + ez * g.uw[2]);
      f[q] = S::ld(fin + L::opp(q) * g.qs + n) + C(2.0 * L::w(L::opp(q)) * 3.0) * rw * eu;
    } else if (t == 3) {
      const int qr = wd == 0 ? L::refl(0, q) : (wd == 1 ? L::refl(1, q) : L::refl(2, q));
      f[q] = S::ld(fin + qr * g.qs + n);
    } else {
      f[q] = S::ld(fin + q * g.qs + n);
    }
  }
}

// Pull for rows that touch no wall: only x can wrap, handled by selecting the
// wrapped column; y/z offsets are constants of q.
template <class L, class S>
__device__ __forceinline__ void pull_interior(const Geom& g, const typename S::T* __restrict__ fin,
                                              int i, int j, int k, typename S::C (&f)[L::Q]) {
  const int im = (i == 0) ? g.nx - 1 : i - 1;
  const int ip = (i == g.nx - 1) ? 0 : i + 1;
  const long long row = (long long)g.nx * (j + (long long)g.ny * k);
  const long long sxy = (long long)g.nx * g.ny;
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
    const int xs = ex == 1 ? im : (ex == -1 ? ip : i);
    f[q] = S::ld(fin + q * g.qs + (row - (long long)ey * g.nx - (long long)ez * sxy + xs));
  }
}

// True when no population of this node can come from outside the box or
// across a periodic face other than x.
template <class L>
__device__ __forceinline__ bool row_is_interior(const Geom& g, int j, int k) {
  const bool yin = j > 0 && j < g.ny - 1;
  const bool zin = (L::D == 2) || (k > 0 && k < g.nz - 1);
  return yin && zin && g.face[0] == 0 && g.face[1] == 0;
}

template <class L, class S, bool kPull>
__device__ __forceinline__ void load_node(const Geom& g, const typename S::T* __restrict__ fin,
                                          int i, int j, int k, long long n,
                                          typename S::C (&f)[L::Q]) {
  if (!kPull) {
#pragma unroll
    for (int q = 0; q < L::Q; q++) f[q] = S::ld(fin + q * g.qs + n);
  } else if (row_is_interior<L>(g, j, k)) {
    pull_interior<L, S>(g, fin, i, j, k, f);
  } else {
    pull_general<L, S>(g, fin, i, j, k, n, f);
  }
}

// Moments: rho (or its deviation) and sum_q e_q f_q, summed in q order like
// couplb_lattice.h:166-174.
template <class L, class C>
__device__ __forceinline__ void moments(const C (&f)[L::Q], C& r, C& jx, C& jy, C& jz) {
  r = C(0); jx = C(0); jy = C(0); jz = C(0);
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    r += f[q];
    if (L::ex(q) == 1) jx += f[q]; else if (L::ex(q) == -1) jx -= f[q];
    if (L::ey(q) == 1) jy += f[q]; else if (L::ey(q) == -1) jy -= f[q];
    if (L::D == 3) { if (L::ez(q) == 1) jz += f[q]; else if (L::ez(q) == -1) jz -= f[q]; }
  }
}

// ---------------------------------------------------------------------------
// K1: fused stream (step k-1) + external force + moments + BGK/Guo collision
// (step k).  One thread per node, threads along x.
template <class L, class S, bool kPull>
__global__ void __launch_bounds__(256) k_stream_collide(const LBArgs<S> a) {
  using C = typename S::C;
  const Geom& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long n = i + (long long)g.nx * (j + (long long)g.ny * k);

  C f[L::Q];
  load_node<L, S, kPull>(g, a.fin, i, j, k, n, f);

  C r, jx, jy, jz;
  moments<L, C>(f, r, jx, jy, jz);
  // r is rho (plain) or the density deviation (shifted)
  C rho = S::kShift ? C(g.rho0) + r : r;
  const C rho_c = clamp_rho(rho, a.status, kStClamps);
  if (rho_c != rho) { rho = rho_c; r = S::kShift ? rho - C(g.rho0) : rho; }

  // apply_external_force (fix_couplb.cpp:693-707): F += g * rho[n], rho[n]
  // being the density the last moment pass stored.
  C Fx = C(0), Fy = C(0), Fz = C(0);
  if (a.Fx) { Fx = C(a.Fx[n]); Fy = C(a.Fy[n]); Fz = C(a.Fz[n]); }
  if (a.rho_mode != kRhoNone) {
    C rp;
    if (a.rho_mode == kRhoField) rp = S::kShift ? C(g.rho0) + C(a.rho_field[n]) : C(a.rho_field[n]);
    else rp = rho;
    Fx += C(a.grav[0]) * rp;
    Fy += C(a.grav[1]) * rp;
    Fz += C(a.grav[2]) * rp;
  }
  if (a.write_rho) a.rho_field[n] = typename S::A(S::kShift ? r : rho);

  // compute_macroscopic(true): u = (sum e f + F/2) / rho
  const C inv_r = C(1) / rho;
  const C ux = (jx + C(0.5) * Fx) * inv_r;
  const C uy = (jy + C(0.5) * Fy) * inv_r;
  const C uz = (jz + C(0.5) * Fz) * inv_r;

  // BGK + Guo (couplb_collision.h:35-57), with 1/cs2 = 3, 1/cs4 = 9
  const C om = C(a.omega);
  const C half_om = C(1) - C(0.5) * om;
  const C uu = ux * ux + uy * uy + uz * uz;
  const C uf = ux * Fx + uy * Fy + uz * Fz;
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const C cx = C(L::ex(q)), cy = C(L::ey(q)), cz = C(L::ez(q));
    const C w = C(L::w(q));
    const C eu = cx * ux + cy * uy + cz * uz;
    const C ef = cx * Fx + cy * Fy + cz * Fz;
    const C poly = C(3) * eu + C(4.5) * eu * eu - C(1.5) * uu;
    const C fe = S::kShift ? w * (r + rho * poly) : w * rho * (C(1) + poly);
    const C si = w * half_om * (C(3) * (ef - uf) + C(9) * eu * ef);
    S::st(a.fout + q * g.qs + n, f[q] + (-om * (f[q] - fe) + si));
  }
}

// ---------------------------------------------------------------------------
// K2: moments of the post-stream state without the Guo term
// (compute_macroscopic(false), couplb_lattice.h:155-202).  Writes rho (or its
// deviation when shifted) and u.
template <class S>
struct MacroArgs {
  Geom g;
  const typename S::T* __restrict__ fin;
  typename S::A* __restrict__ rho;
  typename S::A* __restrict__ ux;
  typename S::A* __restrict__ uy;
  typename S::A* __restrict__ uz;
  int* status;
};

template <class L, class S, bool kPull>
__global__ void __launch_bounds__(256) k_macro(const MacroArgs<S> a) {
  using C = typename S::C;
  const Geom& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long n = i + (long long)g.nx * (j + (long long)g.ny * k);
  C f[L::Q];
  load_node<L, S, kPull>(g, a.fin, i, j, k, n, f);
  C r, jx, jy, jz;
  moments<L, C>(f, r, jx, jy, jz);
  C rho = S::kShift ? C(g.rho0) + r : r;
  const C rho_c = clamp_rho(rho, a.status, kStMacroClamps);
  if (rho_c != rho) { rho = rho_c; r = S::kShift ? rho - C(g.rho0) : rho; }
  const C inv_r = C(1) / rho;
  a.rho[n] = typename S::A(S::kShift ? r : rho);
  a.ux[n] = typename S::A(jx * inv_r);
  a.uy[n] = typename S::A(jy * inv_r);
  a.uz[n] = typename S::A(jz * inv_r);
}

// Materialise: pull the post-collision state into the post-stream state
// (streaming alone), so it can be exported or restarted from.
template <class L, class S>
__global__ void __launch_bounds__(256) k_materialize(Geom g, const typename S::T* __restrict__ fin,
                                                     typename S::T* __restrict__ fout) {
  using C = typename S::C;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long n = i + (long long)g.nx * (j + (long long)g.ny * k);
  C f[L::Q];
  load_node<L, S, true>(g, fin, i, j, k, n, f);
#pragma unroll
  for (int q = 0; q < L::Q; q++) S::st(fout + q * g.qs + n, f[q]);
}

// Equilibrium initial state (Grid::init_equilibrium, couplb_lattice.h:137-154).
template <class L, class S>
__global__ void k_init_eq(Geom g, typename S::T* __restrict__ f, double rho, double ux, double uy,
                          double uz, typename S::A* __restrict__ rho_field) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double cs2 = 1.0 / 3.0, cs4 = cs2 * cs2;
  const double uu = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const double eu = L::ex(q) * ux + L::ey(q) * uy + L::ez(q) * uz;
    const double fe = L::w(q) * rho * (1.0 + eu / cs2 + 0.5 * eu * eu / cs4 - 0.5 * uu / cs2);
    S::st(f + q * g.qs + n, typename S::C(S::kShift ? fe - L::w(q) * g.rho0 : fe));
  }
  if (rho_field) rho_field[n] = typename S::A(S::kShift ? rho - g.rho0 : rho);
}

// Import of reference-layout populations (double, ghost-inclusive G nodes):
// the interior values are stored (shifted / scaled as the format needs).
template <class L, class S>
__global__ void k_import_f(Geom g, const double* __restrict__ src, long long G,
                           typename S::T* __restrict__ f) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int i = n % g.nx;
  const int j = (n / g.nx) % g.ny;
  const int k = n / ((long long)g.nx * g.ny);
  const int gx = g.nx + 2, gy = g.ny + 2;
  const long long gn = (i + 1) + (long long)gx * ((j + 1) + (long long)gy * (L::D == 3 ? k + 1 : 0));
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const double v = src[q * G + gn];
    S::st(f + q * g.qs + n, typename S::C(S::kShift ? v - L::w(q) * g.rho0 : v));
  }
}

// Classification of a ghost-inclusive node (reference layout) for exports:
// returns -1 for a periodic image or interior node (with the interior index
// in *src), else the wall type (1..4).
__device__ __forceinline__ int classify_ghost(const Geom& g, int D, int ig, int jg, int kg,
                                              long long* src) {
  const int gx = g.nx + 2, gy = g.ny + 2, gz = (D == 3) ? g.nz + 2 : 1;
  int t = 0;
  const bool ox = ig == 0 || ig == gx - 1;
  const bool oy = jg == 0 || jg == gy - 1;
  const bool oz = (D == 3) && (kg == 0 || kg == gz - 1);
  if (ox) { const int ft = ig == 0 ? g.face[0] : g.face[1]; if (ft) t = ft; }
  if (oy) { const int ft = jg == 0 ? g.face[2] : g.face[3]; if (ft) t = ft; }
  if (oz) { const int ft = kg == 0 ? g.face[4] : g.face[5]; if (ft) t = ft; }
  if (t) return t;
  int i = ig - 1, j = jg - 1, k = (D == 3) ? kg - 1 : 0;
  i = i < 0 ? g.nx - 1 : (i >= g.nx ? 0 : i);
  j = j < 0 ? g.ny - 1 : (j >= g.ny ? 0 : j);
  if (D == 3) k = k < 0 ? g.nz - 1 : (k >= g.nz ? 0 : k);
  *src = i + (long long)g.nx * (j + (long long)g.ny * k);
  return -1;
}

// Export of the post-stream state to the reference layout.
template <class L, class S>
__global__ void k_export_f(Geom g, const typename S::T* __restrict__ f, long long G,
                           double* __restrict__ dst) {
  const long long gn = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (gn >= G) return;
  const int gx = g.nx + 2, gy = g.ny + 2;
  const int ig = gn % gx, jg = (gn / gx) % gy, kg = gn / ((long long)gx * gy);
  long long src = 0;
  const int t = classify_ghost(g, L::D, ig, jg, kg, &src);
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    double v;
    if (t > 0) v = L::w(q) * g.rho0;
    else {
      v = double(S::ld(f + q * g.qs + src));
      if (S::kShift) v += L::w(q) * g.rho0;
    }
    dst[q * G + gn] = v;
  }
}

// Export of the moments to the reference layout; wall ghosts get the values of
// enforce_wall_ghost_fields (fix_couplb.cpp:800-809) with rho_lb = 1.
template <class S>
__global__ void k_export_macro(Geom g, int D, const typename S::A* __restrict__ rho,
                               const typename S::A* __restrict__ ux,
                               const typename S::A* __restrict__ uy,
                               const typename S::A* __restrict__ uz, long long G,
                               double* __restrict__ drho, double* __restrict__ dux,
                               double* __restrict__ duy, double* __restrict__ duz) {
  const long long gn = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (gn >= G) return;
  const int gx = g.nx + 2, gy = g.ny + 2;
  const int ig = gn % gx, jg = (gn / gx) % gy, kg = gn / ((long long)gx * gy);
  long long src = 0;
  const int t = classify_ghost(g, D, ig, jg, kg, &src);
  double r, a, b, c;
  if (t > 0) {
    r = 1.0;
    a = b = c = 0.0;
    if (t == 2) { a = g.uw[0]; b = g.uw[1]; c = (D == 3) ? g.uw[2] : 0.0; }
  } else {
    r = double(rho[src]);
    if (S::kShift) r += g.rho0;
    a = double(ux[src]); b = double(uy[src]); c = double(uz[src]);
  }
  if (drho) drho[gn] = r;
  if (dux) dux[gn] = a;
  if (duy) duy[gn] = b;
  if (duz) duz[gn] = c;
}

// Force field export (interior values, ghosts zero) and import.
template <class S>
__global__ void k_export_force(Geom g, int D, const typename S::A* __restrict__ Fx,
                               const typename S::A* __restrict__ Fy,
                               const typename S::A* __restrict__ Fz, long long G,
                               double* __restrict__ dx, double* __restrict__ dy,
                               double* __restrict__ dz) {
  const long long gn = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (gn >= G) return;
  const int gx = g.nx + 2, gy = g.ny + 2;
  const int ig = gn % gx, jg = (gn / gx) % gy, kg = gn / ((long long)gx * gy);
  const bool inside = ig >= 1 && ig <= g.nx && jg >= 1 && jg <= g.ny &&
                      (D == 2 || (kg >= 1 && kg <= g.nz));
  double a = 0, b = 0, c = 0;
  if (inside) {
    const long long n = (ig - 1) + (long long)g.nx * ((jg - 1) + (long long)g.ny * (D == 3 ? kg - 1 : 0));
    a = double(Fx[n]); b = double(Fy[n]); c = double(Fz[n]);
  }
  dx[gn] = a; dy[gn] = b; dz[gn] = c;
}

template <class S>
__global__ void k_import_force(Geom g, int D, const double* __restrict__ sx,
                               const double* __restrict__ sy, const double* __restrict__ sz,
                               typename S::A* __restrict__ Fx, typename S::A* __restrict__ Fy,
                               typename S::A* __restrict__ Fz) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int i = n % g.nx, j = (n / g.nx) % g.ny, k = n / ((long long)g.nx * g.ny);
  const int gx = g.nx + 2, gy = g.ny + 2;
  const long long gn = (i + 1) + (long long)gx * ((j + 1) + (long long)gy * (D == 3 ? k + 1 : 0));
  Fx[n] = typename S::A(sx[gn]);
  Fy[n] = typename S::A(sy[gn]);
  Fz[n] = typename S::A(sz[gn]);
}

// ---------------------------------------------------------------------------
// a20 reductions over the moment fields in FP64 (couplb_lattice.h:203-242):
// per block: max u^2, sum rho, sum rho*u.  Block partials go to `part`
// (5 doubles per block) and k_reduce_final sums them in a fixed order, so the
// result does not depend on scheduling.
template <class S>
__global__ void __launch_bounds__(256) k_diag_partial(long long N, double rho0,
                                                      const typename S::A* __restrict__ rho,
                                                      const typename S::A* __restrict__ ux,
                                                      const typename S::A* __restrict__ uy,
                                                      const typename S::A* __restrict__ uz,
                                                      double* __restrict__ part) {
  double m2 = 0, sm = 0, px = 0, py = 0, pz = 0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    double r = double(rho[n]);
    if (S::kShift) r += rho0;
    const double a = double(ux[n]), b = double(uy[n]), c = double(uz[n]);
    const double u2 = a * a + b * b + c * c;
    m2 = u2 > m2 ? u2 : m2;
    sm += r;
    px += r * a; py += r * b; pz += r * c;
  }
  __shared__ double sh[5][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
    px += __shfl_xor_sync(0xffffffffu, px, o);
    py += __shfl_xor_sync(0xffffffffu, py, o);
    pz += __shfl_xor_sync(0xffffffffu, pz, o);
  }
  if (lane == 0) { sh[0][wid] = m2; sh[1][wid] = sm; sh[2][wid] = px; sh[3][wid] = py; sh[4][wid] = pz; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    double o[5] = {0, 0, 0, 0, 0};
    for (int w = 0; w < nw; w++) {
      o[0] = fmax(o[0], sh[0][w]);
      for (int c = 1; c < 5; c++) o[c] += sh[c][w];
    }
    for (int c = 0; c < 5; c++) part[blockIdx.x * 5 + c] = o[c];
  }
}

__global__ void k_reduce_final(int nblocks, const double* __restrict__ part,
                               double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double o[5] = {0, 0, 0, 0, 0};
  for (int b = 0; b < nblocks; b++) {
    o[0] = fmax(o[0], part[b * 5]);
    for (int c = 1; c < 5; c++) o[c] += part[b * 5 + c];
  }
  out[0] = sqrt(o[0]);
  for (int c = 1; c < 5; c++) out[c] = o[c];
}

// y-profile sums of FixCoupLB::write_profile (fix_couplb.cpp:906-910): for
// every j, the sums over i and k of ux, uy and rho.  One block per j, FP64,
// fixed reduction order.
template <class S>
__global__ void __launch_bounds__(256) k_y_profile(Geom g, const typename S::A* __restrict__ rho,
                                                   const typename S::A* __restrict__ ux,
                                                   const typename S::A* __restrict__ uy,
                                                   double* __restrict__ out) {
  const int j = blockIdx.x;
  const long long cnt = (long long)g.nx * g.nz;
  double a = 0, b = 0, c = 0;
  for (long long t = threadIdx.x; t < cnt; t += blockDim.x) {
    const int i = t % g.nx;
    const long long k = t / g.nx;
    const long long n = i + (long long)g.nx * (j + (long long)g.ny * k);
    a += double(ux[n]);
    b += double(uy[n]);
    double r = double(rho[n]);
    if (S::kShift) r += g.rho0;
    c += r;
  }
  __shared__ double sh[3][256];
  sh[0][threadIdx.x] = a; sh[1][threadIdx.x] = b; sh[2][threadIdx.x] = c;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[j] = sh[0][0];
    out[g.ny + j] = sh[1][0];
    out[2 * g.ny + j] = sh[2][0];
  }
}

}  // namespace couplb
