// lbm_kernels.cuh -- LBM kernels of one subdomain.
//
// Device layout (interior nodes only, no ghost layer):
//   node n = i + nx*(j + ny*k), 0 <= i < nx, 0 <= j < ny, 0 <= k < nz
//   population q of node n at f[pidx(q, n)] = f[q*qs + n], qs = N rounded up
//   to 64 elements (every q plane starts 256-byte aligned; storage.cuh).
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
// variants of the fused LB kernel (the "kernel" option of a handle)
// (value 1 was a shared-memory staged variant, since removed)
enum KernelKind : int { kKernelAuto = -1, kKernelPlain = 0, kKernelPacked = 2 };

// Geometry + boundary description shared by all lattice kernels.
struct Geom {
  int nx, ny, nz;
  long long qs;      // q-plane stride in elements
  int face[6];       // wall type per face: xlo xhi ylo yhi zlo zhi
  double uw[3];      // type-2 wall velocity
  double rho0;       // shift / reference density
  // z faces that border another subdomain (slab decomposition along z): the
  // populations that cross the face, taken from the neighbour's boundary
  // plane after its last LB step (couplb_halo_attach); null = the face wraps
  // onto this subdomain's other face (or is a wall)
  const void* halo[2];
};

// Slot of population q in a z-face halo: the five populations that cross a
// z face in one direction (ez = +1: 5, 11, 14, 15, 18; ez = -1: 6, 12, 13, 16,
// 17 in the D3Q19 order), each one plane of nx * ny values.
template <class L>
__host__ __device__ constexpr int halo_slot(int q) {
  int s = 0;
  for (int p = 0; p < q; p++)
    if (L::ez(p) == L::ez(q)) s++;
  return s;
}
constexpr int kHaloQ = 5;

// Element index of population q of interior node n (storage.cuh, kTile).
template <class L, class S, class I>
__device__ __forceinline__ I pidx(int q, I n, I qs) {
  if constexpr (S::kTile == 0) {
    return (I)q * qs + n;
  } else {
    return ((n / (I)S::kTile) * (I)L::Q + (I)q) * (I)S::kTile + n % (I)S::kTile;
  }
}

template <class S>
struct LBArgs {
  Geom g;
  const typename S::T* __restrict__ fin;
  typename S::T* __restrict__ fout;
  // IBM force field {fx, fy, fz, 0} per node (F[4n + c]), or null; the step
  // reads it and leaves it zero (clear_forces, couplb_lattice.h:243-247) by
  // zeroing the nonzero entries
  typename S::A* __restrict__ F;
  const unsigned char* __restrict__ seg_force;  // per 8 nodes (n >> 3): force present, or null = all
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

// Density the moving-wall rule uses for the receiving node n
// (couplb_streaming.h:86,112-118): rho[n] of the last compute_macroscopic(true),
// i.e. the clamped density the previous fused launch computed at n, which it
// stored in the density field; floored at RHO_CLAMP_FRAC * rho0.
template <class S>
__device__ __forceinline__ typename S::C moving_wall_rho(const typename S::A* rho_field, size_t n,
                                                         double rho0) {
  using C = typename S::C;
  const C r = S::kShift ? C(rho0) + C(rho_field[n]) : C(rho_field[n]);
  const C fl = C(RHO_CLAMP_FRAC * rho0 < RHO_MIN ? RHO_MIN : RHO_CLAMP_FRAC * rho0);
  return (r < fl) ? fl : r;
}

template <class L>
__device__ __forceinline__ bool near_moving_wall(const Geom& g, int i, int j, int k) {
  bool m = (g.face[0] == 2 && i == 0) || (g.face[1] == 2 && i == g.nx - 1) ||
           (g.face[2] == 2 && j == 0) || (g.face[3] == 2 && j == g.ny - 1);
  if (L::D == 3) m = m || (g.face[4] == 2 && k == 0) || (g.face[5] == 2 && k == g.nz - 1);
  return m;
}

// Pull of all Q populations of node (i,j,k) with the reference's boundary
// rules (couplb_streaming.h:99-129).  The source x - e_q of an interior node
// is either interior, or on one or more ghost planes; on a ghost node the wall
// set last (x, then y, then z: couplb_boundary.h, fix_couplb.cpp:529-531)
// decides the rule, and a ghost node without wall is a periodic image.
template <class L, class S, class I>
__device__ __forceinline__ void pull_general(const Geom& g, const typename S::T* __restrict__ fin,
                                             const typename S::A* __restrict__ rho_field, int i,
                                             int j, int k, I n, typename S::C (&f)[L::Q]) {
  using C = typename S::C;
  const I qs = (I)g.qs;
  const I sx = (I)g.nx, sxy = (I)g.nx * (I)g.ny;
  C rw = C(0);
  if (near_moving_wall<L>(g, i, j, k)) rw = moving_wall_rho<S>(rho_field, n, g.rho0);
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
    int si = i - ex, sj = j - ey, sk = k - ez;
    const bool ox = si < 0 || si >= g.nx;
    const bool oy = sj < 0 || sj >= g.ny;
    const bool oz = (L::D == 3) && (sk < 0 || sk >= g.nz);
    if (!(ox || oy || oz)) {
      f[q] = S::ld(fin + pidx<L, S, I>(q, (I)(si + (I)sj * sx + (I)sk * sxy), qs));
      continue;
    }
    int t = 0, wd = 0;
    if (ox) { const int ft = si < 0 ? g.face[0] : g.face[1]; if (ft) { t = ft; wd = 0; } }
    if (oy) { const int ft = sj < 0 ? g.face[2] : g.face[3]; if (ft) { t = ft; wd = 1; } }
    if (oz) { const int ft = sk < 0 ? g.face[4] : g.face[5]; if (ft) { t = ft; wd = 2; } }
    if (t == 0) {
      si = si < 0 ? si + g.nx : (si >= g.nx ? si - g.nx : si);
      sj = sj < 0 ? sj + g.ny : (sj >= g.ny ? sj - g.ny : sj);
      const void* hz = oz ? g.halo[sk < 0 ? 0 : 1] : nullptr;
      if (L::D == 3 && hz) {
        // the neighbour subdomain's boundary plane (its exchange face)
        const typename S::T* hp = static_cast<const typename S::T*>(hz);
        f[q] = S::ld(hp + (size_t)halo_slot<L>(q) * sxy + (I)si + (I)sj * sx);
        continue;
      }
      if (L::D == 3) sk = sk < 0 ? sk + g.nz : (sk >= g.nz ? sk - g.nz : sk);
      f[q] = S::ld(fin + pidx<L, S, I>(q, (I)si + (I)sj * sx + (I)sk * sxy, qs));
    } else if (t == 1) {
      f[q] = S::ld(fin + pidx<L, S, I>(L::opp(q), n, qs));
    } else if (t == 2) {
      const C eu = C(ex * g.uw[0] + ey * g.uw[1] + ez * g.uw[2]);
      f[q] = S::ld(fin + pidx<L, S, I>(L::opp(q), n, qs)) + C(2.0 * L::w(L::opp(q)) * 3.0) * rw * eu;
    } else if (t == 3) {
      const int qr = wd == 0 ? L::refl(0, q) : (wd == 1 ? L::refl(1, q) : L::refl(2, q));
      f[q] = S::ld(fin + pidx<L, S, I>(qr, n, qs));
    } else {
      f[q] = S::ld(fin + pidx<L, S, I>(q, n, qs));
    }
  }
}

// Pull for rows that touch no wall: only x can wrap, handled by selecting the
// wrapped column; y/z offsets are constants of q.
template <class L, class S, class I>
__device__ __forceinline__ void pull_interior(const Geom& g, const typename S::T* __restrict__ fin,
                                              int i, int j, int k, typename S::C (&f)[L::Q]) {
  const I qs = (I)g.qs;
  const I sx = (I)g.nx, sxy = (I)g.nx * (I)g.ny;
  const I row = (I)j * sx + (I)k * sxy;
  const I im = (i == 0) ? g.nx - 1 : i - 1;
  const I ip = (i == g.nx - 1) ? 0 : i + 1;
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
    const I xs = ex == 1 ? im : (ex == -1 ? ip : (I)i);
    const I ro = row - (I)(ey * g.nx) - (I)ez * sxy;   // unsigned wrap-around is exact
    f[q] = S::ld(fin + pidx<L, S, I>(q, ro + xs, qs));
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

template <class L, class S, class I, bool kPull>
__device__ __forceinline__ void load_node(const Geom& g, const typename S::T* __restrict__ fin,
                                          const typename S::A* __restrict__ rho_field, int i,
                                          int j, int k, I n, typename S::C (&f)[L::Q]) {
  if (!kPull) {
    const I qs = (I)g.qs;
#pragma unroll
    for (int q = 0; q < L::Q; q++) f[q] = S::ld(fin + pidx<L, S, I>(q, n, qs));
  } else if (row_is_interior<L>(g, j, k)) {
    pull_interior<L, S, I>(g, fin, i, j, k, f);
  } else {
    pull_general<L, S, I>(g, fin, rho_field, i, j, k, n, f);
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

// BGK + Guo collision of one node (couplb_collision.h:35-57) written over
// the pairs (q, opp(q)) = (2p+1, 2p+2), e_{2p+2} = -e_{2p+1}: the even part
// of the equilibrium and source is shared by the pair, the odd part flips sign.
// 1/cs2 = 3, 1/cs4 = 9.  Produces the post-collision increment d_q:
//   d_q = -omega (f_q - feq_q) + S_q.
// r is rho (plain) or its deviation (shifted), rho the full density.
template <class L, class C>
__device__ __forceinline__ void collision_increment(const C (&f)[L::Q], C r, C rho, C ux, C uy,
                                                    C uz, C Fx, C Fy, C Fz, C om, bool shifted,
                                                    C (&d)[L::Q]) {
  const C hom = C(1) - C(0.5) * om;
  const C uu15 = C(1.5) * (ux * ux + uy * uy + uz * uz);
  const C uf3 = C(3) * (ux * Fx + uy * Fy + uz * Fz);
  {
    const C w = C(L::w(0));
    const C fe = shifted ? w * (r - rho * uu15) : w * rho * (C(1) - uu15);
    d[0] = -om * (f[0] - fe) + w * hom * (-uf3);
  }
#pragma unroll
  for (int q = 1; q < L::Q; q += 2) {
    const C cx = C(L::ex(q)), cy = C(L::ey(q)), cz = C(L::ez(q));
    const C w = C(L::w(q));
    const C eu = cx * ux + cy * uy + cz * uz;
    const C ef = cx * Fx + cy * Fy + cz * Fz;
    const C even = C(4.5) * eu * eu - uu15;
    const C odd = C(3) * eu;
    C fp, fm;
    if (shifted) {
      const C a = r + rho * even, b = rho * odd;
      fp = w * (a + b); fm = w * (a - b);
    } else {
      const C wr = w * rho;
      fp = wr * (C(1) + even + odd); fm = wr * (C(1) + even - odd);
    }
    const C se = w * hom * (C(9) * eu * ef - uf3);
    const C so = w * hom * (C(3) * ef);
    d[q] = -om * (f[q] - fp) + (se + so);
    d[q + 1] = -om * (f[q + 1] - fm) + (se - so);
  }
}

// Exact conservation of the FP32 increment: in exact arithmetic the BGK + Guo
// increment carries no mass and exactly the momentum F; FP32 rounding of the
// equilibrium leaves residuals of ~1e-11 per node and step that do not
// decorrelate from step to step in slowly varying flows and act as a spurious
// body force.  The residuals are summed and removed from the rest population
// (mass) and from the three axis pairs (momentum), which leaves the
// second-order moments untouched.
//
// The shifted (FP32-arithmetic) collision with the conservation correction of
// conserve_fp32 folded in: increments are produced pair by pair, their FP64
// mass / momentum residuals accumulated, the 12 (D3Q19) or 4 (D2Q9) diagonal
// populations stored at once, and only the rest and axis increments kept for
// the correction -- fewer live registers than holding all Q increments.
template <class L, class S, class I>
__device__ __forceinline__ void collide_store_conserved(const float (&f)[L::Q], float r, float rho,
                                                        float ux, float uy, float uz, float Fx,
                                                        float Fy, float Fz, float om,
                                                        typename S::T* __restrict__ fout, I qs,
                                                        I n) {
  const float hom = 1.0f - 0.5f * om;
  const float uu15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  const float uf3 = 3.0f * (ux * Fx + uy * Fy + uz * Fz);
  // residual sums in FP32: their own rounding (~1e-13 on increments of ~1e-6)
  // is two orders below the residuals they remove and does not correlate in time
  float m = 0.0f, px = -Fx, py = -Fy, pz = -Fz;
  float d0, da[2 * L::D];
  {
    const float w = float(L::w(0));
    d0 = -om * (f[0] - w * (r - rho * uu15)) + w * hom * (-uf3);
    m += d0;
  }
#pragma unroll
  for (int q = 1; q < L::Q; q += 2) {
    const float cx = float(L::ex(q)), cy = float(L::ey(q)), cz = float(L::ez(q));
    const float w = float(L::w(q));
    const float eu = cx * ux + cy * uy + cz * uz;
    const float ef = cx * Fx + cy * Fy + cz * Fz;
    const float aa = r + rho * (4.5f * eu * eu - uu15), bb = rho * (3.0f * eu);
    const float se = w * hom * (9.0f * eu * ef - uf3);
    const float so = w * hom * (3.0f * ef);
    const float dp = -om * (f[q] - w * (aa + bb)) + (se + so);
    const float dm = -om * (f[q + 1] - w * (aa - bb)) + (se - so);
    const float dd = dp - dm;
    m += dp + dm;
    if (L::ex(q) == 1) px += dd; else if (L::ex(q) == -1) px -= dd;
    if (L::ey(q) == 1) py += dd; else if (L::ey(q) == -1) py -= dd;
    if (L::D == 3) { if (L::ez(q) == 1) pz += dd; else if (L::ez(q) == -1) pz -= dd; }
    if (q < 2 * L::D) {
      da[q - 1] = dp;
      da[q] = dm;
    } else {
      S::st(fout + pidx<L, S, I>(q, n, qs), f[q] + dp);
      S::st(fout + pidx<L, S, I>(q + 1, n, qs), f[q + 1] + dm);
    }
  }
  // remove the residuals: mass from the rest population, momentum from the
  // axis pairs (q = 1,2 along x; 3,4 along y; 5,6 along z)
  S::st(fout + pidx<L, S, I>(0, n, qs), f[0] + (d0 - m));
  const float pr[3] = {0.5f * px, 0.5f * py, 0.5f * pz};
#pragma unroll
  for (int a = 0; a < L::D; a++) {
    S::st(fout + pidx<L, S, I>(2 * a + 1, n, qs), f[2 * a + 1] + (da[2 * a] - pr[a]));
    S::st(fout + pidx<L, S, I>(2 * a + 2, n, qs), f[2 * a + 2] + (da[2 * a + 1] + pr[a]));
  }
}

// ---------------------------------------------------------------------------
// K1: fused stream (step k-1) + external force + moments + BGK/Guo collision
// (step k).  One thread per node, threads along x.
//   write_rho: 0 none, 1 only nodes next to a moving wall, 2 every node.
// Everything after the pull, for node (i,j,k) = n with its post-stream
// populations in f.
template <class L, class S, class I>
__device__ __forceinline__ void node_update(const LBArgs<S>& a, typename S::C (&f)[L::Q], int i,
                                            int j, int k, I n, bool has_force) {
  using C = typename S::C;
  const Geom& g = a.g;
  const I qs = (I)g.qs;
  // The force of a flagged node is loaded before any other memory operation
  // of the update, so that its latency overlaps the population loads.
  // apply_external_force (fix_couplb.cpp:693-707): F += g * rho[n], rho[n]
  // being the density the last moment pass stored.
  C Fx = C(0), Fy = C(0), Fz = C(0);
  if (has_force) {
    using A = typename S::A;
    A* p = a.F + 4 * (size_t)n;
    const A fx = p[0], fy = p[1], fz = p[2];
    Fx = C(fx); Fy = C(fy); Fz = C(fz);
    if (fx != A(0) || fy != A(0) || fz != A(0)) { p[0] = A(0); p[1] = A(0); p[2] = A(0); }
  }
  C r, jx, jy, jz;
  moments<L, C>(f, r, jx, jy, jz);
  // r is rho (plain) or the density deviation (shifted)
  C rho = S::kShift ? C(g.rho0) + r : r;
  const C rho_c = clamp_rho(rho, a.status, kStClamps);
  if (rho_c != rho) { rho = rho_c; r = S::kShift ? rho - C(g.rho0) : rho; }

  if (a.rho_mode != kRhoNone) {
    C rp;
    if (a.rho_mode == kRhoField) rp = S::kShift ? C(g.rho0) + C(a.rho_field[n]) : C(a.rho_field[n]);
    else rp = rho;
    Fx += C(a.grav[0]) * rp;
    Fy += C(a.grav[1]) * rp;
    Fz += C(a.grav[2]) * rp;
  }
  if (a.write_rho == 2 || (a.write_rho == 1 && near_moving_wall<L>(g, i, j, k)))
    a.rho_field[n] = typename S::A(S::kShift ? r : rho);

  // compute_macroscopic(true): u = (sum e f + F/2) / rho
  const C inv_r = C(1) / rho;
  const C ux = (jx + C(0.5) * Fx) * inv_r;
  const C uy = (jy + C(0.5) * Fy) * inv_r;
  const C uz = (jz + C(0.5) * Fz) * inv_r;

  if constexpr (S::kShift) {
    collide_store_conserved<L, S, I>(f, r, rho, ux, uy, uz, Fx, Fy, Fz, float(a.omega), a.fout, qs, n);
  } else {
    C d[L::Q];
    collision_increment<L, C>(f, r, rho, ux, uy, uz, Fx, Fy, Fz, C(a.omega), false, d);
#pragma unroll
    for (int q = 0; q < L::Q; q++) S::st(a.fout + pidx<L, S, I>(q, n, qs), f[q] + d[q]);
  }
}

template <class L, class S, class I, bool kPull>
__global__ void __launch_bounds__(256) k_stream_collide(const LBArgs<S> a) {
  using C = typename S::C;
  const Geom& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const I n = (I)i + (I)g.nx * ((I)j + (I)g.ny * (I)k);
  const bool hf = a.F && (!a.seg_force || a.seg_force[n >> 3]);
  C f[L::Q];
  load_node<L, S, I, kPull>(g, a.fin, a.rho_field, i, j, k, n, f);
  node_update<L, S, I>(a, f, i, j, k, n, hf);
}

// Status word slot of the bounded device waits (grid barriers of the
// cooperative IBM kernels) that gave up.
enum : int { kStTimeout = 3 };

// ---------------------------------------------------------------------------
// K2: moments of the post-stream state without the Guo term
// (compute_macroscopic(false), couplb_lattice.h:155-202).  Writes rho (or its
// deviation when shifted) and u.
template <class S>
struct MacroArgs {
  Geom g;
  const typename S::T* __restrict__ fin;
  const typename S::A* __restrict__ rho_field;
  typename S::A* __restrict__ rho;
  typename S::A* __restrict__ ux;
  typename S::A* __restrict__ uy;
  typename S::A* __restrict__ uz;
  int* status;
};

template <class L, class S, bool kPull>
__global__ void __launch_bounds__(256) k_macro(const MacroArgs<S> a) {
  using C = typename S::C;
  using I = size_t;
  const Geom& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const I n = (I)i + (I)g.nx * ((I)j + (I)g.ny * (I)k);
  C f[L::Q];
  load_node<L, S, I, kPull>(g, a.fin, a.rho_field, i, j, k, n, f);
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
                                                     const typename S::A* __restrict__ rho_field,
                                                     typename S::T* __restrict__ fout) {
  using C = typename S::C;
  using I = size_t;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const I n = (I)i + (I)g.nx * ((I)j + (I)g.ny * (I)k);
  C f[L::Q];
  load_node<L, S, I, true>(g, fin, rho_field, i, j, k, n, f);
#pragma unroll
  for (int q = 0; q < L::Q; q++) S::st(fout + pidx<L, S, I>(q, n, (I)g.qs), f[q]);
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
    S::st(f + pidx<L, S, long long>(q, n, g.qs), typename S::C(S::kShift ? fe - L::w(q) * g.rho0 : fe));
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
    S::st(f + pidx<L, S, long long>(q, n, g.qs), typename S::C(S::kShift ? v - L::w(q) * g.rho0 : v));
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
      v = double(S::ld(f + pidx<L, S, long long>(q, src, g.qs)));
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

// Force field export (interior values, ghosts zero) and import; the device
// field is interleaved, F[4n + c].
template <class S>
__global__ void k_export_force(Geom g, int D, const typename S::A* __restrict__ F, long long G,
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
    a = double(F[4 * n]); b = double(F[4 * n + 1]); c = double(F[4 * n + 2]);
  }
  dx[gn] = a; dy[gn] = b; dz[gn] = c;
}

template <class S>
__global__ void k_import_force(Geom g, int D, const double* __restrict__ sx,
                               const double* __restrict__ sy, const double* __restrict__ sz,
                               typename S::A* __restrict__ F) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int i = n % g.nx, j = (n / g.nx) % g.ny, k = n / ((long long)g.nx * g.ny);
  const int gx = g.nx + 2, gy = g.ny + 2;
  const long long gn = (i + 1) + (long long)gx * ((j + 1) + (long long)gy * (D == 3 ? k + 1 : 0));
  F[4 * n] = typename S::A(sx[gn]);
  F[4 * n + 1] = typename S::A(sy[gn]);
  F[4 * n + 2] = typename S::A(sz[gn]);
  F[4 * n + 3] = typename S::A(0);
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

// One block of kReduceThreads: thread t sums blocks t, t + kReduceThreads,
// ... in order, then a fixed-shape shared-memory tree combines the threads
// (a single thread walking the partials waited on one load per block).
constexpr int kReduceThreads = 256;
static __global__ void __launch_bounds__(kReduceThreads) k_reduce_final(int nblocks, const double* __restrict__ part,
                                                                        double* __restrict__ out) {
  double o[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += kReduceThreads) {
    o[0] = fmax(o[0], part[b * 5]);
    for (int c = 1; c < 5; c++) o[c] += part[b * 5 + c];
  }
  __shared__ double sh[5][kReduceThreads];
  for (int c = 0; c < 5; c++) sh[c][threadIdx.x] = o[c];
  __syncthreads();
  for (int h = kReduceThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + h]);
      for (int c = 1; c < 5; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sqrt(sh[0][0]);
    for (int c = 1; c < 5; c++) out[c] = sh[c][0];
  }
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

// Halo pack: the populations of the boundary plane of face `side` (0: k = 0,
// 1: k = nz - 1) that cross it (ez = -1 for side 0, +1 for side 1), from the
// post-collision store of the last LB step, into kHaloQ planes of nx * ny
// values in halo_slot order: the neighbour's halo of its facing side.
template <class L, class S>
__global__ void k_halo_pack(Geom g, const typename S::T* __restrict__ fin, int side,
                            typename S::T* __restrict__ out) {
  const long long sxy = (long long)g.nx * g.ny;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= kHaloQ * sxy) return;
  const int slot = (int)(e / sxy);
  const long long m = e % sxy;
  const int ez = side ? 1 : -1;
  int q = -1;
#pragma unroll
  for (int p = 0; p < L::Q; p++)
    if (L::ez(p) == ez && halo_slot<L>(p) == slot) q = p;
  const long long k = side ? g.nz - 1 : 0;
  out[e] = fin[pidx<L, S, long long>(q, m + k * sxy, g.qs)];
}

}  // namespace couplb
