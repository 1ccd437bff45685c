// ibm_kernels.cuh -- immersed-boundary coupling of one MD sub-step.
//
// One warp per marker: the 4^D stencil nodes of the marker are split over
// the 32 lanes (two nodes per lane in 3D), the interpolation sums are
// warp-reduced with shuffles, lane 0 forms the penalty force, and every lane
// spreads onto its own fluid nodes with atomics.  The window, its clipping to
// the ghost-inclusive box and the per-type weights are those of
// IBM::interpolate / IBM::spread (couplb_ibm.h:57-133); a periodic ghost node
// of the window reads and receives through its interior image, which is what
// exchange_velocity / exchange_forces do on one rank.
#pragma once
#include "lbm_kernels.cuh"

namespace couplb {

// delta_roma (couplb_ibm.h:11-22)
template <class R>
__device__ __forceinline__ R delta_roma(R r) {
  const R ar = fabs(r);
  if (ar <= R(0.5)) {
    const R a = R(1) - R(3) * r * r;
    return (R(1) + sqrt(a > R(0) ? a : R(0))) / R(3);
  }
  if (ar <= R(1.5)) {
    const R a = R(-2) + R(6) * ar - R(3) * r * r;
    return (R(5) - R(3) * ar - sqrt(a > R(0) ? a : R(0))) / R(6);
  }
  return R(0);
}

// delta_peskin4 (couplb_ibm.h:24-35)
template <class R>
__device__ __forceinline__ R delta_peskin4(R r) {
  const R ar = fabs(r);
  if (ar <= R(1)) {
    const R a = R(1) + R(4) * ar - R(4) * ar * ar;
    return (R(3) - R(2) * ar + sqrt(a > R(0) ? a : R(0))) / R(8);
  }
  if (ar <= R(2)) {
    const R a = R(-7) + R(12) * ar - R(4) * ar * ar;
    return (R(5) - R(2) * ar - sqrt(a > R(0) ? a : R(0))) / R(8);
  }
  return R(0);
}

template <int DELTA, class R>
__device__ __forceinline__ R delta1(R r) {
  return DELTA == 0 ? delta_roma<R>(r) : delta_peskin4<R>(r);
}

template <class S>
struct IbmArgs {
  Geom g;
  const typename S::A* __restrict__ ux;   // moments of the post-stream state
  const typename S::A* __restrict__ uy;
  const typename S::A* __restrict__ uz;
  typename S::A* Fx;                      // Eulerian force field (accumulated)
  typename S::A* Fy;
  typename S::A* Fz;
  int n;
  const double* __restrict__ x;           // n*3, MD units
  const double* __restrict__ v;           // n*3
  const double* __restrict__ m;           // n
  const int* __restrict__ active;         // n or null
  double* fout;                           // n*3 marker forces
  int accumulate;                         // 1: fout += F, 0: fout = F (0 for inactive)
  double* ftot;                           // [3] FP64 sum of the spread grid force
  double lo[3];
  int off[3];
  double inv_dx, xi_over_dt, inv_N, vs, fs, dvr;
};

// Weight arithmetic in the storage's compute type: FP64 for the parity form,
// FP32 for the shifted forms.  Sums are carried in FP64 either way.
template <class L, class S, int DELTA>
__global__ void __launch_bounds__(256) k_ibm_substep(const IbmArgs<S> a) {
  using R = typename S::C;
  const int mk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (mk >= a.n) return;
  if (a.active && !a.active[mk]) {
    if (!a.accumulate && lane < 3) a.fout[3 * mk + lane] = 0.0;
    return;
  }
  const Geom& g = a.g;
  const double xp = a.x[3 * mk], yp = a.x[3 * mk + 1], zp = a.x[3 * mk + 2];
  // IBM::phys_to_local (couplb_ibm.h:49-55)
  const double lx = (xp - a.lo[0]) * a.inv_dx - a.off[0] + 1.0;
  const double ly = (yp - a.lo[1]) * a.inv_dx - a.off[1] + 1.0;
  const double lz = (L::D == 3) ? ((zp - a.lo[2]) * a.inv_dx - a.off[2] + 1.0) : 0.0;
  const int i0 = (int)floor(lx), j0 = (int)floor(ly);
  const int k0 = (L::D == 3) ? (int)floor(lz) : 0;
  const int gx = g.nx + 2, gy = g.ny + 2, gz = (L::D == 3) ? g.nz + 2 : 1;
  constexpr int NS = (L::D == 3) ? 64 : 16;

  double ui = 0, vi = 0, wi = 0, ws = 0, wss = 0;
  long long sn0 = -1, sn1 = -1;   // fluid nodes of this lane (interior index)
  double sd0 = 0, sd1 = 0;
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int s = lane + 32 * rep;
    if (s >= NS) break;
    const int ig = i0 - 1 + (s & 3);
    const int jg = j0 - 1 + ((s >> 2) & 3);
    const int kg = (L::D == 3) ? k0 - 1 + (s >> 4) : 0;
    if (ig < 0 || ig >= gx || jg < 0 || jg >= gy || kg < 0 || kg >= gz) continue;
    R d = delta1<DELTA, R>(R(lx - ig)) * delta1<DELTA, R>(R(ly - jg));
    if (L::D == 3) d *= delta1<DELTA, R>(R(lz - kg));
    long long src = 0;
    const int t = classify_ghost(g, L::D, ig, jg, kg, &src);
    const double dd = double(d);
    if (t < 0) {
      ui += double(a.ux[src]) * dd;
      vi += double(a.uy[src]) * dd;
      wi += double(a.uz[src]) * dd;
      ws += dd;
      wss += dd;
      if (rep == 0) { sn0 = src; sd0 = dd; } else { sn1 = src; sd1 = dd; }
    } else if (t == 1 || t == 3) {
      ws += dd;
    } else if (t == 2) {
      ui += g.uw[0] * dd;
      vi += g.uw[1] * dd;
      wi += (L::D == 3 ? g.uw[2] : 0.0) * dd;
      ws += dd;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ui += __shfl_xor_sync(0xffffffffu, ui, o);
    vi += __shfl_xor_sync(0xffffffffu, vi, o);
    wi += __shfl_xor_sync(0xffffffffu, wi, o);
    ws += __shfl_xor_sync(0xffffffffu, ws, o);
    wss += __shfl_xor_sync(0xffffffffu, wss, o);
  }
  double u0 = 0, u1 = 0, u2 = 0;
  if (ws > DELTA_TOL) {
    const double iw = 1.0 / ws;
    u0 = ui * iw; u1 = vi * iw; u2 = wi * iw;
  }
  // penalty force (fix_couplb.cpp:777-781)
  const double mass = a.m[mk];
  const double F0 = mass * a.xi_over_dt * (u0 * a.vs - a.v[3 * mk]);
  const double F1 = mass * a.xi_over_dt * (u1 * a.vs - a.v[3 * mk + 1]);
  const double F2 = mass * a.xi_over_dt * (u2 * a.vs - a.v[3 * mk + 2]);
  if (lane == 0) {
    if (a.accumulate) {
      a.fout[3 * mk] += F0; a.fout[3 * mk + 1] += F1; a.fout[3 * mk + 2] += F2;
    } else {
      a.fout[3 * mk] = F0; a.fout[3 * mk + 1] = F1; a.fout[3 * mk + 2] = F2;
    }
  }
  // spread -F/(N * force_scale) (fix_couplb.cpp:788-792, couplb_ibm.h:124-132)
  if (wss < DELTA_TOL) return;
  const double sc = a.dvr / wss;
  const double fl0 = -F0 * a.inv_N / a.fs, fl1 = -F1 * a.inv_N / a.fs, fl2 = -F2 * a.inv_N / a.fs;
  if (sn0 >= 0) {
    const double w = sd0 * sc;
    atomicAdd(a.Fx + sn0, typename S::A(fl0 * w));
    atomicAdd(a.Fy + sn0, typename S::A(fl1 * w));
    atomicAdd(a.Fz + sn0, typename S::A(fl2 * w));
  }
  if (sn1 >= 0) {
    const double w = sd1 * sc;
    atomicAdd(a.Fx + sn1, typename S::A(fl0 * w));
    atomicAdd(a.Fy + sn1, typename S::A(fl1 * w));
    atomicAdd(a.Fz + sn1, typename S::A(fl2 * w));
  }
  if (lane == 0 && a.ftot) {
    atomicAdd(a.ftot, fl0 * a.dvr);
    atomicAdd(a.ftot + 1, fl1 * a.dvr);
    atomicAdd(a.ftot + 2, fl2 * a.dvr);
  }
}

}  // namespace couplb
