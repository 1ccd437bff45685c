// ibm_methods.cuh -- IBM forcing beyond the single penalty pass: the
// iterative (multi-direct forcing) corrections, the slip residual that judges
// the learned correction, and the training-sample capture.
//
// No counterpart in the reference, which applies one penalty pass.  The
// definitions (restated on the CPU by the oracle):
//   u_corr(x) = u0(x) + (G(x)/rho(x) + g_lb)/2 at fluid nodes: u0 and rho of
//               the refresh, G the IBM force field so far, g_lb the body force;
//   U_i       = the reference's interpolation of u_corr (couplb_ibm.h:57-90);
//   dF_i      = m xi/dt (U_i vs - v_i), added to the atom and spread as
//               -dF_i/(N fs) with the reference's spread weights; all dF_i of
//               a pass are formed before any is spread (Jacobi);
//   slip_i    = |U_i vs - v_i| after the last pass.
//
// One cooperative launch runs the whole sub-step: warps loop over the markers;
// the first phase fills each marker's stencil record at a refresh, forms the
// penalty force (plus the network correction) and spreads it, and grid-wide
// barriers (bounded waits, error flag on timeout) separate it and each
// "form all dF" from the following "spread all dF".  The learned method
// measures the slip first and runs the corrections only when its RMS exceeds
// the tolerance, so the fallback costs nothing when the network is good enough.
#pragma once
#include "ibm_kernels.cuh"

namespace couplb {

constexpr int kSlipSlots = 32;
// status words (cumulative until reset): slip checks made, fallbacks taken
enum : int { kStSlipChecks = 4, kStFallbacks = 5 };
// default poll limit of a grid barrier (each failed poll sleeps ~100 ns);
// the handle option "barrier_spin" replaces it (tests drive a barrier to its
// limit with 0)
constexpr long long kBarrierSpin = 1LL << 21;
// slip_tol at or above which the learned method has no fallback (and so no
// slip check)
constexpr double kNoFallback = 1e300;

// State of one launch of k_ibm_method.  Two alternate: each launch zeroes the
// other one for the next launch.
// Slip accumulators are striped over kSlipSlots by marker index: a single
// word hit by every marker serialises in L2.  [0]: the learned check,
// [1]: after the last pass.
struct PassState {
  unsigned bar_count, bar_gen;
  int fell_back;                               // the learned method ran the corrections
  int checked;                                 // a slip check ran
  double s2[2][kSlipSlots];                    // slip^2 sums
  unsigned long long max_bits[2][kSlipSlots];  // max slip (non-negative double bits)
  int count[2][kSlipSlots];                    // markers
};

template <class S>
struct PassArgs {
  IbmArgs<S> a;
  double* dF;           // n*3: the increment of the current pass
  PassState* ps;        // zeroed state of this launch
  PassState* ps_next;   // zeroed here for the next launch
  int fill;             // first phase computes the stencil records (refresh)
  int* status;
  int ncorr;            // iterative corrections (passes - 1)
  int check_first;      // learned: slip check first, corrections only above tol
  int measure_last;     // slip after the last pass into residual 1 (handle option ibm_slip)
  double slip_tol;      // MD velocity units
  double g_lb[3];       // body force of the LB steps, lattice units
  float* rows;          // n x kMlpRow training rows, or null
  long long spin;       // grid-barrier poll limit
};

// Grid-wide barrier of a cooperative launch.  Returns false (and counts a
// timeout) if the other blocks did not arrive within `spin` failed polls; the
// caller then returns, so every block ends after at most one wait per
// remaining barrier.  The arrival counter of a launch that gave up is left
// behind in its PassState, which the next launch does not use (it zeroes it
// for the launch after).
__device__ __forceinline__ bool grid_barrier(PassState* ps, int* status, long long spin) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &ps->bar_gen;
    const unsigned g0 = *gen;
    __threadfence();
    int good = 1;
    if (atomicAdd(&ps->bar_count, 1u) + 1 == gridDim.x) {
      atomicExch(&ps->bar_count, 0u);
      __threadfence();
      atomicAdd(&ps->bar_gen, 1u);
    } else {
      long long it = 0;
      while (*gen == g0) {
        if (++it > spin) {
          good = 0;
          if (status) atomicAdd(status + kStTimeout, 1);
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ void load_force(const float* F, size_t n, double G[3]) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(F + 4 * n));
  G[0] = v.x; G[1] = v.y; G[2] = v.z;
}
__device__ __forceinline__ void load_force(const double* F, size_t n, double G[3]) {
  G[0] = __ldcg(F + 4 * n); G[1] = __ldcg(F + 4 * n + 1); G[2] = __ldcg(F + 4 * n + 2);
}

// Marker window of the reference (couplb_ibm.h:62-86).
struct MarkerWindow {
  double lx, ly, lz;
  int i0, j0, k0;
};

template <class L, class S>
__device__ __forceinline__ MarkerWindow marker_window(const IbmArgs<S>& a, int mk) {
  MarkerWindow w;
  w.lx = (a.x[3 * mk] - a.lo[0]) * a.inv_dx - a.off[0] + 1.0;
  w.ly = (a.x[3 * mk + 1] - a.lo[1]) * a.inv_dx - a.off[1] + 1.0;
  w.lz = (L::D == 3) ? ((a.x[3 * mk + 2] - a.lo[2]) * a.inv_dx - a.off[2] + 1.0) : 0.0;
  w.i0 = (int)floor(w.lx);
  w.j0 = (int)floor(w.ly);
  w.k0 = (L::D == 3) ? (int)floor(w.lz) : 0;
  return w;
}

// Interpolated u_corr of marker mk (every lane returns it).
template <class L, class S, int DELTA>
__device__ __forceinline__ void interp_corr(const PassArgs<S>& P, int mk, int lane, double U[3]) {
  using R = typename S::C;
  const IbmArgs<S>& a = P.a;
  const Geom& g = a.g;
  const MarkerWindow w = marker_window<L, S>(a, mk);
  constexpr int NS = (L::D == 3) ? 64 : 16;
  const StencilKey key = a.skey[mk];
  const bool hit = key.epoch == a.cur_epoch && key.i0 == w.i0 && key.j0 == w.j0 && key.k0 == w.k0;
  const typename S::A* rec = stencil_record(a, mk);
  const LaneNodes<R> ln = lane_nodes<L, DELTA, R>(g, w.lx, w.ly, w.lz, w.i0, w.j0, w.k0, lane, a.wrap);
  double ui = 0, vi = 0, wi = 0, ws = 0;
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int s = lane + 32 * rep;
    if (s >= NS) break;
    const int t = ln.t[rep];
    if (t == -2) continue;
    const double dd = double(ln.d[rep]);
    if (t < 0) {
      const size_t n = (size_t)ln.n[rep];
      double u0, u1, u2, rho;
      node_state<L, S>(a, hit, rec, s, ln.i, ln.j, ln.k[rep], n, u0, u1, u2, rho);
      double G[3];
      load_force(a.F, n, G);
      const double ir = 1.0 / rho;
      u0 = u0 + 0.5 * (G[0] * ir + P.g_lb[0]);
      u1 = u1 + 0.5 * (G[1] * ir + P.g_lb[1]);
      u2 = u2 + 0.5 * (G[2] * ir + (L::D == 3 ? P.g_lb[2] : 0.0));
      ui += u0 * dd; vi += u1 * dd; wi += u2 * dd; ws += dd;
    } else if (t == 1 || t == 3) {
      ws += dd;
    } else if (t == 2) {
      ui += g.uw[0] * dd; vi += g.uw[1] * dd; wi += (L::D == 3 ? g.uw[2] : 0.0) * dd; ws += dd;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ui += __shfl_xor_sync(0xffffffffu, ui, o);
    vi += __shfl_xor_sync(0xffffffffu, vi, o);
    wi += __shfl_xor_sync(0xffffffffu, wi, o);
    ws += __shfl_xor_sync(0xffffffffu, ws, o);
  }
  if (ws > DELTA_TOL) {
    const double iw = 1.0 / ws;
    U[0] = ui * iw; U[1] = vi * iw; U[2] = wi * iw;
  } else {
    U[0] = U[1] = U[2] = 0.0;
  }
}

// Spread -dF/(N fs) of marker mk with the reference's weights
// (couplb_ibm.h:92-133).
template <class L, class S, int DELTA>
__device__ __forceinline__ void spread_marker(const IbmArgs<S>& a, int mk, int lane,
                                              const double dF[3], double* tot3 = nullptr) {
  using R = typename S::C;
  const Geom& g = a.g;
  const MarkerWindow w = marker_window<L, S>(a, mk);
  constexpr int NS = (L::D == 3) ? 64 : 16;
  long long sn0 = -1, sn1 = -1;
  double sd0 = 0.0, sd1 = 0.0;
  double wss = 0.0;
  const LaneNodes<R> ln = lane_nodes<L, DELTA, R>(g, w.lx, w.ly, w.lz, w.i0, w.j0, w.k0, lane, a.wrap);
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int s = lane + 32 * rep;
    if (s >= NS) break;
    if (ln.t[rep] != -1) continue;
    const double dd = double(ln.d[rep]);
    wss += dd;
    if (rep == 0) { sn0 = ln.n[0]; sd0 = dd; }
    else { sn1 = ln.n[1]; sd1 = dd; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wss += __shfl_xor_sync(0xffffffffu, wss, o);
  if (wss < DELTA_TOL) return;
  const double sc = a.dvr / wss;
  const double fl0 = -dF[0] * a.spread_c, fl1 = -dF[1] * a.spread_c;
  const double fl2 = -dF[2] * a.spread_c;
  if (sn0 >= 0) {
    const double wgt = sd0 * sc;
    spread_add(a.F + 4 * sn0, fl0 * wgt, fl1 * wgt, fl2 * wgt);
    if (a.seg_force) a.seg_force[sn0 >> 3] = 1;
  }
  if (sn1 >= 0) {
    const double wgt = sd1 * sc;
    spread_add(a.F + 4 * sn1, fl0 * wgt, fl1 * wgt, fl2 * wgt);
    if (a.seg_force) a.seg_force[sn1 >> 3] = 1;
  }
  if (lane == 0 && tot3) {
    tot3[0] += fl0 * a.dvr;
    tot3[1] += fl1 * a.dvr;
    tot3[2] += fl2 * a.dvr;
  } else if (lane == 0 && a.ftot) {
    double* t = a.ftot + 4 * (mk & (kFtotSlots - 1));
    atomicAdd(t, fl0 * a.dvr);
    atomicAdd(t + 1, fl1 * a.dvr);
    atomicAdd(t + 2, fl2 * a.dvr);
  }
}

// A warp's running slip sums (lane 0) until its block adds them.
struct SlipAcc {
  double s2 = 0.0, mx = 0.0;
  int cnt = 0;
};

// Slip of marker mk into residual r of the pass state, or (acc) into the
// warp's running sums.
template <class L, class S, int DELTA>
__device__ __forceinline__ void measure_marker(const PassArgs<S>& P, int mk, int lane, int r,
                                               SlipAcc* acc = nullptr) {
  double U[3];
  interp_corr<L, S, DELTA>(P, mk, lane, U);
  if (lane == 0) {
    const IbmArgs<S>& a = P.a;
    double e2 = 0.0;
    for (int c = 0; c < 3; c++) {
      const double e = U[c] * a.vs - a.v[3 * mk + c];
      e2 += e * e;
    }
    if (acc) {
      acc->s2 += e2;
      acc->mx = fmax(acc->mx, sqrt(e2));
      acc->cnt++;
      return;
    }
    const int sl = mk & (kSlipSlots - 1);
    atomicAdd(&P.ps->s2[r][sl], e2);
    atomicMax(&P.ps->max_bits[r][sl], (unsigned long long)__double_as_longlong(sqrt(e2)));
    atomicAdd(&P.ps->count[r][sl], 1);
  }
}

// Per-block sums of the warps' running accumulators, then one set of FP64
// atomics per block: with 2e5 markers, per-marker atomics on the 64 force
// and 32 slip slots queued in L2 for a large part of each pass.  Every thread
// of the block calls these at the same point.
__device__ __forceinline__ void block_add_ftot(double* ftot, double t[3]) {
  __shared__ double part[8][3];
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { part[warp][0] = t[0]; part[warp][1] = t[1]; part[warp][2] = t[2]; }
  __syncthreads();
  if (ftot && threadIdx.x < 3) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += part[w][threadIdx.x];
    atomicAdd(ftot + 4 * (blockIdx.x & (kFtotSlots - 1)) + threadIdx.x, sum);
  }
  __syncthreads();
  t[0] = t[1] = t[2] = 0.0;
}

__device__ __forceinline__ void block_add_slip(PassState* ps, int r, SlipAcc& acc) {
  __shared__ double ps2[8], pmx[8];
  __shared__ int pcnt[8];
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { ps2[warp] = acc.s2; pmx[warp] = acc.mx; pcnt[warp] = acc.cnt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0, mx = 0.0;
    int cnt = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      sum += ps2[w];
      mx = fmax(mx, pmx[w]);
      cnt += pcnt[w];
    }
    if (cnt) {
      const int sl = blockIdx.x & (kSlipSlots - 1);
      atomicAdd(&ps->s2[r][sl], sum);
      atomicMax(&ps->max_bits[r][sl], (unsigned long long)__double_as_longlong(mx));
      atomicAdd(&ps->count[r][sl], cnt);
    }
  }
  __syncthreads();
  acc = SlipAcc();
}

// RMS slip of residual r after the barrier that closed it: warp 0 of the
// block reads the slots (lane = slot) and shares the result; every block
// reduces in the same order, so all take the same decision.
__device__ __forceinline__ double slip_rms(const PassState* ps, int r) {
  static_assert(kSlipSlots == 32, "one slot per lane");
  __shared__ double rms;
  if (threadIdx.x < 32) {
    double s = __ldcg(&ps->s2[r][threadIdx.x]);
    int c = __ldcg(&ps->count[r][threadIdx.x]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (threadIdx.x == 0) rms = c > 0 ? sqrt(s / c) : 0.0;
  }
  __syncthreads();
  return rms;
}

// Training row of marker mk: network input, then the correction beyond the
// penalty pass over (m xi vs / dt), lattice velocity units, then 0.
template <class L, class S>
__device__ __forceinline__ void record_marker(const PassArgs<S>& P, int mk, int lane) {
  const IbmArgs<S>& a = P.a;
  const Geom& g = a.g;
  float* row = P.rows + (size_t)mk * kMlpRow;
  for (int t = lane; t < kMlpRow; t += 32) row[t] = 0.f;
  __syncwarp();
  if (L::D != 3) return;
  const MarkerWindow w = marker_window<L, S>(a, mk);
  const int ox = (w.lx - w.i0) >= 0.5 ? 1 : 0, oy = (w.ly - w.j0) >= 0.5 ? 1 : 0;
  const int oz = (w.lz - w.k0) >= 0.5 ? 1 : 0;
  const int gx = g.nx + 2, gy = g.ny + 2, gz = g.nz + 2;
  const StencilKey key = a.skey[mk];
  const bool hit = key.epoch == a.cur_epoch && key.i0 == w.i0 && key.j0 == w.j0 && key.k0 == w.k0;
  const typename S::A* rec = stencil_record(a, mk);
  if (lane < 27) {
    const int rx = lane % 3, ry = (lane / 3) % 3, rz = lane / 9;
    const int s = (rx + ox) + 4 * (ry + oy) + 16 * (rz + oz);   // window slot
    int ig = w.i0 - 1 + rx + ox, jg = w.j0 - 1 + ry + oy, kg = w.k0 - 1 + rz + oz;
    if (a.wrap & 1) ig = wrap_ghost_index(ig, g.nx);
    if (a.wrap & 2) jg = wrap_ghost_index(jg, g.ny);
    if (a.wrap & 4) kg = wrap_ghost_index(kg, g.nz);
    if (ig >= 0 && ig < gx && jg >= 0 && jg < gy && kg >= 0 && kg < gz) {
      int ii = 0, jj = 0, kk = 0;
      const int t = classify_node(g, 3, ig, jg, kg, ii, jj, kk);
      if (t < 0) {
        const size_t n = (size_t)ii + (size_t)g.nx * ((size_t)jj + (size_t)g.ny * kk);
        double u0, u1, u2;
        node_velocity<L, S>(a, hit, rec, s, ii, jj, kk, n, u0, u1, u2);
        row[3 * lane] = float(u0); row[3 * lane + 1] = float(u1); row[3 * lane + 2] = float(u2);
      } else if (t == 2) {
        row[3 * lane] = float(g.uw[0]); row[3 * lane + 1] = float(g.uw[1]);
        row[3 * lane + 2] = float(g.uw[2]);
      }
    }
  } else if (lane < 30) {
    const int c = lane - 27;
    row[81 + c] = float(a.v[3 * mk + c] / a.vs);
    row[kMlpIn + c] = float(a.corr[3 * mk + c] / (a.m[mk] * a.xi_over_dt * a.vs));
  }
}

// One sub-step of the ITERATIVE or LEARNED method (cooperative launch, blocks
// of 256 threads, at most as many blocks as fit on the device at once;
// LEARNED: D3Q19, dynamic shared memory kLearnedSmem).
template <class L, class S, int DELTA, bool LEARNED>
__global__ void __launch_bounds__(256) k_ibm_method(const PassArgs<S> P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const IbmArgs<S>& a = P.a;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  MlpPacked* net = reinterpret_cast<MlpPacked*>(smem);
  MlpBlockScratch* blk = reinterpret_cast<MlpBlockScratch*>(smem + sizeof(MlpPacked));
  if (LEARNED) mlp_stage_async(net, a.mlp);   // waited for before the first network pass
  if (blockIdx.x == 0) {
    unsigned* z = reinterpret_cast<unsigned*>(P.ps_next);
    for (int i = threadIdx.x; i < (int)(sizeof(PassState) / 4); i += blockDim.x) z[i] = 0u;
  }
  double ft[3] = {0.0, 0.0, 0.0};
  SlipAcc acc;
  // first pass: the reference's penalty pass (+ the network correction; the
  // block's warps step through the markers together, as its network pass
  // needs all of them)
  const int wpb = (int)(blockDim.x >> 5);
  const int mk_end = LEARNED ? (a.n + wpb - 1) / wpb * wpb : a.n;
  for (int mk = gw; mk < mk_end; mk += nw) {
    double t3[3] = {0.0, 0.0, 0.0};
    ibm_substep_body<L, S, DELTA, LEARNED, false>(a, mk, lane, P.fill != 0, net, blk, t3);
    ft[0] += t3[0]; ft[1] += t3[1]; ft[2] += t3[2];
  }
  block_add_ftot(a.ftot, ft);
  // a launch with nothing after the first pass that reads the force field
  // (no check, no correction, no slip statistics) needs no grid barrier
  const bool more = P.check_first || P.ncorr > 0 || P.measure_last;
  if (more && !grid_barrier(P.ps, P.status, P.spin)) return;
  if (P.check_first) {
    for (int mk = gw; mk < a.n; mk += nw)
      if (!a.active || a.active[mk]) measure_marker<L, S, DELTA>(P, mk, lane, 0, &acc);
    block_add_slip(P.ps, 0, acc);
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
    const bool fall = slip_rms(P.ps, 0) > P.slip_tol;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      P.ps->checked = 1;
      if (P.status) atomicAdd(P.status + kStSlipChecks, 1);
      if (fall) {
        P.ps->fell_back = 1;
        if (P.status) atomicAdd(P.status + kStFallbacks, 1);
      }
    }
    if (!fall) {
      if (P.rows)
        for (int mk = gw; mk < a.n; mk += nw) record_marker<L, S>(P, mk, lane);
      return;
    }
  }
  for (int it = 0; it < P.ncorr; it++) {
    for (int mk = gw; mk < a.n; mk += nw) {
      if (a.active && !a.active[mk]) continue;
      double U[3];
      interp_corr<L, S, DELTA>(P, mk, lane, U);
      if (lane == 0) {
        const double c = a.m[mk] * a.xi_over_dt;
        for (int d = 0; d < 3; d++) {
          const double dF = c * (U[d] * a.vs - a.v[3 * mk + d]);
          P.dF[3 * mk + d] = dF;
          a.fout[3 * mk + d] += dF;
          a.corr[3 * mk + d] += dF;
        }
      }
    }
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
    for (int mk = gw; mk < a.n; mk += nw) {
      if (a.active && !a.active[mk]) continue;
      const double dF[3] = {__ldcg(P.dF + 3 * mk), __ldcg(P.dF + 3 * mk + 1),
                            __ldcg(P.dF + 3 * mk + 2)};
      spread_marker<L, S, DELTA>(a, mk, lane, dF, ft);
    }
    block_add_ftot(a.ftot, ft);
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
  }
  for (int mk = gw; mk < a.n; mk += nw) {
    if (a.active && !a.active[mk]) continue;
    if (P.measure_last) measure_marker<L, S, DELTA>(P, mk, lane, 1, &acc);
    if (P.rows) record_marker<L, S>(P, mk, lane);
  }
  if (P.measure_last) block_add_slip(P.ps, 1, acc);
}

// The same sub-step when every marker has a warp of its own (n <= resident
// warps): a lane's two window nodes -- index, weight, type, u0 and 1/rho --
// are computed once and kept in registers across all passes, so a correction
// pass is two force-field loads, three warp reductions and two atomics per
// lane.  Same arithmetic and order as k_ibm_method.
template <class L, class S, int DELTA, bool LEARNED>
__global__ void __launch_bounds__(256) k_ibm_method_resident(const PassArgs<S> P) {
  static_assert(L::D == 3, "resident form: D3Q19");
  using R = typename S::C;
  using A = typename S::A;
  extern __shared__ __align__(16) unsigned char smem[];
  const IbmArgs<S>& a = P.a;
  const Geom& g = a.g;
  const int lane = threadIdx.x & 31;
  const int mk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  MlpPacked* net = reinterpret_cast<MlpPacked*>(smem);
  MlpBlockScratch* blk = reinterpret_cast<MlpBlockScratch*>(smem + sizeof(MlpPacked));
  float* xs = nullptr;
  if (LEARNED) {
    // the network's copy into shared memory overlaps the stencil fill; the
    // forward pass waits for it
    mlp_stage_async(net, a.mlp);
    xs = blk->x + (threadIdx.x >> 5) * kMlpXStride;
    for (int t = lane; t < kMlpXStride; t += 32) xs[t] = 0.f;
    __syncwarp();
  }
  if (blockIdx.x == 0) {
    unsigned* z = reinterpret_cast<unsigned*>(P.ps_next);
    for (int i = threadIdx.x; i < (int)(sizeof(PassState) / 4); i += blockDim.x) z[i] = 0u;
  }
  const bool have = mk < a.n && (!a.active || a.active[mk]);
  if (mk < a.n && !have && !a.accumulate && lane < 3) a.fout[3 * mk + lane] = 0.0;

  // ---- first pass: window, stencil state, penalty (+ network) force, spread
  // Node state, weights and the interpolation sums in the storage's compute
  // type R (FP32 for the shifted formats, as in the single-pass sub-step);
  // marker velocities and forces in FP64.
  long long nd[2] = {-1, -1};      // interior index of a fluid node, else -1
  R dw[2] = {R(0), R(0)};          // delta weight
  R uu[2][3] = {{0, 0, 0}, {0, 0, 0}}, ir[2] = {R(0), R(0)};
  A rh[2] = {A(0), A(0)};          // density of a filled node, for its record
  R ws = 0, wss = 0, uwx = 0, uwy = 0, uwz = 0;   // wall velocity sums
  double F0 = 0, F1 = 0, F2 = 0, c0 = 0, c1 = 0, c2 = 0, mxi = 0, vx = 0, vy = 0, vz = 0;
  if (have) {
    const MarkerWindow w = marker_window<L, S>(a, mk);
    // the marker's mass and velocity load beside its position, off the chain
    // of the stencil fill
    mxi = a.m[mk] * a.xi_over_dt;
    vx = a.v[3 * mk]; vy = a.v[3 * mk + 1]; vz = a.v[3 * mk + 2];
    const StencilKey key = a.skey[mk];
    const bool fill = P.fill != 0;
    const bool hit = key.epoch == a.cur_epoch && key.i0 == w.i0 && key.j0 == w.j0 && key.k0 == w.k0;
    A* rec = stencil_record(a, mk);
    int ox = 0, oy = 0, oz = 0;
    if (LEARNED) {
      ox = (w.lx - w.i0) >= 0.5 ? 1 : 0;
      oy = (w.ly - w.j0) >= 0.5 ? 1 : 0;
      oz = (w.lz - w.k0) >= 0.5 ? 1 : 0;
    }
    R ui = 0, vi = 0, wi = 0;
    const LaneNodes<R> ln = lane_nodes<L, DELTA, R>(g, w.lx, w.ly, w.lz, w.i0, w.j0, w.k0, lane, a.wrap);
#pragma unroll
    for (int rep = 0; rep < 2; rep++) {
      const int s = lane + 32 * rep;
      const int t = ln.t[rep];
      if (t == -2) continue;
      const R dd = ln.d[rep];
      const int ii = ln.i, jj = ln.j, kk = ln.k[rep];
      int p = -1;
      if (LEARNED) {
        const int rx = (s & 3) - ox, ry = ((s >> 2) & 3) - oy, rz = (s >> 4) - oz;
        if (rx >= 0 && rx < 3 && ry >= 0 && ry < 3 && rz >= 0 && rz < 3) p = rx + 3 * ry + 9 * rz;
      }
      if (t < 0) {
        const size_t n = (size_t)ln.n[rep];
        R u0, u1, u2, rho;
        if (fill) {
          // the record is written after the loop, so that the loads of both
          // nodes can be in flight together
          A v0, v1, v2, vr;
          compute_velocity<L, S>(a, ii, jj, kk, n, v0, v1, v2, vr);
          u0 = R(v0); u1 = R(v1); u2 = R(v2); rho = R(vr);
          rh[rep] = vr;
        } else {
          double w0, w1, w2, wr;
          node_state<L, S>(a, hit, rec, s, ii, jj, kk, n, w0, w1, w2, wr);
          u0 = R(w0); u1 = R(w1); u2 = R(w2); rho = R(wr);
        }
        nd[rep] = (long long)n; dw[rep] = dd;
        uu[rep][0] = u0; uu[rep][1] = u1; uu[rep][2] = u2; ir[rep] = R(1) / rho;
        ui += u0 * dd; vi += u1 * dd; wi += u2 * dd; ws += dd; wss += dd;
        if (LEARNED && p >= 0) { xs[3 * p] = float(u0); xs[3 * p + 1] = float(u1); xs[3 * p + 2] = float(u2); }
      } else if (t == 1 || t == 3) {
        ws += dd;
      } else if (t == 2) {
        uwx += R(g.uw[0]) * dd; uwy += R(g.uw[1]) * dd; uwz += R(g.uw[2]) * dd; ws += dd;
        if (LEARNED && p >= 0) {
          xs[3 * p] = float(g.uw[0]); xs[3 * p + 1] = float(g.uw[1]); xs[3 * p + 2] = float(g.uw[2]);
        }
      }
    }
    if (fill) {
#pragma unroll
      for (int rep = 0; rep < 2; rep++) {
        if (nd[rep] < 0) continue;
        const int s = lane + 32 * rep;
        rec[s] = A(uu[rep][0]); rec[64 + s] = A(uu[rep][1]); rec[128 + s] = A(uu[rep][2]);
        rec[192 + s] = rh[rep];
      }
      if (lane == 0) a.skey[mk] = StencilKey{w.i0, w.j0, w.k0, a.cur_epoch};
    }
    ui += uwx; vi += uwy; wi += uwz;
    // not unrolled: this launch runs once per SM and waits on instruction fetch
#pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) {
      ui += __shfl_xor_sync(0xffffffffu, ui, o);
      vi += __shfl_xor_sync(0xffffffffu, vi, o);
      wi += __shfl_xor_sync(0xffffffffu, wi, o);
      ws += __shfl_xor_sync(0xffffffffu, ws, o);
      wss += __shfl_xor_sync(0xffffffffu, wss, o);
      uwx += __shfl_xor_sync(0xffffffffu, uwx, o);
      uwy += __shfl_xor_sync(0xffffffffu, uwy, o);
      uwz += __shfl_xor_sync(0xffffffffu, uwz, o);
    }
    double U0 = 0, U1 = 0, U2 = 0;
    if (ws > R(DELTA_TOL)) {
      const R iw = R(1) / ws;
      U0 = double(ui * iw); U1 = double(vi * iw); U2 = double(wi * iw);
    }
    F0 = mxi * (U0 * a.vs - vx);
    F1 = mxi * (U1 * a.vs - vy);
    F2 = mxi * (U2 * a.vs - vz);
    if (LEARNED && lane < 3) xs[81 + lane] = float((lane == 0 ? vx : (lane == 1 ? vy : vz)) / a.vs);
  }
  if (LEARNED) {
    // the network for the block's markers (every warp takes part)
    __syncwarp();
    float y[3];
    mlp_block_forward<true>(*net, *blk, threadIdx.x >> 5, lane, y);
    if (have) {
      const double sc = mxi * a.vs;
      c0 = sc * double(y[0]); c1 = sc * double(y[1]); c2 = sc * double(y[2]);
      F0 += c0; F1 += c1; F2 += c2;
    }
  }
  if (have) {
    if (lane == 0) {
      a.corr[3 * mk] = c0; a.corr[3 * mk + 1] = c1; a.corr[3 * mk + 2] = c2;
      if (a.accumulate) {
        a.fout[3 * mk] += F0; a.fout[3 * mk + 1] += F1; a.fout[3 * mk + 2] += F2;
      } else {
        a.fout[3 * mk] = F0; a.fout[3 * mk + 1] = F1; a.fout[3 * mk + 2] = F2;
      }
    }
  }
  // spread -F/(N fs) with w = d dvr / wss (couplb_ibm.h:124-132)
  const bool spreads = have && wss >= R(DELTA_TOL);
  const R ssc = spreads ? R(a.dvr) / wss : R(0);
  // Per-block sums before the FP64 slot atomics (total force, slip): one
  // atomic per block and quantity instead of one per marker.  Every thread of
  // the block calls spread and measure at the same points.
  __shared__ double bsum[8][3];
  const int warp = threadIdx.x >> 5;
  const int nwarp = (int)(blockDim.x >> 5);
  auto spread = [&](double f0, double f1, double f2) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    if (spreads) {
      const double fl0 = -f0 * a.spread_c, fl1 = -f1 * a.spread_c, fl2 = -f2 * a.spread_c;
      const R r0 = R(fl0), r1 = R(fl1), r2 = R(fl2);
#pragma unroll
      for (int rep = 0; rep < 2; rep++) {
        if (nd[rep] < 0) continue;
        const R wgt = dw[rep] * ssc;
        spread_add(a.F + 4 * nd[rep], r0 * wgt, r1 * wgt, r2 * wgt);
        if (a.seg_force) a.seg_force[nd[rep] >> 3] = 1;
      }
      t0 = fl0 * a.dvr; t1 = fl1 * a.dvr; t2 = fl2 * a.dvr;
    }
    if (!a.ftot) return;
    if (lane == 0) { bsum[warp][0] = t0; bsum[warp][1] = t1; bsum[warp][2] = t2; }
    __syncthreads();
    if (threadIdx.x < 3) {
      double sum = 0.0;
      for (int w = 0; w < nwarp; w++) sum += bsum[w][threadIdx.x];
      atomicAdd(a.ftot + 4 * (blockIdx.x & (kFtotSlots - 1)) + threadIdx.x, sum);
    }
    __syncthreads();
  };
  // interpolated u_corr from the registers and the current force field
  auto interp_corr_reg = [&](double U[3]) {
    R ui = 0, vi = 0, wi = 0;
    const R half = R(0.5), g0 = R(P.g_lb[0]), g1 = R(P.g_lb[1]), g2 = R(P.g_lb[2]);
#pragma unroll
    for (int rep = 0; rep < 2; rep++) {
      if (nd[rep] < 0) continue;
      double G[3];
      load_force(a.F, (size_t)nd[rep], G);
      const R c0 = uu[rep][0] + half * (R(G[0]) * ir[rep] + g0);
      const R c1 = uu[rep][1] + half * (R(G[1]) * ir[rep] + g1);
      const R c2 = uu[rep][2] + half * (R(G[2]) * ir[rep] + g2);
      ui += c0 * dw[rep]; vi += c1 * dw[rep]; wi += c2 * dw[rep];
    }
#pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) {
      ui += __shfl_xor_sync(0xffffffffu, ui, o);
      vi += __shfl_xor_sync(0xffffffffu, vi, o);
      wi += __shfl_xor_sync(0xffffffffu, wi, o);
    }
    if (ws > R(DELTA_TOL)) {
      const R iw = R(1) / ws;
      U[0] = double((ui + uwx) * iw); U[1] = double((vi + uwy) * iw); U[2] = double((wi + uwz) * iw);
    } else {
      U[0] = U[1] = U[2] = 0.0;
    }
  };
  auto measure = [&](int r) {
    double q = 0.0;
    if (have) {
      double U[3];
      interp_corr_reg(U);
      const double e0 = U[0] * a.vs - vx, e1 = U[1] * a.vs - vy, e2 = U[2] * a.vs - vz;
      q = e0 * e0 + e1 * e1 + e2 * e2;
    }
    if (lane == 0) { bsum[warp][0] = q; bsum[warp][1] = have ? 1.0 : 0.0; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0, mx = 0.0;
      int cnt = 0;
      for (int w = 0; w < nwarp; w++) {
        if (bsum[w][1] == 0.0) continue;
        sum += bsum[w][0];
        mx = fmax(mx, sqrt(bsum[w][0]));
        cnt++;
      }
      if (cnt) {
        const int sl = blockIdx.x & (kSlipSlots - 1);
        atomicAdd(&P.ps->s2[r][sl], sum);
        atomicMax(&P.ps->max_bits[r][sl], (unsigned long long)__double_as_longlong(mx));
        atomicAdd(&P.ps->count[r][sl], cnt);
      }
    }
    __syncthreads();
  };
  spread(F0, F1, F2);
  // a launch with nothing after the first pass that reads the force field
  // (no check, no correction, no slip statistics) needs no grid barrier
  const bool more = P.check_first || P.ncorr > 0 || P.measure_last;
  if (more && !grid_barrier(P.ps, P.status, P.spin)) return;
  if (P.check_first) {
    measure(0);
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
    const bool fall = slip_rms(P.ps, 0) > P.slip_tol;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      P.ps->checked = 1;
      if (P.status) atomicAdd(P.status + kStSlipChecks, 1);
      if (fall) {
        P.ps->fell_back = 1;
        if (P.status) atomicAdd(P.status + kStFallbacks, 1);
      }
    }
    if (!fall) {
      if (P.rows && have) record_marker<L, S>(P, mk, lane);
      return;
    }
  }
  for (int it = 0; it < P.ncorr; it++) {
    double d0 = 0, d1 = 0, d2 = 0;
    if (have) {
      double U[3];
      interp_corr_reg(U);
      d0 = mxi * (U[0] * a.vs - vx);
      d1 = mxi * (U[1] * a.vs - vy);
      d2 = mxi * (U[2] * a.vs - vz);
      c0 += d0; c1 += d1; c2 += d2;
      if (lane == 0) {
        a.fout[3 * mk] += d0; a.fout[3 * mk + 1] += d1; a.fout[3 * mk + 2] += d2;
      }
    }
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
    spread(d0, d1, d2);
    if (!grid_barrier(P.ps, P.status, P.spin)) return;
  }
  if (have && lane == 0) { a.corr[3 * mk] = c0; a.corr[3 * mk + 1] = c1; a.corr[3 * mk + 2] = c2; }
  if (P.measure_last) measure(1);
  if (P.rows && have) {
    __syncwarp();
    record_marker<L, S>(P, mk, lane);
  }
}

}  // namespace couplb
