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
//
// Fluid velocities are not computed for the whole grid.  The reference
// refreshes the moments of every node once per LB cycle
// (compute_macroscopic(false), fix_couplb.cpp:757-760); the populations do
// not change within the cycle, so the velocity of a node is a pure function of
// them.  At the refresh, k_ibm_prefetch computes (arithmetic of k_macro) the
// velocities of each marker's stencil into a contiguous per-marker record;
// the sub-steps of the cycle read the record and compute directly only the
// stencils of markers that moved to another cell.
#pragma once
#include "lbm_kernels.cuh"
#include "mlp_kernels.cuh"

namespace couplb {

// delta_roma (couplb_ibm.h:11-22).  Both branches of the reference are
// formed and one is selected (no divergence between the lanes of a warp); the
// arithmetic of each branch is the reference's.
template <class R>
__device__ __forceinline__ R delta_roma(R r) {
  const R ar = fabs(r);
  const bool inner = ar <= R(0.5);
  const R a = inner ? R(1) - R(3) * r * r : R(-2) + R(6) * ar - R(3) * r * r;
  const R sq = sqrt(a > R(0) ? a : R(0));
  const R num = inner ? R(1) + sq : R(5) - R(3) * ar - sq;
  const R v = num / (inner ? R(3) : R(6));
  return ar <= R(1.5) ? v : R(0);
}

// delta_peskin4 (couplb_ibm.h:24-35), branch-free like delta_roma
template <class R>
__device__ __forceinline__ R delta_peskin4(R r) {
  const R ar = fabs(r);
  const bool inner = ar <= R(1);
  const R a = inner ? R(1) + R(4) * ar - R(4) * ar * ar : R(-7) + R(12) * ar - R(4) * ar * ar;
  const R sq = sqrt(a > R(0) ? a : R(0));
  const R v = (inner ? R(3) - R(2) * ar + sq : R(5) - R(2) * ar - sq) / R(8);
  return ar <= R(2) ? v : R(0);
}

template <int DELTA, class R>
__device__ __forceinline__ R delta1(R r) {
  return DELTA == 0 ? delta_roma<R>(r) : delta_peskin4<R>(r);
}

// Accumulators of the total spread force, each 4 doubles (32 B) apart.
constexpr int kFtotSlots = 64;

// Key of a stencil velocity record (see k_ibm_prefetch).
struct StencilKey {
  int i0, j0, k0;
  unsigned epoch;
};

template <class S>
struct IbmArgs {
  Geom g;
  // populations of the current state and how to read them
  const typename S::T* __restrict__ fin;
  const typename S::A* __restrict__ rho_field;
  int pull;                               // 1: post-collision store (pull), 0: post-stream
  // dense moment arrays, used when they hold this state everywhere
  const typename S::A* cux;
  const typename S::A* cuy;
  const typename S::A* cuz;
  int all_valid;
  const typename S::A* crho;              // with all_valid: density (deviation if shifted)
  // stencil velocity records, one per marker slot (64 x {ux, uy, uz, rho})
  typename S::A* sbuf;
  StencilKey* skey;
  unsigned cur_epoch;
  typename S::A* F;                       // Eulerian force field {fx,fy,fz,0} per node
  unsigned char* seg_force;               // per 8 nodes (n >> 3): a force was spread there
  int n;
  const double* __restrict__ x;           // n*3, MD units
  const double* __restrict__ v;           // n*3
  const double* __restrict__ m;           // n
  const int* __restrict__ active;         // n or null
  double* fout;                           // n*3 marker forces
  int accumulate;                         // 1: fout += F, 0: fout = F (0 for inactive)
  double* ftot;                           // [kFtotSlots][4] FP64 sums of the spread grid force
  double lo[3];
  int off[3];
  double inv_dx, xi_over_dt, inv_N, vs, fs, dvr;
  double spread_c;                        // inv_N / fs: marker force -> spread force
  // forcing methods beyond the single pass (null / unused otherwise)
  double* corr;                           // n*3: correction beyond the penalty pass
  const MlpPacked* mlp;                   // learned correction network
  int wrap;                               // window axes wrapped periodically (bit d: axis d)
  // Slab decomposition along z (couplb_ibm_halo_attach): window planes beyond
  // a z face bound to a neighbour subdomain, zplanes[side] of them (0: the
  // face is not bound; side 0: the plane below the low face, side 1: up to
  // two planes above the high face).  vh: their velocities and densities
  // {ux, uy, uz, rho} as compute_velocity gives them, computed by the
  // neighbour (k_halo_moments); fh: the forces this lattice spreads onto them
  // {fx, fy, fz, 0}, which the neighbour adds to its own field
  // (k_halo_fold).  4 values per node, plane-major.
  const typename S::A* vh[2];
  typename S::A* fh[2];
  int zplanes[2];
  // order in which k_ibm_prefetch (and k_ibm_substep8, when given one) visit
  // the markers: a permutation of 0..n-1 (k_order_*), or null for the index
  // order.  The engine passes it to the refresh only.
  const int* order = nullptr;
};

// Halo plane of the ghost-inclusive z index kg (0: the plane below the low
// face, 1 and 2: the planes above the high face), or -1.
template <class S>
__device__ __forceinline__ int z_halo_plane(const IbmArgs<S>& a, int kg) {
  if (a.zplanes[0] && kg == 0) return 0;
  if (a.zplanes[1] && kg > a.g.nz && kg <= a.g.nz + a.zplanes[1]) return kg - a.g.nz;
  return -1;
}

// Offset (in values) of node (i, j) of halo plane hp in its side's buffer.
__device__ __forceinline__ size_t z_halo_offset(const Geom& g, int hp, int i, int j) {
  return 4 * ((size_t)(hp > 0 ? hp - 1 : 0) * g.nx * g.ny + (size_t)i + (size_t)g.nx * j);
}

// The marker window of the reference is [i0-1, i0+2] per axis clipped to the
// ghost-inclusive box (couplb_ibm.h:64-73, 110-115): near a high periodic face
// a marker loses the plane beyond the ghost layer.  With the "ibm_window wrap"
// option an axis whose two faces are periodic is wrapped instead: the window
// index maps to its interior image, so every node of the window takes part.
// Returns the ghost-inclusive index of that image (1..n).
__device__ __forceinline__ int wrap_ghost_index(int ig, int n) {
  int i = (ig - 1) % n;
  if (i < 0) i += n;
  return i + 1;
}

// Add a spread force to one node of the interleaved force field: one vector
// atomic (16 B, sm_90+) for FP32; three FP64 atomics otherwise.
__device__ __forceinline__ void spread_add(float* p, float a, float b, float c) {
  atomicAdd(reinterpret_cast<float4*>(p), make_float4(a, b, c, 0.f));
}
__device__ __forceinline__ void spread_add(float* p, double a, double b, double c) {
  atomicAdd(reinterpret_cast<float4*>(p), make_float4(float(a), float(b), float(c), 0.f));
}
__device__ __forceinline__ void spread_add(double* p, double a, double b, double c) {
  atomicAdd(p, a);
  atomicAdd(p + 1, b);
  atomicAdd(p + 2, c);
}

// Ghost-inclusive node (ig, jg, kg) -> -1 and the interior coordinates of the
// node or of its periodic image, or the wall type (1..4).
__device__ __forceinline__ int classify_node(const Geom& g, int D, int ig, int jg, int kg, int& i,
                                             int& j, int& k) {
  const int gx = g.nx + 2, gy = g.ny + 2, gz = (D == 3) ? g.nz + 2 : 1;
  int t = 0;
  const bool ox = ig == 0 || ig == gx - 1;
  const bool oy = jg == 0 || jg == gy - 1;
  const bool oz = (D == 3) && (kg == 0 || kg == gz - 1);
  if (ox) { const int ft = ig == 0 ? g.face[0] : g.face[1]; if (ft) t = ft; }
  if (oy) { const int ft = jg == 0 ? g.face[2] : g.face[3]; if (ft) t = ft; }
  if (oz) { const int ft = kg == 0 ? g.face[4] : g.face[5]; if (ft) t = ft; }
  if (t) return t;
  i = ig - 1; j = jg - 1; k = (D == 3) ? kg - 1 : 0;
  i = i < 0 ? g.nx - 1 : (i >= g.nx ? 0 : i);
  j = j < 0 ? g.ny - 1 : (j >= g.ny ? 0 : j);
  if (D == 3) k = k < 0 ? g.nz - 1 : (k >= g.nz ? 0 : k);
  return -1;
}

// The window nodes of one lane: s = lane and s = lane + 32 of the 4^D window
// (3D; s = lane < 16 in 2D).  Both share the x offset lane & 3 and the y
// offset (lane >> 2) & 3 and differ only in z, so the x/y part of the
// classification is done once.  The 1D weights of the window's 4 offsets per
// axis are evaluated once per warp (lane t < 4 D: offset t & 3 of axis t >> 2)
// and fetched with shuffles; a node's weight is (wx * wy) * wz as in
// IBM::interpolate / spread (couplb_ibm.h:68-86, 110-123).  All 32 lanes of
// the warp must call it.
template <class R>
struct LaneNodes {
  int t[2];          // -2 outside the ghost-inclusive box, -1 fluid, else wall type
  long long n[2];    // interior index of a fluid node (or of its periodic image)
  R d[2];            // weight
  int i, j, k[2];    // interior coordinates of a fluid node
  int h[2];          // z halo plane of a fluid node beyond a bound face (z_halo_plane), or -1
};

template <class L, int DELTA, class R>
__device__ __forceinline__ LaneNodes<R> lane_nodes(const Geom& g, double lx, double ly, double lz,
                                                   int i0, int j0, int k0, int lane, int wrap,
                                                   const int* zplanes = nullptr) {
  R w1 = R(0);
  {
    const int ax = lane >> 2, o = lane & 3;
    if (ax < L::D) {
      const double l = ax == 0 ? lx : (ax == 1 ? ly : lz);
      const int b = ax == 0 ? i0 : (ax == 1 ? j0 : k0);
      w1 = delta1<DELTA, R>(R(l - (b - 1 + o)));
    }
  }
  const int sx = lane & 3, sy = (lane >> 2) & 3;
  const R wx = __shfl_sync(0xffffffffu, w1, sx);
  const R wy = __shfl_sync(0xffffffffu, w1, 4 + sy);
  const R wxy = wx * wy;
  const int gx = g.nx + 2, gy = g.ny + 2;
  int ig = i0 - 1 + sx, jg = j0 - 1 + sy;
  if (wrap & 1) ig = wrap_ghost_index(ig, g.nx);
  if (wrap & 2) jg = wrap_ghost_index(jg, g.ny);
  const bool inxy = ig >= 0 && ig < gx && jg >= 0 && jg < gy;
  // classify_node, x then y (a later axis overrides)
  int txy = 0;
  if (ig == 0 || ig == gx - 1) { const int ft = ig == 0 ? g.face[0] : g.face[1]; if (ft) txy = ft; }
  if (jg == 0 || jg == gy - 1) { const int ft = jg == 0 ? g.face[2] : g.face[3]; if (ft) txy = ft; }
  int ii = ig - 1, jj = jg - 1;
  ii = ii < 0 ? g.nx - 1 : (ii >= g.nx ? 0 : ii);
  jj = jj < 0 ? g.ny - 1 : (jj >= g.ny ? 0 : jj);
  const long long nxy = (long long)ii + (long long)g.nx * jj;
  LaneNodes<R> out;
  out.i = ii;
  out.j = jj;
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    out.t[rep] = -2;
    out.n[rep] = -1;
    out.d[rep] = R(0);
    out.k[rep] = 0;
    out.h[rep] = -1;
  }
  if (L::D == 2) {
    if (lane < 16 && inxy) {
      out.t[0] = txy ? txy : -1;
      out.n[0] = nxy;
      out.d[0] = wxy;
    }
    return out;
  }
  const int gz = g.nz + 2;
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int oz = (lane >> 4) + 2 * rep;
    const R wz = __shfl_sync(0xffffffffu, w1, 8 + oz);
    int kg = k0 - 1 + oz;
    if (wrap & 4) kg = wrap_ghost_index(kg, g.nz);
    if (zplanes && inxy) {
      // a plane of the neighbour beyond a bound face: its x/y walls only
      const int hp = (zplanes[0] && kg == 0) ? 0
                   : ((zplanes[1] && kg > g.nz && kg <= g.nz + zplanes[1]) ? kg - g.nz : -1);
      if (hp >= 0) {
        out.t[rep] = txy ? txy : -1;
        out.d[rep] = wxy * wz;
        out.h[rep] = hp;
        continue;
      }
    }
    if (!inxy || kg < 0 || kg >= gz) continue;
    int t = txy;
    if (kg == 0 || kg == gz - 1) { const int ft = kg == 0 ? g.face[4] : g.face[5]; if (ft) t = ft; }
    int kk = kg - 1;
    kk = kk < 0 ? g.nz - 1 : (kk >= g.nz ? 0 : kk);
    out.t[rep] = t ? t : -1;
    out.n[rep] = nxy + (long long)g.nx * g.ny * kk;
    out.d[rep] = wxy * wz;
    out.k[rep] = kk;
  }
  return out;
}

// Velocity of interior node (i,j,k) = n of the post-stream state, with the
// arithmetic of k_macro (compute_macroscopic(false), couplb_lattice.h:155-202).
template <class L, class S>
__device__ __forceinline__ void compute_velocity(const IbmArgs<S>& a, int i, int j, int k, size_t n,
                                                 typename S::A& v0, typename S::A& v1,
                                                 typename S::A& v2, typename S::A& vr) {
  using C = typename S::C;
  C f[L::Q];
  if (a.pull) load_node<L, S, size_t, true>(a.g, a.fin, a.rho_field, i, j, k, n, f);
  else load_node<L, S, size_t, false>(a.g, a.fin, a.rho_field, i, j, k, n, f);
  C r, jx, jy, jz;
  moments<L, C>(f, r, jx, jy, jz);
  C rho = S::kShift ? C(a.g.rho0) + r : r;
  if (rho <= C(RHO_MIN) || !isfinite(rho)) rho = C(RHO_MIN);
  const C inv_r = C(1) / rho;
  v0 = typename S::A(jx * inv_r);
  v1 = typename S::A(jy * inv_r);
  v2 = typename S::A(jz * inv_r);
  vr = typename S::A(rho);
}

// Stencil velocity cache: one record per marker slot holding the velocities of
// the 4^D nodes of a stencil whose base cell is (i0, j0, k0), valid for one
// population state (epoch).  The velocities depend only on the base cell and
// the state, so a record serves any marker whose stencil has that base; a
// marker that moved to another cell since the refresh (or a slot filled by a
// different atom) misses and computes its nodes directly.  Records are
// contiguous (64 x 3 values), so a sub-step reads its marker's stencil as a
// few full cache lines that stay in L2 across the sub-steps of a cycle.  The
// density (kept for the corrected velocity of the iterative passes) follows
// the three velocity components.
constexpr int kRecStride = 64 * 4;
template <class S>
__device__ __forceinline__ typename S::A* stencil_record(const IbmArgs<S>& a, int mk) {
  return a.sbuf + (size_t)mk * kRecStride;
}

// Refresh prefetch of marker mk by one warp: fills its slot's record and key.
template <class L, class S>
__device__ __forceinline__ void prefetch_marker(const IbmArgs<S>& a, int mk, int lane, unsigned epoch) {
  const Geom& g = a.g;
  const double lx = (a.x[3 * mk] - a.lo[0]) * a.inv_dx - a.off[0] + 1.0;
  const double ly = (a.x[3 * mk + 1] - a.lo[1]) * a.inv_dx - a.off[1] + 1.0;
  const double lz = (L::D == 3) ? ((a.x[3 * mk + 2] - a.lo[2]) * a.inv_dx - a.off[2] + 1.0) : 0.0;
  const int i0 = (int)floor(lx), j0 = (int)floor(ly);
  const int k0 = (L::D == 3) ? (int)floor(lz) : 0;
  const int gx = g.nx + 2, gy = g.ny + 2, gz = (L::D == 3) ? g.nz + 2 : 1;
  constexpr int NS = (L::D == 3) ? 64 : 16;
  typename S::A* rec = stencil_record(a, mk);
  // both nodes are computed before either is stored, so that their loads can
  // be in flight together
  typename S::A v[2][4] = {{0, 0, 0, 1}, {0, 0, 0, 1}};
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int s = lane + 32 * rep;
    if (s >= NS) break;
    int ig = i0 - 1 + (s & 3);
    int jg = j0 - 1 + ((s >> 2) & 3);
    int kg = (L::D == 3) ? k0 - 1 + (s >> 4) : 0;
    if (a.wrap & 1) ig = wrap_ghost_index(ig, g.nx);
    if (a.wrap & 2) jg = wrap_ghost_index(jg, g.ny);
    if (a.wrap & 4) kg = wrap_ghost_index(kg, g.nz);
    int ii = 0, jj = 0, kk = 0;
    const int hp = (L::D == 3) ? z_halo_plane(a, kg) : -1;
    if (hp >= 0) {
      // the neighbour's node: x/y classification only, moments from the halo
      if (ig >= 0 && ig < gx && jg >= 0 && jg < gy && classify_node(g, L::D, ig, jg, 1, ii, jj, kk) < 0) {
        const typename S::A* m = a.vh[hp ? 1 : 0] + z_halo_offset(g, hp, ii, jj);
        v[rep][0] = m[0]; v[rep][1] = m[1]; v[rep][2] = m[2]; v[rep][3] = m[3];
      }
    } else if (ig >= 0 && ig < gx && jg >= 0 && jg < gy && kg >= 0 && kg < gz &&
               classify_node(g, L::D, ig, jg, kg, ii, jj, kk) < 0) {
      const size_t n = (size_t)ii + (size_t)g.nx * ((size_t)jj + (size_t)g.ny * kk);
      compute_velocity<L, S>(a, ii, jj, kk, n, v[rep][0], v[rep][1], v[rep][2], v[rep][3]);
    }
  }
#pragma unroll
  for (int rep = 0; rep < 2; rep++) {
    const int s = lane + 32 * rep;
    if (s >= NS) break;
    rec[s] = v[rep][0]; rec[64 + s] = v[rep][1]; rec[128 + s] = v[rep][2]; rec[192 + s] = v[rep][3];
  }
  if (lane == 0) a.skey[mk] = StencilKey{i0, j0, k0, epoch};
}

// Refresh prefetch: one warp per active marker fills its slot's record.
template <class L, class S>
__global__ void __launch_bounds__(256) k_ibm_prefetch(const IbmArgs<S> a) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= a.n) return;
  const int mk = a.order ? a.order[w] : w;
  if (a.active && !a.active[mk]) return;
  prefetch_marker<L, S>(a, mk, lane, a.cur_epoch);
}

// Processing order of the refresh: the markers grouped by bands of
// kOrderPlanes z planes of their cell (y rows in 2D), so that markers whose
// windows share population lines run close together in time and find them
// in L2.  Bands rather than single planes keep runs of markers that the
// caller holds in chain order (rods) together, as far as the atomic ranks
// below follow the index order within a warp.  Every marker is still
// handled once by its own lanes, so the records do not depend on the order.
// A counting sort in three launches: band sizes with each marker's rank in
// its band, the band offsets, the scatter.
constexpr int kOrderPlanes = 8;

template <class L, class S>
__device__ __forceinline__ int order_bucket(const IbmArgs<S>& a, int mk, int nb) {
  constexpr int d = (L::D == 3) ? 2 : 1;
  const double l = ((a.x[3 * mk + d] - a.lo[d]) * a.inv_dx - a.off[d]) * (1.0 / kOrderPlanes);
  int b = 0;   // below the lattice, and NaN: band 0
  if (l >= 0.0) b = l < (double)nb ? (int)l : nb - 1;
  return b;
}

// count[nb] collects the markers whose successor lies within 2 cells on
// every axis: when that is most of them, the caller already keeps the
// markers in a spatial or chain order and the scatter keeps the index order.
template <class L, class S>
__global__ void k_order_count(const IbmArgs<S> a, int nb, int* __restrict__ count, int* __restrict__ rank) {
  const int mk = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool in = mk < a.n;
  const int b = in ? order_bucket<L, S>(a, mk, nb) : -1;
  // one atomic per band and warp (markers in chain order share a few bands,
  // and same-address atomics queue in L2); ranks follow the lane order
  const unsigned peers = __match_any_sync(0xffffffffu, b);
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (in && lane == leader) base = atomicAdd(count + b, __popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  bool near = false;
  if (in) {
    rank[mk] = base + __popc(peers & ((1u << lane) - 1u));
    if (mk + 1 < a.n) {
      near = true;
#pragma unroll
      for (int d = 0; d < L::D; d++) near = near && fabs(a.x[3 * (mk + 1) + d] - a.x[3 * mk + d]) * a.inv_dx < 2.0;
    }
  }
  const unsigned nn = __ballot_sync(0xffffffffu, near);
  if ((threadIdx.x & 31) == 0 && nn) atomicAdd(count + nb, __popc(nn));
}

// Exclusive prefix sum of the nb bucket sizes, in place; one block of 256.
static __global__ void __launch_bounds__(256) k_order_scan(int nb, int* __restrict__ count) {
  __shared__ int part[256];
  const int t = threadIdx.x;
  const int per = (nb + 255) / 256;
  const int lo = min(nb, t * per), hi = min(nb, lo + per);
  int sum = 0;
  for (int b = lo; b < hi; b++) sum += count[b];
  part[t] = sum;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int i = 0; i < 256; i++) {
      const int c = part[i];
      part[i] = run;
      run += c;
    }
  }
  __syncthreads();
  int run = part[t];
  for (int b = lo; b < hi; b++) {
    const int c = count[b];
    count[b] = run;
    run += c;
  }
}

template <class L, class S>
__global__ void k_order_scatter(const IbmArgs<S> a, int nb, const int* __restrict__ start,
                                const int* __restrict__ rank, int* __restrict__ order) {
  const int mk = blockIdx.x * blockDim.x + threadIdx.x;
  if (mk >= a.n) return;
  if (2LL * start[nb] > a.n) order[mk] = mk;   // mostly near neighbours: index order
  else order[start[order_bucket<L, S>(a, mk, nb)] + rank[mk]] = mk;
}

// Velocity of stencil slot s of marker mk (node (i,j,k) = n).
template <class L, class S>
__device__ __forceinline__ void node_velocity(const IbmArgs<S>& a, bool hit,
                                              const typename S::A* rec, int s, int i, int j,
                                              int k, size_t n, double& u0, double& u1, double& u2) {
  if (a.all_valid) {
    u0 = double(a.cux[n]); u1 = double(a.cuy[n]); u2 = double(a.cuz[n]);
  } else if (hit) {
    u0 = double(rec[s]); u1 = double(rec[64 + s]); u2 = double(rec[128 + s]);
  } else {
    typename S::A v0, v1, v2, vr;
    compute_velocity<L, S>(a, i, j, k, n, v0, v1, v2, vr);
    u0 = double(v0); u1 = double(v1); u2 = double(v2);
  }
}

// Velocity and density of stencil slot s (the iterative passes).
template <class L, class S>
__device__ __forceinline__ void node_state(const IbmArgs<S>& a, bool hit, const typename S::A* rec,
                                           int s, int i, int j, int k, size_t n, double& u0,
                                           double& u1, double& u2, double& rho) {
  if (a.all_valid) {
    u0 = double(a.cux[n]); u1 = double(a.cuy[n]); u2 = double(a.cuz[n]);
    rho = S::kShift ? a.g.rho0 + double(a.crho[n]) : double(a.crho[n]);
  } else if (hit) {
    u0 = double(rec[s]); u1 = double(rec[64 + s]); u2 = double(rec[128 + s]);
    rho = double(rec[192 + s]);
  } else {
    typename S::A v0, v1, v2, vr;
    compute_velocity<L, S>(a, i, j, k, n, v0, v1, v2, vr);
    u0 = double(v0); u1 = double(v1); u2 = double(v2); rho = double(vr);
  }
}

// Weight arithmetic, interpolation sums, their warp reductions and the spread
// weights in the storage's compute type: FP64 for the parity form, FP32 for
// the shifted forms (their populations and moments are FP32).  Positions,
// the penalty force and the total-force accumulators are FP64 in both.
//
// LEARNED (D3Q19): the lanes also gather the network input (u0 at the 27
// nodes round(l)-1..round(l)+1 of each axis, then v / vel_scale) into the
// warp's shared scratch xs, the warp runs the correction network, and the
// marker force F = F_penalty + m xi/dt vs y is returned and spread.
//
// FILL: the stencil velocities are computed from the populations and written
// to the marker's record (the work of k_ibm_prefetch, fused).
// HALO: the lattice may have z faces bound to neighbour slabs (false for the
// method kernels, which refuse them: the halo branches compile out).
template <class L, class S, int DELTA, bool LEARNED, bool HALO = true>
__device__ __forceinline__ void ibm_substep_body(const IbmArgs<S>& a, int mk, int lane, bool fill,
                                                 const MlpPacked* P, MlpBlockScratch* blk,
                                                 double* tot3 = nullptr) {
  using R = typename S::C;
  // LEARNED: the 8 warps of the block run the network together (one call of
  // mlp_block_forward per warp), so a warp without a marker still takes part
  const bool valid = mk < a.n && !(a.active && !a.active[mk]);
  if (mk < a.n && !valid && !a.accumulate && lane < 3) a.fout[3 * mk + lane] = 0.0;
  if (!LEARNED && !valid) return;
  float* xs = LEARNED ? blk->x + (threadIdx.x >> 5) * kMlpXStride : nullptr;
  if (LEARNED) {
    for (int t = lane; t < kMlpXStride; t += 32) xs[t] = 0.f;
    __syncwarp();
  }
  const Geom& g = a.g;
  constexpr int NS = (L::D == 3) ? 64 : 16;
  double F0 = 0, F1 = 0, F2 = 0, mass = 0, vmk0 = 0, vmk1 = 0, vmk2 = 0;
  // fluid nodes of this lane: their force entries (interior node or z halo)
  // and segment (-1 for a halo node)
  typename S::A* sp0 = nullptr;
  typename S::A* sp1 = nullptr;
  long long sg0 = -1, sg1 = -1;
  R sd0 = 0, sd1 = 0, wss = 0;
  if (valid) {
    const double xp = a.x[3 * mk], yp = a.x[3 * mk + 1], zp = a.x[3 * mk + 2];
    // IBM::phys_to_local (couplb_ibm.h:49-55)
    const double lx = (xp - a.lo[0]) * a.inv_dx - a.off[0] + 1.0;
    const double ly = (yp - a.lo[1]) * a.inv_dx - a.off[1] + 1.0;
    const double lz = (L::D == 3) ? ((zp - a.lo[2]) * a.inv_dx - a.off[2] + 1.0) : 0.0;
    const int i0 = (int)floor(lx), j0 = (int)floor(ly);
    const int k0 = (L::D == 3) ? (int)floor(lz) : 0;
    // first node of the 27-node network window, in window coordinates
    int ox = 0, oy = 0, oz = 0;
    if (LEARNED) {
      ox = (lx - i0) >= 0.5 ? 1 : 0;
      oy = (ly - j0) >= 0.5 ? 1 : 0;
      oz = (lz - k0) >= 0.5 ? 1 : 0;
    }
    R ui = 0, vi = 0, wi = 0, ws = 0;
    const StencilKey key = a.skey[mk];
    typename S::A* rec = stencil_record(a, mk);
    // The record entries, the marker's velocity and mass are loaded before the
    // key is compared (their addresses do not depend on it), so that their
    // latencies overlap; a miss discards the record values.
    const bool spec = !fill && !a.all_valid;
    typename S::A pre[2][3] = {{0, 0, 0}, {0, 0, 0}};
    if (spec) {
#pragma unroll
      for (int rep = 0; rep < 2; rep++) {
        const int s = lane + 32 * rep;
        if (s < NS) { pre[rep][0] = rec[s]; pre[rep][1] = rec[64 + s]; pre[rep][2] = rec[128 + s]; }
      }
    }
    mass = a.m[mk];
    vmk0 = a.v[3 * mk]; vmk1 = a.v[3 * mk + 1]; vmk2 = a.v[3 * mk + 2];
    const bool hit = key.epoch == a.cur_epoch && key.i0 == i0 && key.j0 == j0 && key.k0 == k0;
    const LaneNodes<R> ln = lane_nodes<L, DELTA, R>(g, lx, ly, lz, i0, j0, k0, lane, a.wrap,
                                                    HALO ? a.zplanes : nullptr);
    bool wall_seen = false;   // a wall node adds to ws but not to wss
#pragma unroll
    for (int rep = 0; rep < 2; rep++) {
      const int s = lane + 32 * rep;
      if (s >= NS) break;
      const int t = ln.t[rep];
      if (t == -2) continue;
      const R dd = ln.d[rep];
      // slot of this node in the network input, or -1
      int p = -1;
      if (LEARNED) {
        const int rx = (s & 3) - ox, ry = ((s >> 2) & 3) - oy, rz = (s >> 4) - oz;
        if (rx >= 0 && rx < 3 && ry >= 0 && ry < 3 && rz >= 0 && rz < 3) p = rx + 3 * ry + 9 * rz;
      }
      if (t < 0) {
        const int hp = HALO ? ln.h[rep] : -1;
        const size_t src = hp >= 0 ? 0 : (size_t)ln.n[rep];
        const int ii = ln.i, jj = ln.j, kk = ln.k[rep];
        R u0, u1, u2;
        if (hp >= 0 && !(spec && hit)) {
          // a node of the neighbour beyond a bound z face: its moments
          const typename S::A* m = a.vh[hp ? 1 : 0] + z_halo_offset(g, hp, ii, jj);
          if (fill) { rec[s] = m[0]; rec[64 + s] = m[1]; rec[128 + s] = m[2]; rec[192 + s] = m[3]; }
          u0 = R(m[0]); u1 = R(m[1]); u2 = R(m[2]);
        } else if (fill) {
          typename S::A v0, v1, v2, vr;
          compute_velocity<L, S>(a, ii, jj, kk, src, v0, v1, v2, vr);
          rec[s] = v0; rec[64 + s] = v1; rec[128 + s] = v2; rec[192 + s] = vr;
          u0 = R(v0); u1 = R(v1); u2 = R(v2);
        } else if (spec && hit) {
          u0 = R(pre[rep][0]); u1 = R(pre[rep][1]); u2 = R(pre[rep][2]);
        } else {
          double w0, w1, w2;
          node_velocity<L, S>(a, hit, rec, s, ii, jj, kk, src, w0, w1, w2);
          u0 = R(w0); u1 = R(w1); u2 = R(w2);
        }
        ui += u0 * dd;
        vi += u1 * dd;
        wi += u2 * dd;
        ws += dd;
        wss += dd;
        typename S::A* tgt = hp >= 0 ? a.fh[hp ? 1 : 0] + z_halo_offset(g, hp, ii, jj) : a.F + 4 * src;
        const long long seg = hp >= 0 ? -1 : (long long)(src >> 3);
        if (rep == 0) { sp0 = tgt; sg0 = seg; sd0 = dd; }
        else { sp1 = tgt; sg1 = seg; sd1 = dd; }
        if (LEARNED && p >= 0) { xs[3 * p] = float(u0); xs[3 * p + 1] = float(u1); xs[3 * p + 2] = float(u2); }
      } else if (t == 1 || t == 3) {
        ws += dd;
        wall_seen = true;
      } else if (t == 2) {
        ui += R(g.uw[0]) * dd;
        vi += R(g.uw[1]) * dd;
        wi += R(L::D == 3 ? g.uw[2] : 0.0) * dd;
        ws += dd;
        wall_seen = true;
        if (LEARNED && p >= 0) {
          xs[3 * p] = float(g.uw[0]); xs[3 * p + 1] = float(g.uw[1]); xs[3 * p + 2] = float(g.uw[2]);
        }
      }
    }
    if (fill && lane == 0) a.skey[mk] = StencilKey{i0, j0, k0, a.cur_epoch};
    // without wall nodes in the window ws and wss are the same sums
    const bool walls = __any_sync(0xffffffffu, wall_seen);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ui += __shfl_xor_sync(0xffffffffu, ui, o);
      vi += __shfl_xor_sync(0xffffffffu, vi, o);
      wi += __shfl_xor_sync(0xffffffffu, wi, o);
      ws += __shfl_xor_sync(0xffffffffu, ws, o);
    }
    if (walls) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) wss += __shfl_xor_sync(0xffffffffu, wss, o);
    } else {
      wss = ws;
    }
    double u0 = 0, u1 = 0, u2 = 0;
    if (ws > R(DELTA_TOL)) {
      const R iw = R(1) / ws;
      u0 = double(ui * iw); u1 = double(vi * iw); u2 = double(wi * iw);
    }
    // penalty force (fix_couplb.cpp:777-781)
    F0 = mass * a.xi_over_dt * (u0 * a.vs - vmk0);
    F1 = mass * a.xi_over_dt * (u1 * a.vs - vmk1);
    F2 = mass * a.xi_over_dt * (u2 * a.vs - vmk2);
  }
  if constexpr (LEARNED) {
    if (valid && lane < 3) xs[81 + lane] = float((lane == 0 ? vmk0 : (lane == 1 ? vmk1 : vmk2)) / a.vs);
    __syncwarp();
    float y[3];
    mlp_block_forward<false>(*P, *blk, threadIdx.x >> 5, lane, y);
    if (!valid) return;
    const double sc = mass * a.xi_over_dt * a.vs;
    const double c0 = sc * double(y[0]), c1 = sc * double(y[1]), c2 = sc * double(y[2]);
    F0 += c0; F1 += c1; F2 += c2;
    if (lane == 0 && a.corr) { a.corr[3 * mk] = c0; a.corr[3 * mk + 1] = c1; a.corr[3 * mk + 2] = c2; }
  } else if (lane == 0 && a.corr) {
    a.corr[3 * mk] = 0.0; a.corr[3 * mk + 1] = 0.0; a.corr[3 * mk + 2] = 0.0;
  }
  if (lane == 0) {
    if (a.accumulate) {
      a.fout[3 * mk] += F0; a.fout[3 * mk + 1] += F1; a.fout[3 * mk + 2] += F2;
    } else {
      a.fout[3 * mk] = F0; a.fout[3 * mk + 1] = F1; a.fout[3 * mk + 2] = F2;
    }
  }
  // spread -F/(N * force_scale) (fix_couplb.cpp:788-792, couplb_ibm.h:124-132)
  if (wss < R(DELTA_TOL)) return;
  const R sc = R(a.dvr) / wss;
  const double fl0 = -F0 * a.spread_c, fl1 = -F1 * a.spread_c, fl2 = -F2 * a.spread_c;
  const R f0 = R(fl0), f1 = R(fl1), f2 = R(fl2);
  if (sp0) {
    const R w = sd0 * sc;   // couplb_ibm.h:128
    spread_add(sp0, f0 * w, f1 * w, f2 * w);
    if (a.seg_force && sg0 >= 0) a.seg_force[sg0] = 1;
  }
  if (sp1) {
    const R w = sd1 * sc;
    spread_add(sp1, f0 * w, f1 * w, f2 * w);
    if (a.seg_force && sg1 >= 0) a.seg_force[sg1] = 1;
  }
  if (lane == 0 && tot3) {
    // the caller sums the markers of its block before one atomic each
    tot3[0] = fl0 * a.dvr;
    tot3[1] = fl1 * a.dvr;
    tot3[2] = fl2 * a.dvr;
  } else if (lane == 0 && a.ftot) {
    // one of kFtotSlots accumulators (32 B apart) by marker index: the
    // same-address FP64 atomics of all markers would serialise in L2
    double* t = a.ftot + 4 * (mk & (kFtotSlots - 1));
    atomicAdd(t, fl0 * a.dvr);
    atomicAdd(t + 1, fl1 * a.dvr);
    atomicAdd(t + 2, fl2 * a.dvr);
  }
}

// One sub-step, one warp per marker.  The total spread force of the block's
// markers is summed in shared memory and added to accumulator slot
// blockIdx % kFtotSlots with three FP64 atomics per block: with a few
// thousand blocks per launch, per-marker atomics on the 64 slots queued in
// L2 and took about as long as the rest of the sub-step (2e5 markers).
template <class L, class S, int DELTA>
__global__ void __launch_bounds__(256) k_ibm_substep(const IbmArgs<S> a) {
  __shared__ double part[8][3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double t3[3] = {0.0, 0.0, 0.0};
  ibm_substep_body<L, S, DELTA, false>(a, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane, false,
                                       nullptr, nullptr, t3);
  if (!a.ftot) return;
  if (lane == 0) { part[warp][0] = t3[0]; part[warp][1] = t3[1]; part[warp][2] = t3[2]; }
  __syncthreads();
  if (threadIdx.x < 3) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += part[w][threadIdx.x];
    atomicAdd(a.ftot + 4 * (blockIdx.x & (kFtotSlots - 1)) + threadIdx.x, sum);
  }
}

// One row of 4 consecutive record or stencil values (16 B for FP32, 32 B for
// FP64; record rows are 16-byte aligned).
__device__ __forceinline__ void load_row4(const float* p, float (&o)[4]) {
  const float4 t = __ldg(reinterpret_cast<const float4*>(p));
  o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void load_row4(const double* p, double (&o)[4]) {
  const double2 t0 = __ldg(reinterpret_cast<const double2*>(p));
  const double2 t1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
  o[0] = t0.x; o[1] = t0.y; o[2] = t1.x; o[3] = t1.y;
}

// One axis of a window node: ghost-inclusive index b + o (b = i0 - 1), wrapped
// to its interior image on a wrapped axis.  t: -2 outside the ghost-inclusive
// box, else the wall type of the ghost plane it lies on (0: none, or a
// periodic face); i: the interior index of the node or of its periodic image.
struct AxisNode {
  int i, t;
};
__device__ __forceinline__ AxisNode axis_node(int b, int o, int n, int flo, int fhi, bool wrap) {
  int ig = b + o;
  if (wrap) ig = wrap_ghost_index(ig, n);
  AxisNode r;
  r.t = (ig < 0 || ig > n + 1) ? -2 : (ig == 0 ? flo : (ig == n + 1 ? fhi : 0));
  const int i = ig - 1;
  r.i = i < 0 ? n - 1 : (i >= n ? 0 : i);
  return r;
}

// One sub-step of a 3D lattice with eight lanes per marker, four markers per
// warp.  A marker whose stencil record is valid for this state -- every
// marker between a refresh and its next move to another cell -- is handled by
// its group of eight lanes: lane l of the group takes the two window rows
// (y, z) = (l & 3, l >> 2) and (l & 3, (l >> 2) + 2), four x nodes each, so its
// record values arrive as six 16-byte loads.  The 1D weights are evaluated
// once per group (lane l: offset l & 3 of axis x or y, and of axis z) and
// fetched with shuffles; a node's weight is (wx * wy) * wz.  Window nodes are
// classified per axis (outside, wall type, periodic image; the type of the
// last axis whose ghost plane holds a wall wins, as in classify_node), so the
// clipped and wrapped windows, walls and moving walls follow the warp-per-
// marker body; the sums are taken over the group's lanes in a fixed order, so
// results differ from that body only by the order of the sums.  Markers whose
// record misses (moved to another cell) or that read dense moments run the
// warp-per-marker body with the whole warp afterwards.  The per-marker work
// that the 32-lane form repeats in every lane (positions, cell, key, penalty
// force) is shared by 8 lanes here, and each lane keeps six loads in flight
// instead of two.
// FP32 fields: 768 threads per SM (at most 85 registers), measured faster
// than the unconstrained allocation (94 registers, 512 threads); FP64 fields
// keep 512 (768 spill several hundred bytes).  Launched with 128 threads per
// block by default (option ibm_block): a block waits only for its own four
// warps before it retires, which took the 256^3 sub-step from 21.9 to 20.3 us
// against blocks of 256.
// HALO: the lattice has a z face bound to a neighbour slab (the instance
// without it drops the halo branches).
template <class L, class S, int DELTA, bool HALO>
__global__ void __launch_bounds__(256, sizeof(typename S::A) == 4 ? 3 : 2) k_ibm_substep8(const IbmArgs<S> a) {
  static_assert(L::D == 3, "the grouped sub-step is the 3D form");
  using R = typename S::C;
  using A = typename S::A;
  constexpr unsigned kFull = 0xffffffffu;
  __shared__ double part[8][3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gl = lane & 7, gb = lane & ~7;
  const int w0 = (int)((((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4);
  const int w = w0 + (lane >> 3);
  const Geom& g = a.g;
  const bool in = w < a.n;
  const int mk = (in && a.order) ? a.order[w] : w;
  // record rows of this lane, loaded before the key is compared (a miss
  // discards them)
  A u[3][2][4];
  double lx = 0, ly = 0, lz = 0, mass = 0, vm0 = 0, vm1 = 0, vm2 = 0;
  int i0 = 0, j0 = 0, k0 = 0;
  bool fast = false, slow = false;
  const int y = gl & 3, zr = gl >> 2;   // rows (y, zr) and (y, zr + 2)
  if (in) {
    const A* rec = stencil_record(a, mk);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int r = 0; r < 2; r++) load_row4(rec + 64 * c + 4 * (gl + 8 * r), u[c][r]);
    const int4 key = __ldg(reinterpret_cast<const int4*>(a.skey + mk));
    // IBM::phys_to_local (couplb_ibm.h:49-55)
    lx = (a.x[3 * mk] - a.lo[0]) * a.inv_dx - a.off[0] + 1.0;
    ly = (a.x[3 * mk + 1] - a.lo[1]) * a.inv_dx - a.off[1] + 1.0;
    lz = (a.x[3 * mk + 2] - a.lo[2]) * a.inv_dx - a.off[2] + 1.0;
    mass = a.m[mk];
    vm0 = a.v[3 * mk]; vm1 = a.v[3 * mk + 1]; vm2 = a.v[3 * mk + 2];
    const bool valid = !(a.active && !a.active[mk]);
    i0 = (int)floor(lx); j0 = (int)floor(ly); k0 = (int)floor(lz);
    const bool hit = (unsigned)key.w == a.cur_epoch && key.x == i0 && key.y == j0 && key.z == k0;
    fast = valid && hit && !a.all_valid;
    slow = valid && !fast;
    // an atom outside the group: zero force unless accumulating
    if (!valid && !a.accumulate && gl < 3) a.fout[3 * mk + gl] = 0.0;
  }
  // 1D weights of the group: lane l holds offset l & 3 of axis x (l < 4) or y
  // (w1), and of axis z (w2)
  const R w1 = delta1<DELTA, R>(R((gl < 4 ? lx : ly) - ((gl < 4 ? i0 : j0) - 1 + (gl & 3))));
  const R w2 = delta1<DELTA, R>(R(lz - (k0 - 1 + (gl & 3))));
  R wx[4];
#pragma unroll
  for (int o = 0; o < 4; o++) wx[o] = __shfl_sync(kFull, w1, gb + o);
  const R wy = __shfl_sync(kFull, w1, gb + 4 + y);
  const R wz[2] = {__shfl_sync(kFull, w2, gb + zr), __shfl_sync(kFull, w2, gb + zr + 2)};
  // classification of the lane's nodes: x offsets (shared by both rows), its
  // y, its two z
  AxisNode nx4[4], ny1, nz2[2];
  int hz[2];   // z halo plane of each row beyond a bound face, or -1
#pragma unroll
  for (int o = 0; o < 4; o++) nx4[o] = axis_node(i0 - 1, o, g.nx, g.face[0], g.face[1], a.wrap & 1);
  ny1 = axis_node(j0 - 1, y, g.ny, g.face[2], g.face[3], a.wrap & 2);
#pragma unroll
  for (int r = 0; r < 2; r++) {
    nz2[r] = axis_node(k0 - 1, zr + 2 * r, g.nz, g.face[4], g.face[5], a.wrap & 4);
    hz[r] = HALO ? z_halo_plane(a, k0 - 1 + zr + 2 * r) : -1;
    if (hz[r] >= 0) nz2[r].t = 0;   // the neighbour's plane: no z wall
  }
  R d[2][4];
  int t[2][4];   // -2 not in the window sums, -1 fluid, else wall type
  R ui = 0, vi = 0, wi = 0, ws = 0, wss = 0;
  bool wall_seen = false;
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int o = 0; o < 4; o++) {
      d[r][o] = (wx[o] * wy) * wz[r];
      const bool outside = nx4[o].t == -2 || ny1.t == -2 || nz2[r].t == -2;
      const int tw = nz2[r].t ? nz2[r].t : (ny1.t ? ny1.t : nx4[o].t);
      t[r][o] = outside ? -2 : (tw ? tw : -1);
      const R dd = d[r][o];
      if (t[r][o] == -1) {
        ui += R(u[0][r][o]) * dd;
        vi += R(u[1][r][o]) * dd;
        wi += R(u[2][r][o]) * dd;
        ws += dd;
        wss += dd;
      } else if (t[r][o] == 1 || t[r][o] == 3) {
        ws += dd;
        wall_seen = true;
      } else if (t[r][o] == 2) {
        ui += R(g.uw[0]) * dd;
        vi += R(g.uw[1]) * dd;
        wi += R(g.uw[2]) * dd;
        ws += dd;
        wall_seen = true;
      }
    }
  // without wall nodes in the window ws and wss are the same sums
  const bool walls = __any_sync(kFull, wall_seen && fast);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    ui += __shfl_xor_sync(kFull, ui, o);
    vi += __shfl_xor_sync(kFull, vi, o);
    wi += __shfl_xor_sync(kFull, wi, o);
    ws += __shfl_xor_sync(kFull, ws, o);
  }
  if (walls) {
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) wss += __shfl_xor_sync(kFull, wss, o);
  } else {
    wss = ws;
  }
  double tot0 = 0, tot1 = 0, tot2 = 0;
  if (fast) {
    double u0 = 0, u1 = 0, u2 = 0;
    if (ws > R(DELTA_TOL)) {
      const R iw = R(1) / ws;
      u0 = double(ui * iw); u1 = double(vi * iw); u2 = double(wi * iw);
    }
    // penalty force (fix_couplb.cpp:777-781)
    const double F0 = mass * a.xi_over_dt * (u0 * a.vs - vm0);
    const double F1 = mass * a.xi_over_dt * (u1 * a.vs - vm1);
    const double F2 = mass * a.xi_over_dt * (u2 * a.vs - vm2);
    if (gl == 0) {
      if (a.accumulate) {
        a.fout[3 * mk] += F0; a.fout[3 * mk + 1] += F1; a.fout[3 * mk + 2] += F2;
      } else {
        a.fout[3 * mk] = F0; a.fout[3 * mk + 1] = F1; a.fout[3 * mk + 2] = F2;
      }
      if (a.corr) { a.corr[3 * mk] = 0.0; a.corr[3 * mk + 1] = 0.0; a.corr[3 * mk + 2] = 0.0; }
    }
    // spread -F/(N * force_scale) onto the fluid nodes (fix_couplb.cpp:788-792,
    // couplb_ibm.h:124-132)
    if (!(wss < R(DELTA_TOL))) {
      const R sc = R(a.dvr) / wss;
      const double fl0 = -F0 * a.spread_c, fl1 = -F1 * a.spread_c, fl2 = -F2 * a.spread_c;
      const R f0 = R(fl0), f1 = R(fl1), f2 = R(fl2);
      const bool xrow = nx4[0].t == 0 && nx4[3].t == 0 && nx4[3].i == nx4[0].i + 3;
#pragma unroll
      for (int r = 0; r < 2; r++) {
        const long long nyz = (long long)g.nx * ((long long)ny1.i + (long long)g.ny * nz2[r].i);
        if (hz[r] >= 0) {
          // onto the neighbour's plane: the halo it adds to its field
          A* hrow = a.fh[hz[r] ? 1 : 0] + z_halo_offset(g, hz[r], 0, ny1.i);
#pragma unroll
          for (int o = 0; o < 4; o++) {
            if (t[r][o] != -1) continue;
            const R w = d[r][o] * sc;
            spread_add(hrow + 4 * nx4[o].i, f0 * w, f1 * w, f2 * w);
          }
          continue;
        }
#pragma unroll
        for (int o = 0; o < 4; o++) {
          if (t[r][o] != -1) continue;
          const long long nn = nyz + nx4[o].i;
          const R w = d[r][o] * sc;   // couplb_ibm.h:128
          spread_add(a.F + 4 * nn, f0 * w, f1 * w, f2 * w);
          if (a.seg_force && !xrow) a.seg_force[nn >> 3] = 1;
        }
        if (a.seg_force && xrow && t[r][0] == -1) {
          const long long n0 = nyz + nx4[0].i;
          a.seg_force[n0 >> 3] = 1;
          a.seg_force[(n0 + 3) >> 3] = 1;
        }
      }
      if (gl == 0) { tot0 = fl0 * a.dvr; tot1 = fl1 * a.dvr; tot2 = fl2 * a.dvr; }
    }
  }
  // markers whose record missed, one at a time with the whole warp
  unsigned todo = __ballot_sync(kFull, slow && gl == 0);
  while (todo) {
    const int b = __ffs(todo) - 1;
    todo &= todo - 1;
    double t3[3] = {0.0, 0.0, 0.0};
    ibm_substep_body<L, S, DELTA, false, HALO>(a, __shfl_sync(kFull, mk, b), lane, false, nullptr, nullptr, t3);
    if (lane == 0) { tot0 += t3[0]; tot1 += t3[1]; tot2 += t3[2]; }
  }
  if (!a.ftot) return;
  // the warp's total: group leaders (lanes 0, 8, 16, 24), then the block's
  tot0 += __shfl_xor_sync(kFull, tot0, 8); tot0 += __shfl_xor_sync(kFull, tot0, 16);
  tot1 += __shfl_xor_sync(kFull, tot1, 8); tot1 += __shfl_xor_sync(kFull, tot1, 16);
  tot2 += __shfl_xor_sync(kFull, tot2, 8); tot2 += __shfl_xor_sync(kFull, tot2, 16);
  if (lane == 0) { part[warp][0] = tot0; part[warp][1] = tot1; part[warp][2] = tot2; }
  __syncthreads();
  if (threadIdx.x < 3) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += part[w][threadIdx.x];
    atomicAdd(a.ftot + 4 * (blockIdx.x & (kFtotSlots - 1)) + threadIdx.x, sum);
  }
}

// Moments {ux, uy, uz, rho} (compute_velocity) of `planes` boundary planes of
// this lattice that a neighbour's IBM windows reach across face `side`: side
// 0, planes 0..planes-1 (the neighbour below reads them above its high face);
// side 1, plane nz-1 (the neighbour above reads it below its low face).
template <class L, class S>
__global__ void k_halo_moments(const IbmArgs<S> a, int side, int planes, typename S::A* __restrict__ out) {
  const Geom& g = a.g;
  const long long sxy = (long long)g.nx * g.ny;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= planes * sxy) return;
  const int p = (int)(e / sxy);
  const long long m = e % sxy;
  const int i = (int)(m % g.nx), j = (int)(m / g.nx);
  const int k = side ? g.nz - 1 : p;
  typename S::A v0, v1, v2, vr;
  compute_velocity<L, S>(a, i, j, k, (size_t)(m + k * sxy), v0, v1, v2, vr);
  out[4 * e] = v0; out[4 * e + 1] = v1; out[4 * e + 2] = v2; out[4 * e + 3] = vr;
}

// Forces a neighbour spread onto this lattice's boundary planes (its halo
// across face `side` of this lattice, layout of IbmArgs::fh) added to the
// force field: side 0 (from the neighbour below), planes 0..planes-1; side 1
// (from above), plane nz-1.  The segments that receive a force are flagged
// for the LB step (the fold of exchange_forces, couplb_streaming.h:217-245).
template <class A>
__global__ void k_halo_fold(Geom g, int side, int planes, const A* __restrict__ in, A* __restrict__ F,
                            unsigned char* __restrict__ seg) {
  const long long sxy = (long long)g.nx * g.ny;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= planes * sxy) return;
  const int p = (int)(e / sxy);
  const long long m = e % sxy;
  const long long n = m + (long long)(side ? g.nz - 1 : p) * sxy;
  const A f0 = in[4 * e], f1 = in[4 * e + 1], f2 = in[4 * e + 2];
  if (f0 == A(0) && f1 == A(0) && f2 == A(0)) return;
  F[4 * n] += f0;
  F[4 * n + 1] += f1;
  F[4 * n + 2] += f2;
  if (seg) seg[n >> 3] = 1;
}

// Dynamic shared memory of the learned sub-step kernels (blocks of 8 warps):
// the packed network, then the block's forward-pass scratch.
constexpr size_t kLearnedSmem = sizeof(MlpPacked) + sizeof(MlpBlockScratch);

}  // namespace couplb
