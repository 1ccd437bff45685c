// lbm_packed.cuh -- the fused stream + collide step for the shifted storage
// formats with two x-neighbour nodes per thread and packed FP32x2 arithmetic.
//
// Thread t owns nodes (2t, 2t+1) of an x-row.  Every quantity of the update
// is a float2 (one lane per node) and goes through the sm_100 paired FP32
// instructions (__ffma2_rn / __fadd2_rn / __fmul2_rn), which halves the ALU
// instructions per node compared with one node per thread.  Populations whose
// source does not move in x are read as one 8-byte (FP32) or 4-byte (half2)
// load; for the x-moving directions the pair (i0-ex, i0+1-ex) straddles a
// pair boundary and is read as the aligned pair plus one scalar.  Rows next to
// a wall use the per-node general pull.
//
// The arithmetic is that of k_stream_collide for the shifted formats (BGK +
// Guo with the exact mass / momentum correction); nx must be even.
#pragma once
#include "lbm_kernels.cuh"

namespace couplb {

__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Pair loads / stores of the storage formats (index of the even node).
template <class S>
struct Pair;

template <>
struct Pair<StoreF32S> {
  __device__ __forceinline__ static float2 ld(const float* p) {
    return __ldg(reinterpret_cast<const float2*>(p));
  }
  __device__ __forceinline__ static float ld1(const float* p) { return __ldg(p); }
  __device__ __forceinline__ static void st(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
};

template <>
struct Pair<StoreF16S> {
  __device__ __forceinline__ static float2 ld(const __half* p) {
    const float2 v = __half22float2(__ldg(reinterpret_cast<const __half2*>(p)));
    return mul2(v, f2(StoreF16S::kInvScale));
  }
  __device__ __forceinline__ static float ld1(const __half* p) { return StoreF16S::ld(p); }

  __device__ __forceinline__ static void st(__half* p, float2 v) {
    *reinterpret_cast<__half2*>(p) = __float22half2_rn(mul2(v, f2(StoreF16S::kScale)));
  }
};

template <class L, class S>
__device__ __forceinline__ void x2_node_pair(const LBArgs<S>& a, int i0, int j, int k) {
  using T = typename S::T;
  using I = unsigned;
  const Geom& g = a.g;
  const I qs = (I)g.qs;
  const I sx = (I)g.nx, sxy = (I)g.nx * (I)g.ny;
  const I n0 = (I)i0 + (I)j * sx + (I)k * sxy;
  // n0 even: both nodes in one force segment; the flag is read first and the
  // force right after the populations, so the latencies overlap
  const bool hf = a.F && (!a.seg_force || a.seg_force[n0 >> 3]);

  float2 f[L::Q];
  if (row_is_interior<L>(g, j, k)) {
    const I row = (I)j * sx + (I)k * sxy;
    const I im = (i0 == 0) ? g.nx - 1 : i0 - 1;      // source of node i0 for ex = +1
    const I ip = (i0 + 2 == g.nx) ? 0 : i0 + 2;      // source of node i0+1 for ex = -1
#pragma unroll
    for (int q = 0; q < L::Q; q++) {
      const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
      const I ro = row - (I)(ey * g.nx) - (I)ez * sxy;   // source row (unsigned wrap is exact)
      // ro + i0 is even (nx even): the pair sits in one tile, 2-element aligned
      const float2 pr = Pair<S>::ld(a.fin + pidx<L, S, I>(q, ro + (I)i0, qs));
      if (ex == 0) {
        f[q] = pr;
      } else if (ex == 1) {
        f[q] = make_float2(Pair<S>::ld1(a.fin + pidx<L, S, I>(q, ro + im, qs)), pr.x);
      } else {
        f[q] = make_float2(pr.y, Pair<S>::ld1(a.fin + pidx<L, S, I>(q, ro + ip, qs)));
      }
    }
  } else {
    float fa[L::Q], fb[L::Q];
    pull_general<L, S, I>(g, a.fin, a.rho_field, i0, j, k, n0, fa);
    pull_general<L, S, I>(g, a.fin, a.rho_field, i0 + 1, j, k, n0 + 1, fb);
#pragma unroll
    for (int q = 0; q < L::Q; q++) f[q] = make_float2(fa[q], fb[q]);
  }

  // apply_external_force (fix_couplb.cpp:693-707)
  float2 Fx = f2(0.f), Fy = f2(0.f), Fz = f2(0.f);
  if (hf) {
    float4* p = reinterpret_cast<float4*>(a.F + 4 * (size_t)n0);
    const float4 fa = p[0], fb = p[1];
    Fx = make_float2(fa.x, fb.x);
    Fy = make_float2(fa.y, fb.y);
    Fz = make_float2(fa.z, fb.z);
    // clear_forces: leave the field zero where it was read nonzero
    if (fa.x != 0.f || fa.y != 0.f || fa.z != 0.f) p[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (fb.x != 0.f || fb.y != 0.f || fb.z != 0.f) p[1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  // moments (density deviation and momentum), q order
  float2 r = f2(0.f), jx = f2(0.f), jy = f2(0.f), jz = f2(0.f);
#pragma unroll
  for (int q = 0; q < L::Q; q++) {
    r = add2(r, f[q]);
    if (L::ex(q) == 1) jx = add2(jx, f[q]); else if (L::ex(q) == -1) jx = sub2(jx, f[q]);
    if (L::ey(q) == 1) jy = add2(jy, f[q]); else if (L::ey(q) == -1) jy = sub2(jy, f[q]);
    if (L::D == 3) { if (L::ez(q) == 1) jz = add2(jz, f[q]); else if (L::ez(q) == -1) jz = sub2(jz, f[q]); }
  }
  const float rho0 = float(g.rho0);
  float2 rho = add2(f2(rho0), r);
  {
    const float cx = clamp_rho(rho.x, a.status, kStClamps);
    const float cy = clamp_rho(rho.y, a.status, kStClamps);
    if (cx != rho.x) { rho.x = cx; r.x = cx - rho0; }
    if (cy != rho.y) { rho.y = cy; r.y = cy - rho0; }
  }

  if (a.rho_mode != kRhoNone) {
    float2 rp = rho;
    if (a.rho_mode == kRhoField) rp = add2(f2(rho0), *reinterpret_cast<const float2*>(a.rho_field + n0));
    Fx = fma2(f2(float(a.grav[0])), rp, Fx);
    Fy = fma2(f2(float(a.grav[1])), rp, Fy);
    Fz = fma2(f2(float(a.grav[2])), rp, Fz);
  }
  if (a.write_rho == 2) {
    *reinterpret_cast<float2*>(a.rho_field + n0) = r;
  } else if (a.write_rho == 1) {
    if (near_moving_wall<L>(g, i0, j, k)) a.rho_field[n0] = r.x;
    if (near_moving_wall<L>(g, i0 + 1, j, k)) a.rho_field[n0 + 1] = r.y;
  }

  // u = (j + F/2) / rho
  const float2 inv_r = make_float2(__fdividef(1.0f, rho.x), __fdividef(1.0f, rho.y));
  const float2 half = f2(0.5f);
  const float2 ux = mul2(fma2(half, Fx, jx), inv_r);
  const float2 uy = mul2(fma2(half, Fy, jy), inv_r);
  const float2 uz = mul2(fma2(half, Fz, jz), inv_r);

  // BGK + Guo over the pairs (q, q+1), increments d, exact mass / momentum
  const float om = float(a.omega);
  const float2 nom = f2(-om);
  const float hom = 1.0f - 0.5f * om;
  const float2 uu15 = mul2(f2(1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
  const float2 uf3 = mul2(f2(3.0f), fma2(ux, Fx, fma2(uy, Fy, mul2(uz, Fz))));
  float2 m, px = make_float2(-Fx.x, -Fx.y), py = make_float2(-Fy.x, -Fy.y),
            pz = make_float2(-Fz.x, -Fz.y);
  float2 d0, da[2 * L::D];
  {
    const float w = float(L::w(0));
    const float2 fe = mul2(f2(w), sub2(r, mul2(rho, uu15)));
    d0 = fma2(nom, sub2(f[0], fe), mul2(f2(-w * hom), uf3));
    m = d0;
  }
#pragma unroll
  for (int q = 1; q < L::Q; q += 2) {
    const int cx = L::ex(q), cy = L::ey(q), cz = L::ez(q);
    const float w = float(L::w(q));
    // e.u and e.F with e components in {-1, 0, 1}
    float2 eu = f2(0.f), ef = f2(0.f);
    if (cx == 1) { eu = add2(eu, ux); ef = add2(ef, Fx); } else if (cx == -1) { eu = sub2(eu, ux); ef = sub2(ef, Fx); }
    if (cy == 1) { eu = add2(eu, uy); ef = add2(ef, Fy); } else if (cy == -1) { eu = sub2(eu, uy); ef = sub2(ef, Fy); }
    if (cz == 1) { eu = add2(eu, uz); ef = add2(ef, Fz); } else if (cz == -1) { eu = sub2(eu, uz); ef = sub2(ef, Fz); }
    const float2 even = fma2(mul2(f2(4.5f), eu), eu, make_float2(-uu15.x, -uu15.y));
    const float2 aa = fma2(rho, even, r);
    const float2 bb = mul2(rho, mul2(f2(3.0f), eu));
    const float2 se = mul2(f2(w * hom), fma2(mul2(f2(9.0f), eu), ef, make_float2(-uf3.x, -uf3.y)));
    const float2 so = mul2(f2(w * hom * 3.0f), ef);
    const float2 fep = mul2(f2(w), add2(aa, bb));
    const float2 fem = mul2(f2(w), sub2(aa, bb));
    const float2 dp = fma2(nom, sub2(f[q], fep), add2(se, so));
    const float2 dm = fma2(nom, sub2(f[q + 1], fem), sub2(se, so));
    const float2 dd = sub2(dp, dm);
    m = add2(m, add2(dp, dm));
    if (cx == 1) px = add2(px, dd); else if (cx == -1) px = sub2(px, dd);
    if (cy == 1) py = add2(py, dd); else if (cy == -1) py = sub2(py, dd);
    if (L::D == 3) { if (cz == 1) pz = add2(pz, dd); else if (cz == -1) pz = sub2(pz, dd); }
    if (q < 2 * L::D) {
      da[q - 1] = dp;
      da[q] = dm;
    } else {
      Pair<S>::st(a.fout + pidx<L, S, I>(q, n0, qs), add2(f[q], dp));
      Pair<S>::st(a.fout + pidx<L, S, I>(q + 1, n0, qs), add2(f[q + 1], dm));
    }
  }
  Pair<S>::st(a.fout + pidx<L, S, I>(0, n0, qs), add2(f[0], sub2(d0, m)));
  const float2 pr[3] = {mul2(half, px), mul2(half, py), mul2(half, pz)};
#pragma unroll
  for (int c = 0; c < L::D; c++) {
    Pair<S>::st(a.fout + pidx<L, S, I>(2 * c + 1, n0, qs), add2(f[2 * c + 1], sub2(da[2 * c], pr[c])));
    Pair<S>::st(a.fout + pidx<L, S, I>(2 * c + 2, n0, qs), add2(f[2 * c + 2], add2(da[2 * c + 1], pr[c])));
  }
}

template <class L, class S, int MINB = 5>
__global__ void __launch_bounds__(128, MINB) k_stream_collide_x2(const LBArgs<S> a) {
  const int i0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i0 < a.g.nx) x2_node_pair<L, S>(a, i0, blockIdx.y, blockIdx.z);
}

}  // namespace couplb
