// storage.cuh -- population storage formats.
//
//   StoreF64  : plain f in FP64, FP64 arithmetic (the parity form).
//   StoreF32S : shifted h = f - w_q*rho0 in FP32, FP32 arithmetic.
//   StoreF16S : shifted h stored as IEEE half scaled by 2^15, FP32 arithmetic
//               (the "FP16S" storage of Lehmann et al., Phys. Rev. E 106,
//               015308 (2022): |h| < 2 for Ma < 0.3, so h*2^15 stays inside
//               the half range while keeping 11 significant bits).
//
// Shifting removes the O(1) rest value w_q*rho0 from every population, so the
// density deviation sum_q h_q and the momentum are computed without the
// cancellation of sum_q f_q - rho0.  The bounce-back, moving-wall and
// free-slip rules commute with the shift because w[q] == w[opp[q]] ==
// w[refl[d][q]].
//
// Layout in HBM (kTile, read through pidx in lbm_kernels.cuh): 0 = one plane
// per population, element q * qs + n; kTile > 0 = tiles of kTile consecutive
// nodes x Q planes.  FP32-shifted uses tiles of 64 nodes (256 B per plane and
// tile, the span of one warp of the packed kernel): the IBM refresh, which
// reads 19 short rows around each stencil node, then finds them within one
// 4.9 KB tile instead of 19 planes 64 MB apart (the same DRAM bytes, better
// DRAM row locality).  Measured on the D3Q19
// workloads against plane-major: fused LB kernel unchanged (36.6 vs 36.7
// GLUPS on 256x128x128), LBM + IBM cycle 0.729 -> 0.710 ms (256^3, 20000
// markers) and 1.560 -> 1.511 ms (rods); tiles of 8 nodes cut the refresh
// more but slowed the LB kernel by 7 %, tiles of 32 by 2 %.
#pragma once
#include <cuda_fp16.h>

namespace couplb {

struct StoreF64 {
  using T = double;  // stored population
  using C = double;  // arithmetic
  using A = double;  // auxiliary fields (force, density, moments)
  static constexpr bool kShift = false;
  static constexpr int kTile = 0;
  __device__ __forceinline__ static C ld(const T* p) { return __ldg(p); }
  __device__ __forceinline__ static C ld_shared(const T* p) { return *p; }
  __device__ __forceinline__ static void st(T* p, C v) { *p = v; }
};

struct StoreF32S {
  using T = float;
  using C = float;
  using A = float;
  static constexpr bool kShift = true;
  static constexpr int kTile = 64;
  __device__ __forceinline__ static C ld(const T* p) { return __ldg(p); }
  __device__ __forceinline__ static C ld_shared(const T* p) { return *p; }
  __device__ __forceinline__ static void st(T* p, C v) { *p = v; }
};

struct StoreF16S {
  using T = __half;
  using C = float;
  using A = float;
  static constexpr bool kShift = true;
  static constexpr int kTile = 0;
  static constexpr float kScale = 32768.0f;
  static constexpr float kInvScale = 1.0f / 32768.0f;
  __device__ __forceinline__ static C ld(const T* p) {
    return __half2float(__ldg(p)) * kInvScale;
  }
  __device__ __forceinline__ static C ld_shared(const T* p) { return __half2float(*p) * kInvScale; }
  __device__ __forceinline__ static void st(T* p, C v) {
    *p = __float2half_rn(v * kScale);
  }
};

}  // namespace couplb
