// lattice.cuh -- D2Q9 / D3Q19 descriptors as compile-time tables.
//
// Same velocity ordering, weights, opposite and mirror tables as the
// reference (couplb_lattice.h:24-75): the C ABI exchanges populations in the
// reference's q order, so the tables have to agree entry for entry.  Every
// kernel loops over q with #pragma unroll, so each lookup below folds to a
// constant.
#pragma once

namespace couplb {

// constants of couplb_lattice.h:13-20
constexpr double RHO_MIN = 1e-10;
constexpr double DELTA_TOL = 1e-12;
constexpr double ZERO_TOL = 1e-15;
constexpr double RHO_CLAMP_FRAC = 0.1;
constexpr double MA_WARN = 0.3;
constexpr double MA_ERROR = 0.5;

struct D2Q9 {
  static constexpr int D = 2;
  static constexpr int Q = 9;
  __host__ __device__ static constexpr int ex(int q) {
    constexpr int t[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int ey(int q) {
    constexpr int t[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr int ez(int) { return 0; }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 4.0 / 9.0 : (q < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
  }
  __host__ __device__ static constexpr int opp(int q) {
    constexpr int t[9] = {0, 2, 1, 4, 3, 6, 5, 8, 7};
    return t[q];
  }
  // index of q with its d-th component mirrored (free-slip walls)
  __host__ __device__ static constexpr int refl(int d, int q) {
    constexpr int t[3][9] = {{0, 2, 1, 3, 4, 8, 7, 6, 5},
                             {0, 1, 2, 4, 3, 7, 8, 5, 6},
                             {0, 1, 2, 3, 4, 5, 6, 7, 8}};
    return t[d][q];
  }
};

struct D3Q19 {
  static constexpr int D = 3;
  static constexpr int Q = 19;
  __host__ __device__ static constexpr int ex(int q) {
    constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[q];
  }
  __host__ __device__ static constexpr int ey(int q) {
    constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int ez(int q) {
    constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
  }
  __host__ __device__ static constexpr int opp(int q) {
    constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
    return t[q];
  }
  __host__ __device__ static constexpr int refl(int d, int q) {
    constexpr int t[3][19] = {
        {0, 2, 1, 3, 4, 5, 6, 10, 9, 8, 7, 14, 13, 12, 11, 15, 16, 17, 18},
        {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15},
        {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16}};
    return t[d][q];
  }
};

}  // namespace couplb
