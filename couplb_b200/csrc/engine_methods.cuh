// engine_methods.cuh -- launch of the cooperative IBM method kernels
// (iterative / learned sub-steps).  The definitions are instantiated in
// engine_methods_f64.cu, _f32.cu and _f16.cu (one storage format each, so the
// heavy method kernels compile in parallel); other units see the declaration.
#pragma once
#include "engine_common.cuh"
#include "mlp_internal.h"

namespace couplb {

template <class L, class S>
int launch_method(couplb_handle* h, PassArgs<S>& P, int delta, bool learned, int n);

#ifdef COUPLB_METHODS_IMPL
namespace eng {
// Blocks of a cooperative kernel that fit on the device at once (cached).
template <class K>
int coop_resident(couplb_handle* h, K kern, size_t smem, int slot, int* out) {
  int& resident = h->coop_blocks[slot];
  if (resident == 0) {
    int coop = 0, sms = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->p.device));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->p.device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (!coop || per_sm < 1)
      return fail(h, COUPLB_ERR_UNSUPPORTED, "the device cannot run the cooperative IBM kernel");
    resident = per_sm * sms;
  }
  *out = resident;
  return COUPLB_OK;
}
}  // namespace eng

// Launch of one ITERATIVE / LEARNED sub-step: cooperative (all blocks
// resident at once) when the launch has a grid barrier, a plain launch of the
// same grid when it has none (one pass, no slip check, no slip statistics).
// In 3D, when every marker gets a warp of its own, the register-resident form
// runs.
template <class K, class A>
int launch_coop_or_plain(couplb_handle* h, K kern, unsigned grid, size_t smem, bool barrier, A& P) {
  using namespace eng;
  if (barrier) {
    void* args[] = {&P};
    CK(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(256), args, smem, h->stream));
  } else {
    kern<<<grid, 256, smem, h->stream>>>(P);
  }
  return COUPLB_OK;
}

template <class L, class S>
int launch_method(couplb_handle* h, PassArgs<S>& P, int delta, bool learned, int n) {
  using namespace eng;
  using K = void (*)(const PassArgs<S>);
  const bool roma = delta == COUPLB_DELTA_ROMA;
  const int di = (learned ? 2 : 0) + (roma ? 0 : 1);
  const size_t smem = learned ? kLearnedSmem : 0;
  const long long want = ((long long)n * 32 + 255) / 256;
  const bool barrier = P.check_first || P.ncorr > 0 || P.measure_last;
  int rc, resident = 0;
  if constexpr (L::D == 3) {
    if (h->ibm_resident) {
      K kr = learned ? (roma ? k_ibm_method_resident<L, S, 0, true> : k_ibm_method_resident<L, S, 1, true>)
                     : (roma ? k_ibm_method_resident<L, S, 0, false> : k_ibm_method_resident<L, S, 1, false>);
      if ((rc = coop_resident(h, kr, smem, 4 + di, &resident))) return rc;
      if (want <= resident) return launch_coop_or_plain(h, kr, (unsigned)want, smem, barrier, P);
    }
  }
  K kern = nullptr;
  if (learned) {
    if constexpr (L::D == 3) kern = roma ? k_ibm_method<L, S, 0, true> : k_ibm_method<L, S, 1, true>;
  } else {
    kern = roma ? k_ibm_method<L, S, 0, false> : k_ibm_method<L, S, 1, false>;
  }
  if (!kern) return fail(h, COUPLB_ERR_UNSUPPORTED, "the learned correction is defined for D3Q19");
  if ((rc = coop_resident(h, kern, smem, di, &resident))) return rc;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(want, resident));
  return launch_coop_or_plain(h, kern, grid, smem, barrier, P);
}

#endif  // COUPLB_METHODS_IMPL

}  // namespace couplb
