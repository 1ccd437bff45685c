"""couplb_diagnostics_noalloc: the stability reductions for callers that
cannot let a library allocate device memory (an MD code whose pool allocator
owns all device memory, or a time loop that must not stall on the device-wide
synchronisation of cudaMalloc / cudaFree).  The entry point takes caller-owned
device inputs and output and keeps its scratch in a fixed device array.

Checked here against the allocating couplb_diagnostics on the same moments,
on two calls in a row (the second call reuses the scratch the first left
behind).  This file is collected last so that a run stopping at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from couplb_b200 import abi
from couplb_b200.lattice import Lattice

pytestmark = pytest.mark.gpu

PREC = {"fp64": abi.FP64, "fp32": abi.FP32_SHIFTED}


def device_moments(L, prec, torch):
    """The lattice's interior moments copied into caller-owned device tensors,
    in the layout the entry point takes (rho as a deviation for shifted formats)."""
    rho, ux, uy, uz = [cases.interior(a, 3).reshape(-1) for a in L.get_macroscopic()]
    if prec == "fp64":
        arrs = [rho, ux, uy, uz]
        dt = torch.float64
    else:
        arrs = [(rho - 1.0).astype(np.float32), ux.astype(np.float32), uy.astype(np.float32),
                uz.astype(np.float32)]
        dt = torch.float32
    return [torch.tensor(a, dtype=dt, device="cuda") for a in arrs]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_noalloc_diagnostics_match_allocating_entry_point(cuda_lib, prec):
    import torch
    n3 = (48, 40, 36)
    L = Lattice(3, *n3, tau=0.7, wall=(0, 0, 1, 1, 0, 0), body_force=True, precision=prec)
    L.set_populations(cases.initial_populations(3, n3, 31))
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for _ in range(3 + 4 * call):
            L.lbm_step((2e-5, 0, 0))
        L.macroscopic()
        ref = L.diagnostics()
        fields = device_moments(L, prec, torch)
        out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = cuda_lib.couplb_diagnostics_noalloc(*[t.data_ptr() for t in fields], fields[0].numel(),
                                                 PREC[prec], 1.0, out.data_ptr(), stream)
        assert rc == abi.OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = np.array([ref.umax, ref.mass, ref.mom[0], ref.mom[1], ref.mom[2]])
        # same inputs, different block partition of the FP64 sums
        np.testing.assert_allclose(got[:2], want[:2], rtol=1e-12)
        np.testing.assert_allclose(got[2:], want[2:], rtol=1e-9, atol=1e-12 * want[1] * want[0])
    L.close()


def test_noalloc_rejects_sizes_above_its_capacity(cuda_lib):
    import torch
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    too_many = 2048 * 32768 + 1
    rc = cuda_lib.couplb_diagnostics_noalloc(t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                             too_many, abi.FP64, 1.0, out.data_ptr(), None)
    assert rc == abi.ERR_TOO_LARGE


def test_noalloc_max_speed_propagates_nan(cuda_lib):
    """A NaN velocity at one node makes max |u| NaN (there is no separate
    non-finite count in this entry point), on two calls in a row."""
    import torch
    n = 5000
    g = torch.Generator().manual_seed(3)
    fields = [torch.rand(n, generator=g, dtype=torch.float64).cuda() * 1e-2 for _ in range(4)]
    fields[0] += 1.0
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call, bad in enumerate((4321, 17)):
        fields[2][bad] = float("nan")
        torch.cuda.synchronize()
        rc = cuda_lib.couplb_diagnostics_noalloc(*[t.data_ptr() for t in fields], n, abi.FP64, 1.0,
                                                 out.data_ptr(), stream)
        assert rc == abi.OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isnan(got[0]), (call, got)
        assert np.isfinite(got[1])
        fields[2][bad] = 0.0
