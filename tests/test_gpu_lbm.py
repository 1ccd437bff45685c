"""GPU lattice kernels against the CPU oracle and the reference's golden vectors.

Tolerances: the FP64 GPU path matches the oracle's fields within
1e-12 relative (max |a-b| / max |b| over the field); the FP32-shifted path is
checked by its relative L2 velocity error against FP64; FP16 storage is
reported with a loose bound.
"""
import os

import numpy as np
import pytest

import cases
from couplb_b200.lattice import Lattice

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_FP64 = 1e-12


def rel(a, b, scale=None):
    s = np.abs(b).max() if scale is None else scale
    return np.abs(a - b).max() / max(s, 1e-300)


def field_errors(out, ref):
    """Relative errors per field; velocity components are measured against the
    largest velocity component of the field (a component that is zero up to
    roundoff has no relative scale of its own)."""
    us = max(np.abs(ref[k]).max() for k in ("ux", "uy", "uz"))
    return {k: rel(out[k], ref[k], us if k in ("ux", "uy", "uz") else None) for k in ref}


def l2(a, b):
    return np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300))


def golden(prefix, name):
    return dict(np.load(os.path.join(GOLDEN, f"{prefix}_{name}.npz")))


@pytest.mark.parametrize("name", sorted(cases.LB_CASES))
def test_fp64_matches_reference_golden(cuda_lib, name):
    out = cases.run_lb_case_gpu(cases.LB_CASES[name], "fp64")
    errs = field_errors(out, golden("lb", name))
    assert max(errs.values()) <= TOL_FP64, errs


@pytest.mark.parametrize("name", ["d3q19_mixed", "d2q9_mixed"])
def test_fp64_matches_port_oracle(cuda_lib, name):
    case = cases.LB_CASES[name]
    out = cases.run_lb_case_gpu(case, "fp64")
    errs = field_errors(out, cases.run_lb_case_oracle(case, "port"))
    assert max(errs.values()) <= TOL_FP64, errs


@pytest.mark.parametrize("prec,tol_f,tol_u", [("fp32", 1e-6, 1e-5), ("fp16", 2e-3, 5e-2)])
@pytest.mark.parametrize("name", sorted(cases.LB_CASES))
def test_reduced_precision_close_to_fp64(cuda_lib, name, prec, tol_f, tol_u):
    out = cases.run_lb_case_gpu(cases.LB_CASES[name], prec)
    ref = golden("lb", name)
    assert rel(out["f"], ref["f"]) <= tol_f
    u = np.stack([out["ux"], out["uy"], out["uz"]])
    ur = np.stack([ref["ux"], ref["uy"], ref["uz"]])
    assert l2(u, ur) <= tol_u, l2(u, ur)


def test_init_equilibrium_matches_reference_feq(cuda_lib):
    from oracle.bindings import OracleGrid
    G = OracleGrid(3, 6, 5, 4, tau=0.8, wall=(0, 0, 1, 1, 0, 0))
    G.init_equilibrium(1.02, 0.01, -0.02, 0.005)
    L = Lattice(3, 6, 5, 4, tau=0.8, wall=(0, 0, 1, 1, 0, 0))
    L.init_equilibrium(1.02, 0.01, -0.02, 0.005)
    a = cases.interior(L.get_populations(), 3)
    b = cases.interior(G.get_f(), 3)
    assert rel(a, b) <= 1e-15


@pytest.mark.parametrize("prec,tol", [("fp64", 0.0), ("fp32", 1e-7), ("fp16", 2e-4)])
def test_population_round_trip(cuda_lib, prec, tol):
    f0 = cases.initial_populations(3, (7, 5, 6), 7)
    L = Lattice(3, 7, 5, 6, tau=0.7, precision=prec)
    L.set_populations(f0)
    f1 = L.get_populations()
    assert np.abs(cases.interior(f1, 3) - cases.interior(f0, 3)).max() <= tol


def test_larger_grid_matches_oracle(cuda_lib):
    """64x32x24 channel with moving and free-slip walls, 15 steps, FP64."""
    case = dict(dim=3, n=(64, 32, 24), tau=0.62, wall=(0, 0, 2, 1, 3, 3), wall_vel=(0.03, 0, 0),
                gravity=(2e-6, 0, 0), steps=15, seed=5, noise=1.0, force=True, refresh_every=6)
    out = cases.run_lb_case_gpu(case, "fp64")
    errs = field_errors(out, cases.run_lb_case_oracle(case, "port"))
    assert max(errs.values()) <= TOL_FP64, errs


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("wall", [(0, 0, 1, 1, 1, 1), (0, 0, 2, 3, 4, 1), (0,) * 6, (1, 2, 0, 0, 3, 3)])
def test_kernel_variants_agree(cuda_lib, prec, wall):
    """The fused-kernel variants: packed (paired FP32) agrees with plain
    within FP32 rounding; every wall layout."""
    n = (64, 20, 12)
    res = {}
    for kern in (0, 2):
        L = Lattice(3, *n, tau=0.7, wall=wall, wall_vel=(0.02, 0.01, 0), body_force=True, precision=prec)
        L.set_option("kernel", kern)
        L.set_populations(cases.initial_populations(3, n, 21))
        for _ in range(6):
            L.lbm_step((1e-5, 0, 2e-6))
        res[kern] = (L.get_populations(), L.get_option("last_kernel"))
        assert L.get_option("timeouts") == 0
        L.close()
    assert res[0][1] == 0
    assert res[2][1] == (0 if prec == "fp64" else 2)
    tol = {"fp64": 0.0, "fp32": 1e-6, "fp16": 2e-3}[prec]
    assert np.abs(res[2][0] - res[0][0]).max() <= tol * np.abs(res[0][0]).max()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 1e-9)])
def test_mass_conservation_periodic(cuda_lib, prec, tol):
    """Fully periodic box without forcing: sum rho is invariant (FP64 sums)."""
    L = Lattice(3, 96, 64, 48, tau=0.7, precision=prec)
    L.set_populations(cases.initial_populations(3, (96, 64, 48), 9))
    m0 = L.diagnostics().mass
    for _ in range(50):
        L.lbm_step()
    L.macroscopic()
    m1 = L.diagnostics().mass
    assert abs(m1 - m0) / m0 <= tol, (m0, m1)


def test_momentum_gain_equals_body_force(cuda_lib):
    """Periodic box with gravity: each LB step adds g * sum(rho_prev) of momentum
    (Guo forcing, fix_couplb.cpp:706 and couplb_collision.h:55)."""
    n = (32, 24, 16)
    g = (3e-6, -1e-6, 2e-6)
    L = Lattice(3, *n, tau=0.8, body_force=True)
    L.set_populations(cases.initial_populations(3, n, 4))
    L.macroscopic()
    d0 = L.diagnostics()
    p0 = np.array(d0.mom)
    L.lbm_step(g)
    L.macroscopic()
    d1 = L.diagnostics()
    dp = np.array(d1.mom) - p0
    np.testing.assert_allclose(dp, np.array(g) * d0.mass, rtol=1e-9)


def test_nonfinite_density_is_reported_not_trapped(cuda_lib):
    """A NaN population: the kernel clamps the density like the reference
    (couplb_lattice.h:178-186) and counts it in the status word."""
    f0 = cases.initial_populations(3, (8, 6, 5), 3)
    f0[4, 3, 3, 3] = np.nan
    L = Lattice(3, 8, 6, 5, tau=0.8)
    L.set_populations(f0)
    L.lbm_step()
    clamps, nonfinite = L.read_status(reset=True)
    assert clamps >= 1 and nonfinite >= 1
    L.set_populations(cases.initial_populations(3, (8, 6, 5), 3))
    L.lbm_step()
    assert L.read_status() == (0, 0)


def test_pipelined_status_read(cuda_lib):
    """couplb_status_post / couplb_status_last: the counts of the post before
    the latest one, without draining the stream."""
    n = (16, 12, 10)
    L = Lattice(3, *n, tau=0.8)
    assert L.status_last() == (0, 0)          # nothing posted yet
    L.set_populations(cases.initial_populations(3, n, 5))
    L.lbm_step()
    L.status_post()
    assert L.status_last() == (0, 0)          # one post: waits for it
    f0 = cases.initial_populations(3, n, 5)
    f0[4, 3, 3, 3] = np.nan
    L.set_populations(f0)
    L.lbm_step()
    L.status_post()                           # sees the non-finite density
    L.lbm_step()
    L.status_post()
    clamps, nonfinite = L.status_last()       # the previous post
    assert nonfinite >= 1 and clamps >= 1
    L.close()
