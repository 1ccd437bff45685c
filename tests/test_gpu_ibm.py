"""GPU immersed-boundary sub-step against the oracle and golden vectors.

Tolerances: per-atom IBM forces within 1e-11 relative, Eulerian
force field within 1e-12 relative, FP64.  The FP32 path is bounded loosely.
"""
import os

import numpy as np
import pytest

import cases
from couplb_b200.lattice import Lattice

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"ibm_{name}.npz")))


@pytest.mark.parametrize("name", sorted(cases.IBM_CASES))
def test_fp64_forces_match_reference(cuda_lib, name):
    out = cases.run_ibm_case_gpu(cases.IBM_CASES[name], "fp64")
    ref = golden(name)
    assert rel(out["fatom"], ref["fatom"]) <= 1e-11, rel(out["fatom"], ref["fatom"])
    for k in ("fx", "fy", "fz"):
        assert rel(out[k], ref[k]) <= 1e-12, (k, rel(out[k], ref[k]))


@pytest.mark.parametrize("name", sorted(cases.IBM_CASES))
def test_fp16_forces_close(cuda_lib, name):
    """FP16 storage (FP32 arithmetic): forces follow the FP64 reference to the
    storage's ~1e-3 relative precision of the populations' deviations."""
    out = cases.run_ibm_case_gpu(cases.IBM_CASES[name], "fp16")
    ref = golden(name)
    assert rel(out["fatom"], ref["fatom"]) <= 2e-2, rel(out["fatom"], ref["fatom"])


@pytest.mark.parametrize("name", sorted(cases.IBM_CASES))
def test_fp32_forces_close(cuda_lib, name):
    out = cases.run_ibm_case_gpu(cases.IBM_CASES[name], "fp32")
    ref = golden(name)
    assert rel(out["fatom"], ref["fatom"]) <= 1e-5
    for k in ("fx", "fy", "fz"):
        assert rel(out[k], ref[k]) <= 1e-5


def test_device_arrays_match_host_arrays(cuda_lib):
    import torch
    case = cases.IBM_CASES["d3_peskin_periodic"]
    x, v, m, active, _ = cases.ibm_atoms(case)
    res = []
    for dev in (False, True):
        L = Lattice(3, *case["n"], tau=case["tau"])
        L.set_populations(cases.initial_populations(3, case["n"], case["seed"]))
        L.set_ibm_params(delta="peskin4", md_per_lb=2, xi_ibm=0.7)
        if dev:
            t = {k: torch.from_numpy(a).cuda() for k, a in dict(x=x, v=v, m=m).items()}
            ta = torch.from_numpy(active).cuda()
            tf = torch.zeros((x.shape[0], 3), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            L.ibm_substep_device(x.shape[0], t["x"].data_ptr(), t["v"].data_ptr(), t["m"].data_ptr(),
                                 tf.data_ptr(), ta.data_ptr(), refresh=True)
            L.synchronize()
            fa = tf.cpu().numpy()
        else:
            fa = np.zeros_like(x)
            L.ibm_substep(x, v, m, fa, active=active, refresh=True)
        res.append((fa, L.get_force_field()))
        L.close()
    assert rel(res[1][0], res[0][0]) <= 1e-14
    for a, b in zip(res[1][1], res[0][1]):
        assert rel(a, b) <= 1e-12


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_momentum_conservation_per_lb_interval(cuda_lib, prec, tol):
    """Periodic box, markers coupled with md_per_lb sub-steps: over one LB
    interval the fluid gains exactly the momentum the markers lose,
    dP_fluid = -(1/N) sum_sub sum_i F_i (docs/theory.md:44-60)."""
    n = (40, 36, 32)
    rng = np.random.default_rng(3)
    na, N = 400, 4
    L = Lattice(3, *n, tau=0.8, precision=prec)
    L.set_populations(cases.initial_populations(3, n, 8))
    L.set_ibm_params(delta="peskin4", md_per_lb=N, xi_ibm=1.0, dt_lbm=1.0)
    x = rng.uniform(0, 1, (na, 3)) * np.array(n)
    v = 0.01 * rng.standard_normal((na, 3))
    m = np.ones(na)
    for cycle in range(3):
        L.lbm_step()
        L.macroscopic()
        p0 = np.array(L.diagnostics().mom)
        fsum = np.zeros(3)
        for s in range(N):
            fa = np.zeros((na, 3))
            L.ibm_substep(np.ascontiguousarray(x + 0.01 * s), v, m, fa, refresh=(s == 0))
            fsum += fa.sum(0)
        L.lbm_step()
        L.macroscopic()
        p1 = np.array(L.diagnostics().mom)
        dp = p1 - p0
        expect = -fsum / N
        assert np.abs(dp - expect).max() <= tol * np.abs(expect).max() + 1e-14, (cycle, dp, expect)
        # the FP64 device accumulator of the spread force agrees as well
        tot = L.ibm_total_force(reset=True)
        assert np.abs(tot - expect).max() <= 1e-12 * np.abs(expect).max()


def _fused_case_run(prec, lag, fused, wall, n=(64, 48, 40), natoms=600, cycles=3, md_per_lb=2, seed=7):
    """LB cycles of couplb_lbm_step_ibm (LB step + refresh sub-step in one
    call) and later sub-steps; returns per-sub-step atom forces, the force
    field, the populations and the records the last fused launch filled."""
    rng = np.random.default_rng(seed)
    hi = np.array(n, float)
    x0 = rng.uniform(0.0, 1.0, (natoms, 3)) * hi
    x0[:40, 2] = rng.uniform(0.0, 1.5, 40)                # next to the low z face
    x0[40:80, 2] = hi[2] - rng.uniform(0.0, 1.5, 40)      # and the high one
    v = 0.01 * rng.standard_normal((natoms, 3))
    m = rng.uniform(0.5, 1.5, natoms)
    L = Lattice(3, *n, tau=0.7, wall=wall, wall_vel=(0.01, 0, 0), body_force=True, precision=prec)
    L.set_populations(cases.initial_populations(3, n, seed))
    L.set_ibm_params(delta="peskin4", md_per_lb=md_per_lb, xi_ibm=0.8)
    L.set_option("fused_refresh", int(fused))
    L.set_option("refresh_lag", lag)
    fs, filled = [], []
    x = x0.copy()
    g = (1e-5, 0.0, 2e-6)
    for c in range(cycles):
        for s in range(md_per_lb):
            x = np.ascontiguousarray(np.mod(x + 0.3 * v, hi))
            fa = np.zeros_like(x)
            if s == 0:
                L.lbm_step_ibm(x, v, m, fa, g_lb=g)
                filled.append(L.get_option("refresh_filled"))
            else:
                L.ibm_substep(x, v, m, fa, refresh=False)
            fs.append(fa)
    out = dict(f=np.stack(fs), F=np.stack(L.get_force_field()), pop=L.get_populations(), filled=filled)
    L.close()
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("wall", [(0,) * 6, (0, 0, 1, 2, 3, 1)])
def test_fused_refresh_matches_separate_refresh(cuda_lib, prec, wall):
    """The LB launch that fills the refresh's stencil records (fused) gives
    the same forces, force field and populations, bit for bit, as the
    separate refresh kernel, for any lag (0: no plane is complete when a block
    looks, so the first sub-step fills every record; 1000: no bucket is
    served; 6: most records are filled in the launch)."""
    ref = _fused_case_run(prec, 8, False, wall)
    assert ref["filled"] == [-1, -1, -1]
    for lag in (0, 6, 1000):
        got = _fused_case_run(prec, lag, True, wall)
        np.testing.assert_array_equal(got["f"], ref["f"])
        np.testing.assert_array_equal(got["F"], ref["F"])
        np.testing.assert_array_equal(got["pop"], ref["pop"])
        if lag == 6:
            assert min(got["filled"]) > 0.5 * 600, got["filled"]
        if lag == 1000:
            assert got["filled"] == [0, 0, 0]


def test_lbm_step_ibm_fp64_matches_oracle(cuda_lib):
    """FP64 (no fused refresh): the combined call is the LB step followed by
    the refresh sub-step of the reference (golden case inputs)."""
    from oracle.bindings import OracleGrid
    case = cases.IBM_CASES["d3_peskin_periodic"]
    n = case["n"]
    x, v, m, active, dxs = cases.ibm_atoms(case)
    L = Lattice(3, *n, tau=case["tau"])
    L.set_populations(cases.initial_populations(3, n, case["seed"]))
    L.set_ibm_params(delta=case["delta"], md_per_lb=case["md_per_lb"], xi_ibm=case["xi"])
    O = OracleGrid(3, *n, tau=case["tau"])
    O.set_f(cases.initial_populations(3, n, case["seed"]))
    ip = cases._ibm_params(case)
    fg, fo = np.zeros_like(x), np.zeros_like(x)
    L.lbm_step_ibm(x, v, m, fg, active=active)
    assert L.get_option("refresh_filled") == -1
    O.lbm_step()
    O.ibm_substep(ip, x, v, m, fo, active=active, refresh=True, fold=True)
    assert rel(fg, fo) <= 1e-11, rel(fg, fo)
    L.close()
    O.close()
