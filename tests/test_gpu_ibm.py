"""GPU immersed-boundary sub-step against the oracle and golden vectors.

Tolerances: per-atom IBM forces within 1e-11 relative, Eulerian
force field within 1e-12 relative, FP64.  The FP32 path is bounded loosely.
"""
import os

import numpy as np
import pytest

import cases
from couplb_b200 import abi
from couplb_b200.lattice import Lattice
from couplb_b200.lib import CoupLBError

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


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_lbm_step_ibm_matches_separate_calls(cuda_lib, prec):
    """couplb_lbm_step_ibm (atom copies overlapped with the LB kernel) gives
    the atom forces of lbm_step + ibm_substep(refresh) bit for bit on the
    first cycle, then agrees to the rounding of the FP32 atomic sums."""
    n = (40, 32, 24)
    rng = np.random.default_rng(7)
    x0 = rng.uniform(0.0, 1.0, (300, 3)) * np.array(n, float)
    v = 0.01 * rng.standard_normal((300, 3))
    m = rng.uniform(0.5, 1.5, 300)
    out = []
    for combined in (False, True):
        L = Lattice(3, *n, tau=0.7, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.01, 0, 0), body_force=True,
                    precision=prec)
        L.set_populations(cases.initial_populations(3, n, 7))
        L.set_ibm_params(delta="peskin4", md_per_lb=2, xi_ibm=0.8)
        x = x0.copy()
        fs = []
        for c in range(3):
            for s in range(2):
                x = np.ascontiguousarray(np.mod(x + 0.3 * v, np.array(n, float)))
                fa = np.zeros_like(x)
                if s == 0 and combined:
                    L.lbm_step_ibm(x, v, m, fa, g_lb=(1e-5, 0.0, 2e-6))
                else:
                    if s == 0:
                        L.lbm_step((1e-5, 0.0, 2e-6))
                    L.ibm_substep(x, v, m, fa, refresh=(s == 0))
                fs.append(fa)
        out.append(np.stack(fs))
        L.close()
    np.testing.assert_array_equal(out[1][:2], out[0][:2])
    assert rel(out[1], out[0]) <= (1e-5 if prec == "fp32" else 1e-3)


def test_lbm_step_ibm_fp64_matches_oracle(cuda_lib):
    """FP64: the combined call is the LB step followed by the refresh
    sub-step of the reference (golden case inputs)."""
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
    O.lbm_step()
    O.ibm_substep(ip, x, v, m, fo, active=active, refresh=True, fold=True)
    assert rel(fg, fo) <= 1e-11, rel(fg, fo)
    L.close()
    O.close()


def _window_case_forces(wrap, xs, prec="fp64", n=(12, 10, 9), wall=(0,) * 6):
    L = Lattice(3, *n, tau=0.8, wall=wall, precision=prec)
    L.set_populations(cases.initial_populations(3, n, 31))
    L.set_ibm_params(delta="peskin4", md_per_lb=1, xi_ibm=0.9)
    L.set_option("ibm_window", wrap)
    v = np.tile([0.004, -0.002, 0.003], (xs.shape[0], 1))
    f = np.zeros_like(xs)
    L.ibm_substep(np.ascontiguousarray(xs), v, np.ones(xs.shape[0]), f, refresh=True)
    F = L.get_force_field()
    L.close()
    return f, F


def test_wrapped_window_is_periodic(cuda_lib):
    """ibm_window wrap: a marker at x = N - 0.25 takes the same nodes and
    weights as its periodic image at x = -0.25 (and likewise in y, z; both
    positions are exact in binary, so are the weights), and the forces agree
    bit for bit; the reference's clipped window (the default) drops a
    different plane for each of them."""
    n = (12, 10, 9)
    base = np.array([[5.3, 4.7, 3.2]])
    for d in range(3):
        hi = base.copy()
        hi[0, d] = n[d] - 0.25
        lo = base.copy()
        lo[0, d] = -0.25
        fw_hi, _ = _window_case_forces(1, hi)
        fw_lo, _ = _window_case_forces(1, lo)
        np.testing.assert_array_equal(fw_hi, fw_lo)
        fc_hi, _ = _window_case_forces(0, hi)
        fc_lo, _ = _window_case_forces(0, lo)
        assert np.abs(fc_hi - fc_lo).max() > 1e-6 * np.abs(fc_hi).max()


@pytest.mark.parametrize("wall", [(0,) * 6, (0, 0, 1, 1, 0, 0)])
def test_wrapped_window_matches_oracle(cuda_lib, wall):
    """FP64 single pass with the wrapped window against the port oracle's
    restatement of it (no reference counterpart): per-atom forces within
    1e-11, force field within 1e-12; markers within two cells of every face."""
    from oracle.bindings import OracleGrid
    n = (12, 10, 9)
    rng = np.random.default_rng(41)
    hi = np.array(n, float)
    xs = rng.uniform(0.0, 1.0, (60, 3)) * hi
    for d in range(3):
        xs[10 * d:10 * d + 5, d] = hi[d] - rng.uniform(0.0, 1.6, 5)
        xs[10 * d + 5:10 * d + 10, d] = rng.uniform(-0.5, 1.6, 5)
    fg, Fg = _window_case_forces(1, xs, wall=wall)
    mask = (0 if wall[0] else 1) | (0 if wall[2] else 2) | (0 if wall[4] else 4)
    O = OracleGrid(3, *n, tau=0.8, wall=wall)
    O.set_f(cases.initial_populations(3, n, 31))
    O.set_ibm_wrap(mask)
    ip = abi.IbmParams()
    ip.delta, ip.md_per_lb, ip.xi_ibm = 1, 1, 0.9
    ip.dt_lbm, ip.dx, ip.vel_scale, ip.force_scale = 1.0, 1.0, 1.0, 1.0
    v = np.tile([0.004, -0.002, 0.003], (xs.shape[0], 1))
    fo = np.zeros_like(xs)
    O.ibm_substep(ip, np.ascontiguousarray(xs), v, np.ones(xs.shape[0]), fo, refresh=True, fold=True)
    Fo = O.get_force()
    O.close()
    assert rel(fg, fo) <= 1e-11, rel(fg, fo)
    for c in range(3):
        a, b = cases.interior(Fg[c], 3), cases.interior(Fo[c], 3)
        assert rel(a, b) <= 1e-12, (c, rel(a, b))


def _grouped_case(prec, group, n=(40, 32, 24), cycles=3, md_per_lb=2, block=None, sort=None):
    """Atom forces per sub-step and the final force field of a walled lattice
    with 300 markers: most windows inside the interior, some at the faces and
    walls; every second marker jumps 0.6 cells in x on each later sub-step
    (a stencil-record miss); one marker in eight is not in the group."""
    rng = np.random.default_rng(19)
    x0 = rng.uniform(0.0, 1.0, (300, 3)) * np.array(n, float)
    x0[:20, 1] = rng.uniform(0.0, 2.5, 20)
    x0[20:40, 2] = n[2] - rng.uniform(0.0, 2.5, 20)
    v = 0.01 * rng.standard_normal((300, 3))
    m = rng.uniform(0.5, 1.5, 300)
    active = (np.arange(300) % 8 != 3).astype(np.int32)
    L = Lattice(3, *n, tau=0.7, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.01, 0, 0), body_force=True, precision=prec)
    L.set_option("ibm_group", group)
    if block:
        L.set_option("ibm_block", block)
    if sort is not None:
        L.set_option("ibm_sort", sort)
    L.set_populations(cases.initial_populations(3, n, 7))
    L.set_ibm_params(delta="peskin4", md_per_lb=md_per_lb, xi_ibm=0.8)
    x = x0.copy()
    fs = []
    for c in range(cycles):
        L.lbm_step((1e-5, 0.0, 2e-6))
        for s in range(md_per_lb):
            if s > 0:
                x[::2, 0] += 0.6
            x = np.ascontiguousarray(np.mod(x + 0.3 * v, np.array(n, float)))
            fa = np.zeros_like(x)
            L.ibm_substep(x, v, m, fa, active=active, refresh=(s == 0))
            fs.append(fa)
    F = [cases.interior(a, 3) for a in L.get_force_field()]
    L.close()
    return np.stack(fs), F


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_grouped_substep_matches_warp_per_marker(cuda_lib, prec, tol):
    """ibm_group 8 (four markers per warp, the default) against 32 (one warp
    per marker): the same forces up to the order of the interpolation sums."""
    f8, F8 = _grouped_case(prec, 8)
    f32, F32 = _grouped_case(prec, 32)
    assert rel(f8, f32) <= tol, rel(f8, f32)
    for c in range(3):
        assert rel(F8[c], F32[c]) <= 10 * tol, (c, rel(F8[c], F32[c]))


@pytest.mark.parametrize("block", [64, 256])
def test_grouped_substep_block_size(cuda_lib, block):
    """The launch shape of the grouped sub-step (option ibm_block, default
    128) leaves each marker's arithmetic alone: FP64 atom forces of the first
    sub-step equal bit for bit; later ones and the force field differ only by
    the order of the spread atomics."""
    f, F = _grouped_case("fp64", 8, block=block)
    fd, Fd = _grouped_case("fp64", 8)
    assert np.array_equal(f[0], fd[0])
    assert rel(f, fd) <= 1e-13, rel(f, fd)
    for c in range(3):
        assert rel(F[c], Fd[c]) <= 1e-13, (c, rel(F[c], Fd[c]))
    L = Lattice(3, 8, 8, 8)
    with pytest.raises(CoupLBError):
        L.set_option("ibm_block", 96)
    assert L.get_option("ibm_block") == 128
    L.close()


@pytest.mark.parametrize("sort", [0, 1])
def test_marker_order(cuda_lib, sort):
    """Option ibm_sort: the refresh visits the markers by z bands of their
    cells, the order remade every ibm_sort refreshes (default 16; 1: every
    refresh; 0: index order).  Each record is still filled once by its
    marker's own lanes: FP64 atom forces of the first sub-step equal bit for
    bit, later ones and the force field differ only by the order of the
    spread sums."""
    f, F = _grouped_case("fp64", 8, sort=sort)
    fd, Fd = _grouped_case("fp64", 8)
    assert np.array_equal(f[0], fd[0])
    assert rel(f, fd) <= 1e-13, rel(f, fd)
    for c in range(3):
        assert rel(F[c], Fd[c]) <= 1e-13, (c, rel(F[c], Fd[c]))


def _chain_case(sort, n=(40, 32, 24), cycles=3):
    """200 markers in chain order (0.21 cells apart along a tilted line)."""
    i = np.arange(200, dtype=np.float64)
    x0 = np.stack([5.0 + 0.15 * i, 4.0 + 0.12 * i, 3.0 + 0.08 * i], axis=1)
    v = np.zeros_like(x0)
    m = np.ones(200)
    L = Lattice(3, *n, tau=0.7, wall=(0, 0, 1, 1, 0, 0), body_force=True)
    L.set_option("ibm_sort", sort)
    L.set_populations(cases.initial_populations(3, n, 5))
    L.set_ibm_params(delta="peskin4", md_per_lb=2, xi_ibm=0.8)
    fs = []
    for c in range(cycles):
        L.lbm_step((1e-5, 0.0, 0.0))
        for s in range(2):
            fa = np.zeros_like(x0)
            L.ibm_substep(x0, v, m, fa, refresh=(s == 0))
            fs.append(fa)
    F = [cases.interior(a, 3) for a in L.get_force_field()]
    L.close()
    return np.stack(fs), F


def test_marker_order_keeps_chains(cuda_lib):
    """Markers within 2 cells of their successor (a chain): the sort keeps
    the index order and the refresh runs without it, so the results match
    ibm_sort 0."""
    f, F = _chain_case(1)
    f0, F0 = _chain_case(0)
    assert np.array_equal(f[0], f0[0])
    assert rel(f, f0) <= 1e-13, rel(f, f0)
    for c in range(3):
        assert rel(F[c], F0[c]) <= 1e-13


def test_grouped_substep_fp64_matches_oracle(cuda_lib):
    """The grouped sub-step (interior markers, record hits and misses,
    inactive atoms, walls) against the oracle: per-atom forces within 1e-11,
    force field within 1e-12, over two LB cycles."""
    from oracle.bindings import OracleGrid
    n = (40, 32, 24)
    fg, Fg = _grouped_case("fp64", 8, n=n, cycles=2)
    rng = np.random.default_rng(19)
    x0 = rng.uniform(0.0, 1.0, (300, 3)) * np.array(n, float)
    x0[:20, 1] = rng.uniform(0.0, 2.5, 20)
    x0[20:40, 2] = n[2] - rng.uniform(0.0, 2.5, 20)
    v = 0.01 * rng.standard_normal((300, 3))
    m = rng.uniform(0.5, 1.5, 300)
    active = (np.arange(300) % 8 != 3).astype(np.int32)
    O = OracleGrid(3, *n, tau=0.7, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.01, 0, 0))
    O.set_f(cases.initial_populations(3, n, 7))
    ip = abi.IbmParams()
    ip.delta, ip.md_per_lb, ip.xi_ibm = 1, 2, 0.8
    ip.dt_lbm, ip.dx, ip.vel_scale, ip.force_scale = 1.0, 1.0, 1.0, 1.0
    x = x0.copy()
    fo = []
    for c in range(2):
        O.lbm_step((1e-5, 0.0, 2e-6))
        for s in range(2):
            if s > 0:
                x[::2, 0] += 0.6
            x = np.ascontiguousarray(np.mod(x + 0.3 * v, np.array(n, float)))
            fa = np.zeros_like(x)
            O.ibm_substep(ip, x, v, m, fa, active=active, refresh=(s == 0), fold=(s == 1))
            fo.append(fa)
    Fo = [cases.interior(a, 3) for a in O.get_force()]
    O.close()
    fo = np.stack(fo)
    assert rel(fg, fo) <= 1e-11, rel(fg, fo)
    for c in range(3):
        assert rel(Fg[c], Fo[c]) <= 1e-12, (c, rel(Fg[c], Fo[c]))
