"""The CPU oracle against the reference: golden vectors made by the
reference's own headers (tests/golden, oracle/_ref), direct comparison with
oracle/_ref where it is built, and the analytic solutions the reference's
validator uses (tests/poiseuille2d/validate.py:75-181)."""
import os

import numpy as np
import pytest

import cases
from oracle.bindings import OracleGrid, available

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(prefix, name):
    return dict(np.load(os.path.join(GOLDEN, f"{prefix}_{name}.npz")))


@pytest.mark.parametrize("name", sorted(cases.LB_CASES))
def test_lb_port_matches_golden(name):
    out = cases.run_lb_case_oracle(cases.LB_CASES[name], kind="port")
    ref = _golden("lb", name)
    for k in ref:
        np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{name}:{k}")


@pytest.mark.parametrize("name", sorted(cases.IBM_CASES))
def test_ibm_port_matches_golden(name):
    out = cases.run_ibm_case_oracle(cases.IBM_CASES[name], kind="port")
    ref = _golden("ibm", name)
    for k in ref:
        np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{name}:{k}")


@pytest.mark.parametrize("name", sorted(cases.FIX_CASES))
def test_fix_port_matches_golden(name):
    out = cases.run_fix_case(cases.FIX_CASES[name], engine="port")
    ref = _golden("fix", name)
    for k in ref:
        if k == "diag":
            # Grid::compute_diagnostics sums with an OpenMP reduction, whose
            # order depends on the thread count (couplb_lattice.h:226-229)
            np.testing.assert_allclose(out[k], ref[k], rtol=1e-13, atol=1e-300, err_msg=f"{name}:{k}")
        else:
            np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{name}:{k}")


@pytest.mark.skipif(not available("ref"), reason="reference sources not built here")
@pytest.mark.parametrize("seed", [101, 102, 103])
def test_port_matches_reference_build_random_walls(seed):
    """Random wall combinations, bit for bit against the reference headers."""
    rng = np.random.default_rng(seed)
    for dim in (2, 3):
        wall = tuple(int(w) for w in rng.integers(0, 5, 6))
        n = (int(rng.integers(3, 8)), int(rng.integers(3, 8)), int(rng.integers(3, 6)) if dim == 3 else 1)
        case = dict(dim=dim, n=n, tau=float(rng.uniform(0.52, 1.5)), wall=wall,
                    wall_vel=tuple(rng.uniform(-0.03, 0.03, 3)), gravity=tuple(rng.uniform(-1e-4, 1e-4, 3)),
                    steps=12, seed=seed, noise=1.0, force=True, refresh_every=5)
        a = cases.run_lb_case_oracle(case, kind="port")
        b = cases.run_lb_case_oracle(case, kind="ref")
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{case}:{k}")


def _channel_profile(kind, wall_hi, steps, g=None, uw=0.0, ny=32):
    G = OracleGrid(2, 8, ny, 1, tau=0.8, wall=(0, 0, 1, wall_hi, 0, 0), wall_vel=(uw, 0, 0), kind=kind)
    for _ in range(steps):
        G.lbm_step(g)
    G.macroscopic(False)
    ux = G.get_macro()[1][0, 1:-1, 1:-1]
    return ux.mean(axis=1)


def test_oracle_poiseuille_analytic():
    """README quick-start deck (8x32, nu=0.1, g=5e-6, 50000 steps): PASS of
    validate.py (max rel. error < 1 %, validate.py:99,111)."""
    g, nu, ny = 5e-6, 0.1, 32
    ux = _channel_profile("port", 1, 50000, g=(g, 0.0, 0.0), ny=ny)
    y = np.arange(ny, dtype=float)
    exact = g / (2 * nu) * (y + 0.5) * (ny - 0.5 - y)
    rel = np.abs(ux - exact).max() / exact.max()
    assert rel < 0.01, rel


def test_oracle_couette_analytic():
    """Moving top wall (type 2): u(y) = Uw (y + dx/2) / H (validate.py:132-153)."""
    uw, ny = 0.01, 16
    ux = _channel_profile("port", 2, 8000, uw=uw, ny=ny)
    y = np.arange(ny, dtype=float)
    exact = uw * (y + 0.5) / ny
    rel = np.abs(ux - exact).max() / uw
    assert rel < 0.01, rel
