"""IBM forcing methods and the correction network on the GPU, against the
CPU oracle's restatement (oracle/couplb_oracle.c, grid_ibm_substep_method and
mlp_*), and the FP64 network gradient against torch autograd.

Tolerances: iterative passes in FP64 storage, per-atom forces within 1e-10
relative and slip within 1e-9 relative (FP64 atomics reorder the field sums);
the network runs in FP32 with BF16 weights, so learned forces are compared
within 1e-5 of the largest force, and gradients within 1e-4 relative.
"""
import numpy as np
import pytest

import cases
from couplb_b200 import abi
from couplb_b200.lattice import Lattice
from couplb_b200.markers import fibonacci_sphere
from couplb_b200.mlp import CorrectionNet
from oracle import bindings as B

pytestmark = pytest.mark.gpu

N = (20, 18, 16)
G_LB = (2e-5, -1e-5, 0.5e-5)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def bf16(a):
    """Round float64 values to the nearest BF16 (ties to even)."""
    f = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def random_net(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    w = rng.normal(size=abi.MLP_NPARAM) * scale
    w[abi.MLP_NPARAM - 3:] *= 0.1
    return bf16(w)


def markers(seed=5):
    x = fibonacci_sphere(3.5, (10.3, 9.1, 7.8))
    rng = np.random.default_rng(seed)
    v = 0.004 * rng.standard_normal(x.shape)
    m = rng.uniform(0.5, 1.5, x.shape[0])
    return x, v, m


def make_pair(prec, delta, wall=(0, 0, 1, 1, 0, 0)):
    f0 = cases.initial_populations(3, N, 11)
    L = Lattice(3, *N, tau=0.8, wall=wall, body_force=True, precision=prec)
    L.set_populations(f0)
    O = B.OracleGrid(3, *N, 0.8, wall=wall)
    O.set_f(f0)
    ip = L.set_ibm_params(delta=delta, md_per_lb=1, xi_ibm=0.9)
    return L, O, ip


def run_steps(L, O, ip, method, passes, steps, slip_tol=0.0, net=None, w=None, s=(1.0, 1.0)):
    x, v, m = markers()
    out = []
    # the corrected velocity uses the body force of the last LB step
    L.lbm_step(G_LB)
    O.lbm_step(G_LB)
    for step in range(steps):
        fg = np.zeros_like(x)
        L.ibm_substep(x, v, m, fg, refresh=True)
        sl = L.ibm_slip()
        fo = np.zeros_like(x)
        _, st, _ = O.ibm_substep_method(ip, x, v, m, fo, method, passes, slip_tol=slip_tol,
                                        mlp=None if w is None else (w, s[0], s[1]), g_lb=G_LB)
        out.append((fg, fo, sl, st))
        L.lbm_step(G_LB)
        O.lbm_step(G_LB)
    return out


@pytest.mark.parametrize("resident", [1, 0])
@pytest.mark.parametrize("delta", ["roma", "peskin4"])
@pytest.mark.parametrize("passes", [1, 3, 5])
def test_iterative_matches_oracle_fp64(cuda_lib, delta, passes, resident):
    L, O, ip = make_pair("fp64", delta)
    L.set_option("ibm_resident", resident)
    L.set_ibm_method("iterative", passes=passes)
    for fg, fo, sl, st in run_steps(L, O, ip, 1, passes, 3):
        assert rel(fg, fo) <= 1e-10, rel(fg, fo)
        assert abs(sl["rms"] - st[2]) <= 1e-9 * st[2], (sl, st)
        assert abs(sl["max"] - st[3]) <= 1e-9 * st[3]
        assert sl["markers"] == st[5]
    L.close()


@pytest.mark.parametrize("resident", [1, 0])
def test_grid_barrier_timeout_returns_and_next_call_works(cuda_lib, resident):
    """The grid barriers of the cooperative sub-step kernel are bounded
    waits.  With a poll limit of 0 every block that is not the last to
    arrive gives up at once: the launch must end, count its timeouts and
    leave the handle usable.  With the default limit restored (and the state
    reset) the next sub-steps match the oracle again and count no timeout."""
    L, O, ip = make_pair("fp64", "peskin4")
    L.set_option("ibm_resident", resident)
    L.set_ibm_method("iterative", passes=3)
    default = L.get_option("barrier_spin")
    assert default > 0 and L.get_option("timeouts") == 0
    x, v, m = markers()
    assert x.shape[0] > 8            # more than one block of eight marker warps
    L.set_option("barrier_spin", 0)
    L.lbm_step(G_LB)
    L.ibm_substep(x, v, m, np.zeros_like(x), refresh=True)
    t = L.get_option("timeouts")
    assert t > 0
    # restore the state (the timed-out sub-step left partial spreads behind)
    L.set_option("barrier_spin", default)
    z = np.zeros(L.G)
    L.set_force_field(z, z, z)
    L.set_populations(cases.initial_populations(3, N, 11))
    for fg, fo, sl, st in run_steps(L, O, ip, 1, 3, 2):
        assert rel(fg, fo) <= 1e-10, rel(fg, fo)
    assert L.get_option("timeouts") == t
    L.close()


def test_iterative_reduces_slip(cuda_lib):
    """Fixed sphere in a uniform stream: each correction pass lowers the slip."""
    x, _, _ = markers()
    rms = []
    for passes in (1, 2, 5):
        L = Lattice(3, *N, tau=0.8)
        L.init_equilibrium(1.0, 0.01, 0.002, 0.0)
        L.set_ibm_params(delta="roma", md_per_lb=1, xi_ibm=1.0)
        L.set_ibm_method("iterative", passes=passes)
        L.ibm_substep(x, np.zeros_like(x), np.ones(x.shape[0]), np.zeros_like(x), refresh=True)
        rms.append(L.ibm_slip()["rms"])
        L.close()
    assert rms[1] < 0.85 * rms[0] and rms[2] < 0.5 * rms[0], rms


def test_iterative_fp32_close_to_oracle(cuda_lib):
    L, O, ip = make_pair("fp32", "roma")
    L.set_ibm_method("iterative", passes=5)
    for fg, fo, sl, st in run_steps(L, O, ip, 1, 5, 2):
        assert rel(fg, fo) <= 2e-5, rel(fg, fo)
        assert abs(sl["rms"] - st[2]) <= 1e-3 * st[2]
    L.close()


@pytest.mark.parametrize("delta", ["roma", "peskin4"])
@pytest.mark.parametrize("resident", [1, 0])
@pytest.mark.parametrize("tol,fell", [(1e9, 0), (0.0, 1)])
def test_learned_matches_oracle(cuda_lib, tol, fell, resident, delta):
    L, O, ip = make_pair("fp64", delta)
    L.set_option("ibm_resident", resident)
    w = random_net(3)
    s = (250.0, 400.0)
    net = CorrectionNet(0, seed=1)
    net.set_weights(w.astype(np.float32), *s)
    L.set_ibm_method("learned", passes=4, slip_tol=tol, model=net)
    for fg, fo, sl, st in run_steps(L, O, ip, 2, 4, 2, slip_tol=tol, w=w, s=s):
        assert rel(fg, fo) <= 1e-5, rel(fg, fo)
        assert sl["fell_back"] == fell == st[4]
        assert abs(sl["check_rms"] - st[0]) <= 1e-4 * st[0]
        assert abs(sl["rms"] - st[2]) <= 1e-4 * st[2]
    assert L.ibm_slip(reset=True)["checks"] == 2
    assert L.ibm_slip()["checks"] == 0
    L.close()
    net.close()


@pytest.mark.parametrize("resident", [1, 0])
def test_learned_without_fallback_runs_no_check(cuda_lib, resident):
    """slip_tol inf: the learned sub-step cannot fall back, so it runs no
    slip check (no count, no grid barrier before the statistics); its forces
    are those of a learned sub-step that never falls back and its slip after
    the last pass is the oracle's."""
    L, O, ip = make_pair("fp64", "peskin4")
    L.set_option("ibm_resident", resident)
    w = random_net(3)
    s = (250.0, 400.0)
    net = CorrectionNet(0, seed=1)
    net.set_weights(w.astype(np.float32), *s)
    L.set_ibm_method("learned", passes=4, slip_tol=float("inf"), model=net)
    for fg, fo, sl, st in run_steps(L, O, ip, 2, 4, 2, slip_tol=1e300, w=w, s=s):
        assert rel(fg, fo) <= 1e-5, rel(fg, fo)
        assert sl["fell_back"] == 0 == st[4]
        assert abs(sl["rms"] - st[2]) <= 1e-4 * st[2]
    assert L.ibm_slip()["checks"] == 0
    L.close()
    net.close()


@pytest.mark.parametrize("resident", [1, 0])
def test_slip_statistics_off_keeps_the_forces(cuda_lib, resident):
    """Handle option ibm_slip 0: the iterative sub-step skips the slip
    measurement after its last pass (no markers counted) and its forces still
    match the oracle."""
    L, O, ip = make_pair("fp64", "roma")
    L.set_option("ibm_resident", resident)
    L.set_ibm_method("iterative", passes=3)
    L.set_option("ibm_slip", 0)
    assert L.get_option("ibm_slip") == 0
    for fg, fo, sl, st in run_steps(L, O, ip, 1, 3, 2):
        assert rel(fg, fo) <= 1e-10, rel(fg, fo)
        assert sl["markers"] == 0
    L.close()


@pytest.mark.parametrize("resident", [1, 0])
def test_record_rows_match_oracle(cuda_lib, resident):
    import torch
    L, O, ip = make_pair("fp64", "roma", wall=(0,) * 6)
    L.set_option("ibm_resident", resident)
    L.set_ibm_method("iterative", passes=3)
    x, v, m = markers()
    n = x.shape[0]
    buf = torch.zeros((3 * n, abi.MLP_ROW), dtype=torch.float32, device="cuda")
    L.ibm_record(buf.data_ptr(), 2 * n + 5)
    rows_o = []
    for step in range(3):
        L.ibm_substep(x, v, m, np.zeros_like(x), refresh=True)
        _, _, r = O.ibm_substep_method(ip, x, v, m, np.zeros_like(x), 1, 3, g_lb=(0, 0, 0),
                                       rows=True)
        rows_o.append(r)
        L.lbm_step(None)
        O.lbm_step(None)
    L.synchronize()
    assert L.ibm_record_count() == 2 * n   # the third sub-step would overflow
    got = buf.cpu().numpy().astype(np.float64)
    ref = np.concatenate(rows_o[:2])
    assert np.abs(got[:2 * n, :84] - ref[:, :84]).max() <= 1e-6 * np.abs(ref[:, :84]).max()
    assert rel(got[:2 * n, 84:87], ref[:, 84:87]) <= 1e-5
    assert not got[2 * n:].any()
    L.close()


def _rows(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, abi.MLP_ROW))
    r[:, :84] = 0.01 * rng.standard_normal((n, 84))
    r[:, 84:87] = 0.003 * rng.standard_normal((n, 3))
    return r


def test_network_forward_and_gradient_vs_oracle(cuda_lib):
    import torch
    w = random_net(9, 0.2)
    s_in, s_out = 80.0, 300.0
    rows = _rows(300, 2)        # 300 rows: four full tiles and a partial one
    net = CorrectionNet(0, seed=2)
    net.set_weights(w.astype(np.float32), s_in, s_out)
    d = torch.from_numpy(rows.astype(np.float32)).cuda()
    rows32 = d.cpu().numpy().astype(np.float64)
    out = torch.zeros((300, 3), dtype=torch.float32, device="cuda")
    net.forward(d.data_ptr(), 300, out.data_ptr())
    torch.cuda.synchronize()
    yo = B.mlp_forward(w, s_in, s_out, rows32[:, :84])
    assert rel(out.cpu().numpy(), yo) <= 1e-5
    loss, g = net.loss_grad(d.data_ptr(), 300)
    lo, go = B.mlp_loss_grad(w, s_in, s_out, rows32)
    assert abs(loss - lo) <= 1e-5 * lo
    assert rel(g.astype(np.float64), go) <= 1e-4, rel(g.astype(np.float64), go)
    # the oracle's FP64 gradient against torch autograd
    tw = torch.tensor(w, requires_grad=True)
    W1, b1 = tw[:5376].view(64, 84), tw[5376:5440]
    W2, b2 = tw[5440:9536].view(64, 64), tw[9536:9600]
    W3, b3 = tw[9600:9792].view(3, 64), tw[9792:]
    x = torch.tensor(rows32[:, :84]) * s_in
    y = torch.relu(torch.relu(x @ W1.T + b1) @ W2.T + b2) @ W3.T + b3
    L = ((y - s_out * torch.tensor(rows32[:, 84:87])) ** 2).sum() / (3 * 300)
    L.backward()
    assert rel(go, tw.grad.numpy()) <= 1e-12
    net.close()


def test_network_training_fits_a_linear_map(cuda_lib):
    import torch
    rng = np.random.default_rng(4)
    n = 40000
    rows = _rows(n, 5)
    A = 0.1 * rng.standard_normal((3, 84))
    rows[:, 84:87] = rows[:, :84] @ A.T
    d = torch.from_numpy(rows.astype(np.float32)).cuda()
    net = CorrectionNet(0, seed=3)
    net.fit_scales(d.data_ptr(), n)
    l0, _ = net.loss_grad(d.data_ptr(), n)
    tl, vl = net.train(d.data_ptr(), n, epochs=15, batch=1024, lr=3e-3, n_val=4000)
    assert tl < 0.05 * l0 and vl < 0.08 * l0, (l0, tl, vl)
    w, si, so = net.get_weights()
    assert np.isfinite(w).all() and si > 0 and so > 0
    net.close()


def test_network_save_load(cuda_lib, tmp_path):
    net = CorrectionNet(0, seed=5)
    w, si, so = net.get_weights()
    p = tmp_path / "net.clbmlp"
    net.save(p)
    other = CorrectionNet(0, seed=6)
    other.load(p)
    w2, si2, so2 = other.get_weights()
    assert np.array_equal(w, w2) and (si, so) == (si2, so2)
    p.write_bytes(b"CLBMLP01" + b"\0" * 10)
    with pytest.raises(Exception):
        other.load(p)
    net.close()
    other.close()


def test_method_errors(cuda_lib):
    from couplb_b200.lib import CoupLBError
    L = Lattice(3, 8, 8, 8, tau=0.8)
    L.set_ibm_params(delta="peskin4")
    with pytest.raises(CoupLBError):
        L.set_ibm_method("learned", passes=5)            # no network
    with pytest.raises(CoupLBError):
        L.set_ibm_method("iterative", passes=0)
    net = CorrectionNet(0)
    L.set_ibm_method("learned", passes=5, slip_tol=1e-3, model=net)
    L2 = Lattice(2, 8, 8, tau=0.8)
    with pytest.raises(CoupLBError):
        L2.set_ibm_method("learned", passes=5, model=net)
    L.close()
    L2.close()
    net.close()


def test_trained_network_gains_over_single_pass(cuda_lib):
    """Rows from 5-pass iterative runs of a small sphere train the network on
    the GPU; on an unseen sub-cell offset the learned correction removes most
    of the slip the single penalty pass leaves, and the check passes without
    falling back at 1.5x the iterative slip."""
    from couplb_b200 import sphere_drag as SD
    kw = dict(n=48, radius=6.0, g=4e-6)
    rows = SD.generate_rows(4, 400, 2, **{k: kw[k] for k in ("n", "radius")})
    assert rows.shape[0] == 4 * 200 * 452
    net, tl, vl = SD.train_net(rows, epochs=25, batch=2048)
    assert vl < 0.2, (tl, vl)
    slip = {}
    for name, m in [("single", dict(method="iterative", passes=1)),
                    ("iter5", dict(method="iterative", passes=5)),
                    ("learned", dict(method="learned", passes=5, slip_tol=1e30, net=net))]:
        c = SD.SphereCase(offset=(0.37, 0.61, 0.23), **kw)
        c.set_method(**m)
        sl, _ = c.run(400, slip_from=300)
        slip[name] = float(np.mean(sl))
        c.close()
    assert slip["learned"] < 0.3 * slip["single"], slip
    assert slip["learned"] < 1.5 * slip["iter5"], slip
    c = SD.SphereCase(offset=(0.37, 0.61, 0.23), **kw)
    c.set_method("learned", passes=5, slip_tol=1.5 * slip["iter5"], net=net)
    c.run(400)
    d = c.L.ibm_slip()
    assert d["checks"] == 400 and d["fallbacks"] <= 40, d
    c.close()
    net.close()


@pytest.mark.parametrize("name", sorted(cases.METHOD_FIX_CASES))
def test_fix_method_matches_port(cuda_lib, name):
    """`fix couplb ... ibm_method iterative ibm_passes N` through the fix hooks
    against the port oracle's fix sequencing (atoms move, sub-steps fold)."""
    case = cases.METHOD_FIX_CASES[name]
    ref = cases.run_fix_case(case, "port")
    out = cases.run_fix_case(case, "gpu")
    assert rel(out["f_atoms"], ref["f_atoms"]) <= 1e-10, rel(out["f_atoms"], ref["f_atoms"])
    assert rel(out["x"], ref["x"]) <= 1e-12
    assert np.abs(out["f"] - ref["f"]).max() <= 1e-12


@pytest.mark.parametrize("slip_tol", [0.0, 1e-12])
def test_fix_learned_matches_port(cuda_lib, tmp_path, slip_tol):
    """`ibm_method learned mlp_model FILE`: never falling back (slip_tol 0)
    and always falling back (slip_tol 1e-12)."""
    net = CorrectionNet(0, seed=8)
    net.set_weights(random_net(12, 0.2).astype(np.float32), 150.0, 300.0)
    path = tmp_path / "net.clbmlp"
    net.save(path)
    net.close()
    case = dict(cases.METHOD_FIX_CASES["cluster_iterative"])
    case["cmd"] = dict(case["cmd"], ibm_method=2, ibm_passes=3, slip_tol=slip_tol, mlp_model=str(path))
    ref = cases.run_fix_case(case, "port")
    out = cases.run_fix_case(case, "gpu")
    # FP32 network inside 20 coupled MD steps: differences grow with the dynamics
    assert rel(out["f_atoms"], ref["f_atoms"]) <= 1e-4, rel(out["f_atoms"], ref["f_atoms"])
    assert rel(out["x"], ref["x"]) <= 1e-6


@pytest.mark.parametrize("delta", ["roma", "peskin4"])
def test_iterative_2d_matches_oracle(cuda_lib, delta):
    """D2Q9 (general form of the cooperative kernel): a ring of markers in a
    channel with no-slip walls on y, 3 passes, against the port oracle."""
    n2 = (24, 18, 1)
    f0 = cases.initial_populations(2, n2, 13)
    wall = (0, 0, 1, 1, 0, 0)
    L = Lattice(2, 24, 18, tau=0.8, wall=wall, body_force=True)
    L.set_populations(f0)
    O = B.OracleGrid(2, 24, 18, 1, 0.8, wall=wall)
    O.set_f(f0)
    ip = L.set_ibm_params(delta=delta, md_per_lb=1, xi_ibm=0.8)
    L.set_ibm_method("iterative", passes=3)
    th = np.linspace(0, 2 * np.pi, 20, endpoint=False)
    x = np.stack([12.2 + 4 * np.cos(th), 9.1 + 4 * np.sin(th), np.zeros_like(th)], 1)
    v = np.zeros_like(x)
    m = np.ones(len(x))
    g2 = (2e-5, 0.0, 0.0)
    L.lbm_step(g2)
    O.lbm_step(g2)
    for step in range(3):
        fg = np.zeros_like(x)
        L.ibm_substep(x, v, m, fg, refresh=True)
        sl = L.ibm_slip()
        fo = np.zeros_like(x)
        _, st, _ = O.ibm_substep_method(ip, x, v, m, fo, 1, 3, g_lb=g2)
        assert rel(fg, fo) <= 1e-10, rel(fg, fo)
        assert abs(sl["rms"] - st[2]) <= 1e-9 * st[2]
        L.lbm_step(g2)
        O.lbm_step(g2)
    L.close()
