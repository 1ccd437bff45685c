"""The fix core on the GPU: hook sequencing against the reference's golden
runs, the README quick-start Poiseuille deck through the profile output, and
checkpoint / restart."""
import os
import struct

import numpy as np
import pytest

import cases
from couplb_b200 import md
from couplb_b200.fix import FixCoupLB

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", sorted(cases.FIX_CASES))
def test_fix_sequence_matches_reference(cuda_lib, name):
    out = cases.run_fix_case(cases.FIX_CASES[name], engine="gpu")
    ref = dict(np.load(os.path.join(GOLDEN, f"fix_{name}.npz")))
    assert rel(out["f"], ref["f"]) <= 1e-12
    assert rel(out["f_atoms"], ref["f_atoms"]) <= 1e-11
    assert rel(out["x"], ref["x"]) <= 1e-13
    assert rel(out["v"], ref["v"]) <= 1e-11
    assert out["diag"].shape == ref["diag"].shape
    assert rel(out["diag"], ref["diag"]) <= 1e-11


def read_profile(path):
    blocks, cur = {}, None
    header = open(path).readline()
    for line in open(path):
        s = line.strip()
        if s.startswith("# step ="):
            cur = int(s.split("=")[1])
            blocks[cur] = []
        elif s and not s.startswith("#"):
            blocks[cur].append([float(t) for t in s.split()])
    return header, {k: np.array(v) for k, v in blocks.items()}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_quickstart_poiseuille_profile(cuda_lib, tmp_path, precision):
    """README.md:7-31 deck (8x32, nu 0.1, g 5e-6, wall_y 1 1, 50000 steps) with
    `output`: the validator criterion of tests/poiseuille2d/validate.py:99,111."""
    out = tmp_path / "prof.dat"
    fix = FixCoupLB(f"flow noatoms couplb 8 32 1 0.1 1.0 wall_y 1 1 gravity 5e-6 0.0 0.0 "
                    f"check_every 2000 output 10000 {out} precision {precision}".split(), dimension=2)
    fix.init(boxlo=(0, 0, -0.5), boxhi=(8, 32, 0.5), dt=1.0)
    md.run(fix, md.empty_atoms(), 50000, 1.0)
    header, blocks = read_profile(out)
    assert header.startswith("# H=Ny=32 tau=0.800000 nu=1.0000e-01 nu_lb=0.100000 rho=1.0000 kernel=roma")
    assert sorted(blocks) == [0, 10000, 20000, 30000, 40000, 50000]
    d = blocks[50000]
    y, ux = d[:, 2], d[:, 4]
    exact = 5e-6 / (2 * 0.1) * (y + 0.5) * (32 - 0.5 - y)
    assert np.abs(ux - exact).max() / exact.max() < 0.01
    assert any("CoupLB step 50000: Ma=" in m for m in fix.messages)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_poiseuille3d_profile(cuda_lib, tmp_path, precision):
    """tests/poiseuille3d/in.poiseuille3d (D3Q19 8x32x8, nu 0.1, g 5e-6,
    wall_y 1 1, x and z periodic, 50000 steps, profile every 5000) with the
    criterion of tests/poiseuille2d/validate.py:99,111 on the z-averaged
    profile (fix_couplb.cpp:903-979)."""
    out = tmp_path / "p3d.dat"
    fix = FixCoupLB(f"flow noatoms couplb 8 32 8 0.1 1.0 wall_y 1 1 gravity 5e-6 0.0 0.0 "
                    f"output 5000 {out} check_every 2000 precision {precision}".split(), dimension=3)
    fix.init(boxlo=(0, 0, 0), boxhi=(8, 32, 8), dt=1.0, periodicity=(1, 0, 1))
    md.run(fix, md.empty_atoms(), 50000, 1.0)
    header, blocks = read_profile(out)
    assert header.startswith("# H=Ny=32 tau=0.800000")
    assert sorted(blocks) == list(range(0, 50001, 5000))
    d = blocks[50000]
    y, ux, uy = d[:, 2], d[:, 4], d[:, 5]
    exact = 5e-6 / (2 * 0.1) * (y + 0.5) * (32 - 0.5 - y)
    assert np.abs(ux - exact).max() / exact.max() < 0.01
    assert np.abs(uy).max() < 1e-6 * exact.max()


def test_profile_matches_oracle_moments(cuda_lib, tmp_path):
    """Profile lines (fix_couplb.cpp:960-970) from the oracle's moments."""
    from oracle.bindings import OracleGrid
    out = tmp_path / "p.dat"
    fix = FixCoupLB(f"f all couplb 6 9 5 0.1 1.0 wall_y 1 2 wall_vel 0.02 0 0 gravity 1e-5 0 0 "
                    f"output 20 {out}".split(), dimension=3)
    fix.init(boxlo=(0, 0, 0), boxhi=(6, 9, 5), dt=1.0)
    md.run(fix, md.empty_atoms(), 20, 1.0)
    _, blocks = read_profile(out)
    G = OracleGrid(3, 6, 9, 5, tau=0.8, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.02, 0, 0))
    for _ in range(20):
        G.lbm_step((1e-5, 0, 0))
    G.macroscopic(False)
    rho, ux, uy, _ = [cases.interior(a, 3) for a in G.get_macro()]
    got = blocks[20]
    np.testing.assert_allclose(got[:, 3], rho.mean(axis=(0, 2)), rtol=1e-8)
    us = np.abs(ux).max()
    np.testing.assert_allclose(got[:, 4], ux.mean(axis=(0, 2)), rtol=1e-9, atol=1e-12 * us)
    np.testing.assert_allclose(got[:, 5], uy.mean(axis=(0, 2)), rtol=1e-9, atol=1e-12 * us)


def test_checkpoint_format_and_restart(cuda_lib, tmp_path):
    """couplb_io.h:660-829 layout; a restarted run continues bit for bit."""
    pre = str(tmp_path / "ck")
    args = "f all couplb 6 5 4 0.1 1.0 wall_z 1 2 wall_vel 0.01 0 0 gravity 1e-5 0 0".split()
    fix = FixCoupLB(args + ["checkpoint", "10", pre], dimension=3)
    fix.init(boxlo=(0, 0, 0), boxhi=(6, 5, 4), dt=1.0)
    md.run(fix, md.empty_atoms(), 10, 1.0)
    f10 = fix.lattice.get_populations()
    md.run(fix, md.empty_atoms(), 7, 1.0, start_step=10, setup=False)
    f17 = fix.lattice.get_populations()
    raw = open(pre + ".0.clbk", "rb").read()
    magic, ver, step, D, Q = struct.unpack_from("<IiqII", raw, 0)
    dims = struct.unpack_from("<9i", raw, 24)
    assert (magic, ver, step, D, Q) == (0x434C424B, 1, 10, 3, 19)
    assert dims == (6, 5, 4, 0, 0, 0, 6, 5, 4)
    fck = np.frombuffer(raw, dtype="<f8", offset=60)
    assert fck.size == 19 * 8 * 7 * 6
    np.testing.assert_array_equal(cases.interior(fck.reshape(19, 6, 7, 8), 3), cases.interior(f10, 3))

    fix2 = FixCoupLB(args + ["restart", pre], dimension=3)
    fix2.init(boxlo=(0, 0, 0), boxhi=(6, 5, 4), dt=1.0, ntimestep=10)
    md.run(fix2, md.empty_atoms(), 7, 1.0, start_step=10)
    np.testing.assert_array_equal(cases.interior(fix2.lattice.get_populations(), 3), cases.interior(f17, 3))


@pytest.mark.parametrize("body,msg", [
    (b"XXXX", "bad magic"),
    (struct.pack("<Ii", 0x434C424B, 2), "unsupported version 2"),
    (struct.pack("<Iiq", 0x434C424B, 1, 5) + struct.pack("<ii", 2, 9), "D/Q mismatch"),
    (struct.pack("<IiqII", 0x434C424B, 1, 5, 3, 19) + struct.pack("<9i", 6, 5, 5, 0, 0, 0, 6, 5, 4),
     "local grid mismatch"),
    (struct.pack("<IiqII", 0x434C424B, 1, 5, 3, 19) + struct.pack("<9i", 6, 5, 4, 0, 0, 0, 6, 5, 4)
     + b"\0" * 64, "short read"),
])
def test_corrupt_checkpoints_are_rejected(cuda_lib, tmp_path, body, msg):
    pre = str(tmp_path / "bad")
    open(pre + ".0.clbk", "wb").write(body)
    fix = FixCoupLB(f"f all couplb 6 5 4 0.1 1.0 restart {pre}".split(), dimension=3)
    with pytest.raises(Exception) as e:
        fix.init(boxlo=(0, 0, 0), boxhi=(6, 5, 4), dt=1.0)
    assert msg in str(e.value)


def test_init_errors(cuda_lib):
    fix = FixCoupLB("f all couplb 8 32 1 0.1 1.0".split(), dimension=2)
    with pytest.raises(Exception, match="non-cubic grid cells"):
        fix.init(boxlo=(0, 0, -0.5), boxhi=(8, 16, 0.5), dt=1.0)
    fix = FixCoupLB("f all couplb 8 32 1 0.001 1.0".split(), dimension=2)
    fix.init(boxlo=(0, 0, -0.5), boxhi=(8, 32, 0.5), dt=1e-3)
    assert any("tau very close to 0.5" in m for m in fix.messages)
    fix = FixCoupLB("f all couplb 8 32 1 0.1 1.0 wall_y 2 2 wall_vel 0.5 0 0".split(), dimension=2)
    with pytest.raises(Exception, match="wall Ma > 0.5"):
        fix.init(boxlo=(0, 0, -0.5), boxhi=(8, 32, 0.5), dt=1.0)
