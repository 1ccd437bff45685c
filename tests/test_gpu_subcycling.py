"""IBM sub-cycling against the reference's own acceptance test
(tests/subcycling/validate.sh:20-399), run through the fix hooks.

A 2D channel in physical units (96 x 64 nodes, dx 0.625, nu 0.1, rho 1.26,
gravity 2e-4, dt_LB 0.08333, walls on y) is spun up for 10000 LB steps and
checkpointed (validate.sh:79-102); three runs restart from the checkpoint
with one free particle (mass 0.161, v0 = (-0.3, 0), Roma kernel, velocity
Verlet) at md_per_lb 1, 4 and 10 for 2000 LB steps each (:104-290), sampling
the particle at setup and every 10 LB steps after.  The reference's four
checks (:306-399):

1. the particle ends moving downstream (vx > 0);
2. md_per_lb 4 and 10 follow md_per_lb 1 within 2 % in vx (samples after
   the fifth, |vx_ref| >= 0.01);
3. no drift across the channel (|vy| < 0.01);
4. the first sampled force is O(1) (0.1 < |fx| < 20).
"""
import numpy as np
import pytest

from couplb_b200 import md
from couplb_b200.fix import FixCoupLB

pytestmark = pytest.mark.gpu

DX, NX, NY = 0.625, 96, 64
DT_LB = 0.08333
BOX = ((0.0, 0.0, -0.5), (NX * DX, NY * DX, 0.5))
FLOW = f"flow all couplb {NX} {NY} 1 0.1 1.26 wall_y 1 1 gravity 2e-4 0.0 0.0 kernel roma"


def _track(pre, md_per_lb, lb_steps=2000, every=10):
    fix = FixCoupLB((FLOW + f" md_per_lb {md_per_lb} restart {pre}").split(), dimension=2)
    dt = DT_LB / md_per_lb
    fix.init(*BOX, dt)
    xc = (BOX[1][0] / 2, BOX[1][1] / 2, 0.0)
    at = md.Atoms([xc], v=[(-0.3, 0.0, 0.0)], mass=np.array([0.161]))
    rows = []

    def sample(step):
        if step % (every * md_per_lb) == 0:
            rows.append((at.v[0, 0], at.v[0, 1], at.f[0, 0]))

    # the first row is the setup step, as `fix print` writes it
    fix.setup(at.struct(), 0)
    sample(0)
    md.run(fix, at, lb_steps * md_per_lb, dt, setup=False, box=BOX, on_step=sample)
    fix.close()
    return np.array(rows)


def test_subcycling_follows_md_per_lb_1(cuda_lib, tmp_path):
    pre = str(tmp_path / "ckpt_pois")
    spin = FixCoupLB((FLOW + f" check_every 5000 checkpoint 10000 {pre}").split(), dimension=2)
    spin.init(*BOX, DT_LB)
    md.run(spin, md.empty_atoms(), 10000, DT_LB)
    spin.close()

    base = _track(pre, 1)
    assert base.shape == (201, 3)
    assert base[-1, 0] > 0.0                                # check 1
    for m in (4, 10):                                       # check 2
        t = _track(pre, m)
        assert t.shape == base.shape
        ref = base[5:, 0]
        keep = np.abs(ref) >= 0.01
        err = np.abs(t[5:, 0] - ref)[keep] / np.abs(ref)[keep]
        assert err.max() < 0.02, (m, err.max())
    assert np.abs(base[:, 1]).max() < 0.01                  # check 3
    assert 0.1 < abs(base[0, 2]) < 20.0                     # check 4
