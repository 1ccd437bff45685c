"""The reference's two drag decks run through the fix hooks: a point force
(tests/drag_forces_point/in.drag_point) and a rigid sphere against
Hasimoto's periodic-array correction (tests/drag_forces_sphere/in.drag_sphere).

Sphere deck: 96^3 cells of dx 0.5 (L = 48), nu 0.1, rho 1, Roma kernel, dt 0.25; a sphere
of radius 3 carried by 162 markers of total mass 50, pushed by a total force
0.005 along x (`fix addforce`), moving as one rigid body (`fix rigid/nve
single`: the summed force drives the body's velocity, every marker gets it),
and a compensating body force -F / (rho L^3) on the fluid.  After 30000
steps the body's velocity is compared with U_Stokes K(R/L), K = 1 - 2.837 R/L
+ 4.19 (R/L)^3 (in.drag_sphere:46-66).  The deck has no pass threshold; the
markers here are a Fibonacci spiral (the deck reads an icosahedral set), and
the test holds the error within 15 % and the cross-flow velocity small.
"""
import numpy as np
import pytest

from couplb_b200 import md
from couplb_b200.fix import FixCoupLB
from couplb_b200.markers import fibonacci_sphere

pytestmark = pytest.mark.gpu


def test_rigid_sphere_terminal_velocity_vs_hasimoto(cuda_lib):
    nc, dxp, radius, nm = 96, 0.5, 3.0, 162
    L = nc * dxp
    f_total, m_total, dt, steps = 0.005, 50.0, 0.25, 30000
    g_comp = -f_total / (1.0 * L ** 3)
    fix = FixCoupLB(f"flow sphere couplb {nc} {nc} {nc} 0.1 1.0 kernel roma "
                    f"gravity {g_comp!r} 0.0 0.0 check_every 2000".split(), dimension=3)
    fix.init((0.0, 0.0, 0.0), (L, L, L), dt)
    at = md.Atoms(fibonacci_sphere(radius, (L / 2, L / 2, L / 2), n=nm), mass=np.full(nm, m_total / nm))
    st = at.struct()
    V = np.zeros(3)

    def forces(step, setup=False):
        at.f[:] = 0.0
        at.f[:, 0] = f_total / nm           # fix addforce, before fix couplb
        if setup:
            fix.setup(st, step)
        else:
            fix.post_force(st, step)
        return at.f.sum(axis=0)

    F = forces(0, setup=True)
    for step in range(1, steps + 1):
        # velocity Verlet of the body's centre of mass (no torque on the
        # symmetric body, so no rotation)
        V += 0.5 * dt * F / m_total
        at.x += dt * V
        at.x[:] = np.mod(at.x, L)
        at.v[:] = V
        F = forces(step)
        V += 0.5 * dt * F / m_total
        at.v[:] = V
        fix.end_of_step(step)
    d = fix.last_diag()
    fix.close()
    assert d.nonfinite == 0 and d.clamps == 0
    a = radius / L
    u_corr = f_total / (6.0 * np.pi * 0.1 * radius) * (1.0 - 2.837 * a + 4.19 * a ** 3)
    err = (V[0] - u_corr) / u_corr
    print(f"U measured {V[0]:.6e}, Hasimoto {u_corr:.6e}, error {100 * err:.2f} %")
    assert abs(err) < 0.15, err
    assert abs(V[1]) < 1e-2 * V[0] and abs(V[2]) < 1e-2 * V[0]


def test_point_force_drag_deck(cuda_lib):
    """tests/drag_forces_point/in.drag_point: one particle (mass 1) at the
    centre of a periodic 32^3 box (nu 0.1, Roma), pushed by a constant 1e-3
    along x for 10000 steps (fix addforce + fix nve).  The deck's checks:
    v_y and v_z stay at machine zero (< 1e-8), v_x ends positive and steady,
    the mass is constant with no density clamps and Ma < 0.1; and its
    physics notes: at steady state the IBM drag balances the push (Newton 3)
    and the total momentum (fluid + particle) grows linearly at the push."""
    fix = FixCoupLB("flow all couplb 32 32 32 0.1 1.0 kernel roma check_every 500".split(), dimension=3)
    fix.init((-16.0,) * 3, (16.0,) * 3, 1.0)
    at = md.Atoms([(0.0, 0.0, 0.0)], mass=np.array([1.0]))
    at.fext = np.array([[1e-3, 0.0, 0.0]])
    rows = []

    def on_step(step):
        if step % 500 == 0:
            d = fix.last_diag()
            rows.append((step, *at.v[0], at.f[0, 0], d.mom[0], d.mass, d.umax, d.clamps))

    md.run(fix, at, 10000, 1.0, box=((-16.0,) * 3, (16.0,) * 3), on_step=on_step)
    fix.close()
    r = np.array(rows)
    step, vx, vy, vz, ftot, pf, mass, umax, clamps = r.T
    assert np.abs(vy).max() < 1e-8 and np.abs(vz).max() < 1e-8
    assert vx[-1] > 0 and abs(vx[-1] - vx[-5]) < 0.1 * vx[-1]       # 8000 -> 10000
    assert np.all(clamps == 0) and np.abs(mass - mass[0]).max() < 1e-12 * mass[0]
    assert umax.max() / 3 ** -0.5 < 0.1
    assert abs(ftot[-1]) < 1e-2 * 1e-3                               # drag = push
    p = pf + 1.0 * vx                                                # fluid + particle
    slope = (p[-1] - p[9]) / (step[-1] - step[9])                    # 5000 -> 10000
    assert abs(slope - 1e-3) < 1e-3 * 1e-3, slope
