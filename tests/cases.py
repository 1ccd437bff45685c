"""Seeded small problems run on the CPU oracles and on the GPU.

Inputs are rebuilt from the seeds every time; tests/golden/*.npz keep the
outputs of the reference build for the same inputs.  Arrays returned are the
interior nodes of the reference layout: populations (Q, nz, ny, nx), fields
(nz, ny, nx).
"""
import numpy as np

from couplb_b200 import abi

LB_CASES = {
    # 2D channel of the reference quick start (README.md:7-31), short
    "d2q9_poiseuille": dict(dim=2, n=(8, 32, 1), tau=0.8, wall=(0, 0, 1, 1, 0, 0), wall_vel=(0, 0, 0),
                            gravity=(5e-6, 0, 0), steps=200, seed=11, noise=0.0, force=False,
                            refresh_every=0),
    # every wall type on one 2D box, moving walls, initial force field, refreshes
    "d2q9_mixed": dict(dim=2, n=(9, 7, 1), tau=0.7, wall=(1, 2, 3, 4, 0, 0), wall_vel=(0.01, 0.02, 0),
                       gravity=(2e-5, -1e-5, 0), steps=30, seed=12, noise=1.0, force=True,
                       refresh_every=7),
    "d3q19_channel": dict(dim=3, n=(8, 6, 5), tau=0.65, wall=(0, 0, 1, 1, 1, 1), wall_vel=(0, 0, 0),
                          gravity=(1e-5, 0, 0), steps=50, seed=13, noise=1.0, force=False,
                          refresh_every=0),
    "d3q19_mixed": dict(dim=3, n=(7, 6, 5), tau=0.9, wall=(2, 3, 1, 4, 3, 2),
                        wall_vel=(0.01, -0.02, 0.005), gravity=(1e-5, 2e-6, -3e-6), steps=30, seed=14,
                        noise=1.0, force=True, refresh_every=4),
    "d3q19_periodic": dict(dim=3, n=(6, 5, 4), tau=0.55, wall=(0, 0, 0, 0, 0, 0), wall_vel=(0, 0, 0),
                           gravity=None, steps=40, seed=15, noise=1.0, force=True, refresh_every=0),
    "d3q19_open_x": dict(dim=3, n=(6, 5, 4), tau=0.75, wall=(4, 4, 0, 0, 2, 1),
                         wall_vel=(0.02, 0.0, 0.0), gravity=(0, 1e-5, 0), steps=25, seed=16, noise=1.0,
                         force=False, refresh_every=3),
}

IBM_CASES = {
    "d3_peskin_periodic": dict(dim=3, n=(10, 9, 8), tau=0.8, wall=(0,) * 6, wall_vel=(0, 0, 0),
                               delta=1, md_per_lb=2, xi=0.7, natoms=60, seed=21, subs=3),
    "d3_roma_walls": dict(dim=3, n=(10, 9, 8), tau=0.8, wall=(0, 0, 1, 2, 3, 4),
                          wall_vel=(0.01, 0, 0.02), delta=0, md_per_lb=3, xi=1.0, natoms=60, seed=22,
                          subs=4),
    "d3_peskin_walls": dict(dim=3, n=(9, 10, 8), tau=0.6, wall=(1, 3, 0, 0, 2, 2),
                            wall_vel=(0.0, 0.01, 0.0), delta=1, md_per_lb=1, xi=0.5, natoms=50, seed=23,
                            subs=2),
    "d2_peskin": dict(dim=2, n=(12, 10, 1), tau=0.8, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.02, 0, 0),
                      delta=1, md_per_lb=2, xi=0.8, natoms=30, seed=24, subs=3),
    "d2_roma_periodic": dict(dim=2, n=(11, 9, 1), tau=0.7, wall=(0,) * 6, wall_vel=(0, 0, 0),
                             delta=0, md_per_lb=1, xi=1.0, natoms=30, seed=25, subs=2),
}


def make_cfg(Nx, Ny, Nz, nu, rho, dimension=3, md_per_lb=1, xi_ibm=1.0, gravity=None, wall=(0,) * 6,
             wall_vel=(0.0,) * 3, delta=0, check_every=0, output_every=0, output_file="",
             precision=0, ibm_method=0, ibm_passes=5, slip_tol=0.0, mlp_model=""):
    c = abi.FixConfig()
    c.Nx, c.Ny, c.Nz, c.nu, c.rho = Nx, Ny, Nz, nu, rho
    c.md_per_lb, c.xi_ibm = md_per_lb, xi_ibm
    if gravity is not None:
        for d in range(3):
            c.gstyle[d] = abi.G_CONSTANT
            c.gconst[d] = gravity[d]
    for i in range(6):
        c.wall[i] = wall[i]
    for d in range(3):
        c.wall_vel[d] = wall_vel[d]
    c.delta = delta
    c.check_every = check_every
    c.output_every = output_every
    c.output_file = output_file.encode()
    c.precision = precision
    c.dimension = dimension
    c.ibm_method, c.ibm_passes, c.slip_tol = ibm_method, ibm_passes, slip_tol
    c.mlp_model = mlp_model.encode()
    return c


FIX_CASES = {
    # point particle pushed through a periodic box, sub-stepped (in.drag_point:25-55)
    "point_drag": dict(cmd=dict(Nx=12, Ny=12, Nz=12, nu=0.1, rho=1.0, md_per_lb=2, delta=0,
                                check_every=5),
                       dimension=3, box=((-6, -6, -6), (6, 6, 6)), dt=0.5, nsteps=40, seed=31,
                       natoms=1, fext=(1e-3, 0, 0)),
    # 2D channel with gravity and free markers (stale-density + IBM refresh path)
    "channel_markers": dict(cmd=dict(Nx=16, Ny=12, Nz=1, nu=0.1, rho=1.0, md_per_lb=3, delta=1,
                                     gravity=(2e-5, 0, 0), wall=(0, 0, 1, 1, 0, 0), check_every=4),
                            dimension=2, box=((0, 0, -0.5), (16, 12, 0.5)), dt=1.0 / 3.0, nsteps=30,
                            seed=32, natoms=8, fext=None),
    # physical units (dx != 1, rho != 1), like tests/subcycling/validate.sh:20-35
    "units_channel": dict(cmd=dict(Nx=12, Ny=10, Nz=1, nu=0.1, rho=1.26, md_per_lb=4, delta=0,
                                   gravity=(2e-4, 0, 0), wall=(0, 0, 1, 1, 0, 0), check_every=8),
                          dimension=2, box=((0, 0, -0.5), (7.5, 6.25, 0.5)), dt=0.08333 / 4,
                          nsteps=24, seed=33, natoms=3, fext=None, mass=0.161),
}

# IBM forcing methods at the fix level (no reference counterpart: checked
# against the port oracle only)
METHOD_FIX_CASES = {
    "cluster_iterative": dict(cmd=dict(Nx=16, Ny=14, Nz=12, nu=0.1, rho=1.0, md_per_lb=2, delta=0,
                                       gravity=(3e-5, 0, 0), ibm_method=1, ibm_passes=3,
                                       check_every=5),
                              dimension=3, box=((0, 0, 0), (16, 14, 12)), dt=0.5, nsteps=20,
                              seed=41, natoms=24, fext=None),
    # xi 0.3, mass 2: with xi 1 and mass 1 the Peskin4 overlap of this cluster
    # makes the correction gain exceed 2 and the passes diverge
    "cluster_iterative_peskin_walls": dict(cmd=dict(Nx=16, Ny=14, Nz=12, nu=0.1, rho=1.0, md_per_lb=1,
                                                    delta=1, gravity=(3e-5, 0, 0), ibm_method=1,
                                                    ibm_passes=4, wall=(0, 0, 1, 1, 0, 0), xi_ibm=0.3),
                                           dimension=3, box=((0, 0, 0), (16, 14, 12)), dt=1.0,
                                           nsteps=12, seed=42, natoms=24, fext=None, mass=2.0),
}


# ---------------------------------------------------------------------------
def ghost_shape(dim, n):
    nx, ny, nz = n
    return ((nz + 2) if dim == 3 else 1, ny + 2, nx + 2)


def interior(a, dim):
    """Interior nodes of a ghost-inclusive array (..., gz, gy, gx)."""
    if dim == 3:
        return a[..., 1:-1, 1:-1, 1:-1]
    return a[..., :, 1:-1, 1:-1]


def initial_populations(dim, n, seed, noise=1.0):
    """feq(rho, u) with random rho, u plus a non-equilibrium part (ghosts too)."""
    rng = np.random.default_rng(seed)
    sh = ghost_shape(dim, n)
    if dim == 3:
        E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                      [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1],
                      [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]], float)
        W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    else:
        E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [1, 1, 0], [-1, -1, 0],
                      [1, -1, 0], [-1, 1, 0]], float)
        W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    if noise == 0.0:
        rho = np.ones(sh)
        u = np.zeros((3,) + sh)
    else:
        rho = 1.0 + 0.01 * rng.standard_normal(sh)
        u = 0.02 * rng.standard_normal((3,) + sh)
    if dim == 2:
        u[2] = 0.0
    eu = np.einsum("qd,d...->q...", E, u)
    uu = (u * u).sum(0)
    f = W[:, None, None, None] * rho * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * uu)
    if noise:
        f = f + 1e-3 * W[:, None, None, None] * rng.standard_normal(f.shape)
    return np.ascontiguousarray(f)


def initial_force(dim, n, seed):
    rng = np.random.default_rng(seed + 1000)
    sh = ghost_shape(dim, n)
    return [1e-4 * rng.standard_normal(sh) for _ in range(3)]


def ibm_atoms(case):
    rng = np.random.default_rng(case["seed"])
    nx, ny, nz = case["n"]
    na = case["natoms"]
    hi = np.array([nx, ny, nz if case["dim"] == 3 else 1], float)
    x = rng.uniform(-0.6, 1.0, (na, 3)) * (hi + 1.2)
    x[: na // 6] = np.floor(x[: na // 6]) + 0.5      # exactly mid-cell in local coords
    x[na // 6: na // 3] = np.round(x[na // 6: na // 3])  # exactly on nodes
    if case["dim"] == 2:
        x[:, 2] = 0.0
    v = 0.01 * rng.standard_normal((na, 3))
    m = rng.uniform(0.5, 2.0, na)
    active = (rng.uniform(size=na) > 0.1).astype(np.int32)
    # per-substep displacement of the markers
    dxs = 0.05 * rng.standard_normal((case["subs"], na, 3))
    if case["dim"] == 2:
        dxs[..., 2] = 0
    return x, v, m, active, dxs


# ---------------------------------------------------------------------------
def run_lb_case_oracle(case, kind="port"):
    from oracle.bindings import OracleGrid
    dim, n = case["dim"], case["n"]
    G = OracleGrid(dim, *n, tau=case["tau"], wall=case["wall"], wall_vel=case["wall_vel"], kind=kind)
    G.set_f(initial_populations(dim, n, case["seed"], case["noise"]))
    if case["force"]:
        G.set_force(*initial_force(dim, n, case["seed"]))
    for s in range(1, case["steps"] + 1):
        G.lbm_step(case["gravity"])
        if case["refresh_every"] and s % case["refresh_every"] == 0:
            G.macroscopic(False)
    G.macroscopic(False)
    rho, ux, uy, uz = G.get_macro()
    return dict(f=interior(G.get_f(), dim), rho=interior(rho, dim), ux=interior(ux, dim),
                uy=interior(uy, dim), uz=interior(uz, dim))


def run_lb_case_gpu(case, precision="fp64"):
    from couplb_b200.lattice import Lattice
    dim, n = case["dim"], case["n"]
    L = Lattice(dim, *n, tau=case["tau"], wall=case["wall"], wall_vel=case["wall_vel"],
                body_force=case["gravity"] is not None, precision=precision)
    L.set_populations(initial_populations(dim, n, case["seed"], case["noise"]))
    if case["force"]:
        L.set_force_field(*initial_force(dim, n, case["seed"]))
    for s in range(1, case["steps"] + 1):
        L.lbm_step(case["gravity"])
        if case["refresh_every"] and s % case["refresh_every"] == 0:
            L.macroscopic()
    L.macroscopic()
    rho, ux, uy, uz = L.get_macroscopic()
    out = dict(f=interior(L.get_populations(), dim), rho=interior(rho, dim), ux=interior(ux, dim),
               uy=interior(uy, dim), uz=interior(uz, dim))
    L.close()
    return out


def _ibm_params(case):
    ip = abi.IbmParams()
    ip.delta, ip.md_per_lb, ip.xi_ibm = case["delta"], case["md_per_lb"], case["xi"]
    ip.dt_lbm, ip.dx, ip.vel_scale, ip.force_scale = 1.0, 1.0, 1.0, 1.0
    return ip


def run_ibm_case_oracle(case, kind="port"):
    from oracle.bindings import OracleGrid
    dim, n = case["dim"], case["n"]
    G = OracleGrid(dim, *n, tau=case["tau"], wall=case["wall"], wall_vel=case["wall_vel"], kind=kind)
    G.set_f(initial_populations(dim, n, case["seed"]))
    x, v, m, active, dxs = ibm_atoms(case)
    ip = _ibm_params(case)
    fs = []
    for s in range(case["subs"]):
        xs = np.ascontiguousarray(x + dxs[s])
        fa = np.zeros_like(x)
        G.ibm_substep(ip, xs, v, m, fa, active=active, refresh=(s == 0), fold=(s == case["subs"] - 1))
        fs.append(fa)
    fx, fy, fz = G.get_force()
    return dict(fatom=np.stack(fs), fx=interior(fx, dim), fy=interior(fy, dim), fz=interior(fz, dim))


def run_ibm_case_gpu(case, precision="fp64"):
    from couplb_b200.lattice import Lattice
    dim, n = case["dim"], case["n"]
    L = Lattice(dim, *n, tau=case["tau"], wall=case["wall"], wall_vel=case["wall_vel"],
                precision=precision)
    L.set_populations(initial_populations(dim, n, case["seed"]))
    x, v, m, active, dxs = ibm_atoms(case)
    L.set_ibm_params(delta=case["delta"], md_per_lb=case["md_per_lb"], xi_ibm=case["xi"])
    fs = []
    for s in range(case["subs"]):
        xs = np.ascontiguousarray(x + dxs[s])
        fa = np.zeros_like(x)
        L.ibm_substep(xs, v, m, fa, active=active, refresh=(s == 0))
        fs.append(fa)
    fx, fy, fz = L.get_force_field()
    out = dict(fatom=np.stack(fs), fx=interior(fx, dim), fy=interior(fy, dim), fz=interior(fz, dim))
    L.close()
    return out


def fix_atoms(case):
    from couplb_b200.md import Atoms
    rng = np.random.default_rng(case["seed"])
    lo, hi = np.array(case["box"][0], float), np.array(case["box"][1], float)
    na = case["natoms"]
    x = lo + (hi - lo) * rng.uniform(0.1, 0.9, (na, 3))
    v = 0.01 * rng.standard_normal((na, 3))
    if case["dimension"] == 2:
        x[:, 2] = 0.0
        v[:, 2] = 0.0
    mass = np.full(na, case.get("mass", 1.0))
    at = Atoms(x, v, mass)
    if case["fext"] is not None:
        at.fext = np.tile(np.array(case["fext"], float), (na, 1))
    return at


def run_fix_case(case, engine="port", precision=0):
    """Full fix sequencing through couplb_b200.md.run on one engine:
    'port' / 'ref' (CPU oracles) or 'gpu' (the CUDA fix core)."""
    from couplb_b200 import md
    cmd = dict(case["cmd"])
    cfg = make_cfg(dimension=case["dimension"], precision=precision, **cmd)
    lo, hi = case["box"]
    if engine in ("port", "ref"):
        from oracle.bindings import OracleFix
        dom = abi.make_domain(case["dimension"], lo, hi, case["dt"])
        fix = OracleFix(cfg, dom, kind=engine)
        grid = fix.grid
        diags = []

        def on_step(step):
            if cfg.check_every and step % cfg.check_every == 0:
                diags.append(fix.last_diag()[0])
    else:
        from couplb_b200.fix import FixCoupLB
        fix = FixCoupLB(cfg, dimension=case["dimension"])
        fix.init(lo, hi, case["dt"])
        grid = fix.lattice
        diags = []

        def on_step(step):
            if cfg.check_every and step % cfg.check_every == 0:
                d = fix.last_diag()
                diags.append(np.array([d.umax, d.mass, d.mom[0], d.mom[1], d.mom[2]]))
    at = fix_atoms(case)
    md.run(fix, at, case["nsteps"], case["dt"], on_step=on_step)
    dim = case["dimension"]
    if engine in ("port", "ref"):
        f = interior(grid.get_f(), dim)
    else:
        f = interior(grid.get_populations(), dim)
    out = dict(x=at.x.copy(), v=at.v.copy(), f_atoms=at.f.copy(), f=f,
               diag=np.array(diags) if diags else np.zeros((0, 5)))
    fix.close()
    return out
