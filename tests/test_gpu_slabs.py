"""Slab decomposition along z on the GPU: a lattice run as 2 or 3 z slabs
(halo faces packed and attached after every LB step, couplb_halo_pack /
couplb_halo_attach) steps exactly like the whole lattice -- the same
arithmetic per node, only the source of the crossing populations differs --
so populations and moments agree bit for bit, FP64 and FP32-shifted, with a
periodic z or walls on the z faces, moving walls and a body force."""
import numpy as np
import pytest

import cases
from couplb_b200.lattice import Lattice
from couplb_b200.lib import CoupLBError
from couplb_b200.slabs import SlabLattice

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("nslab", [2, 3])
@pytest.mark.parametrize("wall", [(0, 0, 1, 1, 0, 0), (0, 0, 1, 2, 3, 1), (0,) * 6])
def test_slabs_step_like_the_whole_lattice(cuda_lib, prec, nslab, wall):
    n = (24, 14, 19)
    f0 = cases.initial_populations(3, n, 17)
    kw = dict(tau=0.7, wall=wall, wall_vel=(0.02, 0.0, 0.01), body_force=True, precision=prec)
    L = Lattice(3, *n, **kw)
    L.set_populations(f0)
    S = SlabLattice(*n, nslab, **kw)
    S.set_populations(f0)
    g = (1e-5, -2e-6, 3e-6)
    for _ in range(12):
        L.lbm_step(g)
        S.lbm_step(g)
    np.testing.assert_array_equal(S.get_populations(), L.get_populations()[:, 1:-1, 1:-1, 1:-1])
    L.macroscopic()
    want = [a[1:-1, 1:-1, 1:-1] for a in L.get_macroscopic()]
    for got, ref in zip(S.get_macroscopic(), want):
        np.testing.assert_array_equal(got, ref)
    d = L.diagnostics()
    umax, mass, mom = S.diagnostics()
    assert umax == d.umax
    assert abs(mass - d.mass) <= 1e-12 * d.mass
    L.close()
    S.close()


def test_halo_face_rules(cuda_lib):
    L = Lattice(3, 8, 6, 5, tau=0.8, wall=(0, 0, 0, 0, 1, 0))
    import torch
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(CoupLBError):     # the z-low face is a wall
        L._ck(L.L.couplb_halo_attach(L.h, 0, dummy.data_ptr()))
    buf = torch.zeros(int(L.L.couplb_halo_bytes(L.h)), dtype=torch.uint8, device="cuda")
    assert buf.numel() == 5 * 8 * 6 * 8
    with pytest.raises(CoupLBError):     # post-stream state: nothing to pack yet
        L._ck(L.L.couplb_halo_pack(L.h, 1, buf.data_ptr()))
    L._ck(L.L.couplb_halo_attach(L.h, 1, buf.data_ptr()))
    L.set_ibm_params(delta="peskin4")
    x = np.array([[4.0, 3.0, 2.5]])
    with pytest.raises(CoupLBError):     # a halo face without its IBM halo
        L.ibm_substep(x, np.zeros_like(x), np.ones(1), np.zeros_like(x))
    nb = int(L.L.couplb_ibm_halo_bytes(L.h, 2))
    assert nb == 2 * 8 * 6 * 4 * 8
    vel = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    frc = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    with pytest.raises(CoupLBError):     # the low face is a wall
        L._ck(L.L.couplb_ibm_halo_attach(L.h, 0, 1, vel.data_ptr(), frc.data_ptr()))
    with pytest.raises(CoupLBError):     # at most 2 planes above
        L._ck(L.L.couplb_ibm_halo_attach(L.h, 1, 3, vel.data_ptr(), frc.data_ptr()))
    L._ck(L.L.couplb_ibm_halo_attach(L.h, 1, 2, vel.data_ptr(), frc.data_ptr()))
    L.ibm_substep(x, np.zeros_like(x), np.ones(1), np.zeros_like(x))
    L.set_ibm_method("iterative", passes=2)
    with pytest.raises(CoupLBError):     # the correction methods are single-slab
        L.ibm_substep(x, np.zeros_like(x), np.ones(1), np.zeros_like(x))
    L.close()


def _slab_markers(n, nslab, seed=23):
    """Markers across the box, a third of them within two cells of a slab
    face (internal faces and the global z faces)."""
    from couplb_b200.slabs import partition
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, (240, 3)) * np.array(n, float)
    faces = [z0 for z0, _ in partition(n[2], nslab)] + [n[2]]
    for k in range(80):
        x[k, 2] = (faces[k % len(faces)] + rng.uniform(-2.0, 2.0)) % n[2]
    v = 0.01 * rng.standard_normal(x.shape)
    m = rng.uniform(0.5, 1.5, x.shape[0])
    return x, v, m


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("nslab", [2, 3])
@pytest.mark.parametrize("window", [0, 1])
@pytest.mark.parametrize("wall", [(0, 0, 1, 2, 0, 0), (0, 0, 0, 0, 1, 1)])
@pytest.mark.parametrize("idle", [False, True])
def test_ibm_on_slabs_matches_the_whole_lattice(cuda_lib, prec, tol, nslab, window, wall, idle):
    """IBM sub-steps on z slabs (halo moments after every LB step, spread
    forces folded into the neighbours before the next): the per-atom forces,
    the force field and the populations of the whole lattice, over three LB
    cycles of two sub-steps, markers near every slab face, clipped and
    wrapped windows."""
    n = (20, 14, 19)
    f0 = cases.initial_populations(3, n, 5)
    kw = dict(tau=0.75, wall=wall, wall_vel=(0.01, 0.0, 0.0), body_force=True, precision=prec)
    ibm = dict(delta="peskin4", md_per_lb=2, xi_ibm=0.8)
    L = Lattice(3, *n, **kw)
    L.set_option("ibm_window", window)
    L.set_populations(f0)
    L.set_ibm_params(**ibm)
    S = SlabLattice(*n, nslab, **kw)
    S.set_option("ibm_window", window)
    S.set_populations(f0)
    S.set_ibm_params(**ibm)
    x0, v, m = _slab_markers(n, nslab)
    if idle:
        # markers in the lowest few planes only: the other slabs refresh
        # without markers of their own
        x0[:, 2] = np.mod(x0[:, 2], 3.0)
    g = (1e-5, 0.0, 2e-6)
    box = np.array(n, float)
    x = x0.copy()
    for c in range(3):
        L.lbm_step(g)
        S.lbm_step(g)
        for s in range(2):
            x = np.ascontiguousarray(np.mod(x + 0.5 * v, box))
            fl, fs = np.zeros_like(x), np.zeros_like(x)
            L.ibm_substep(x, v, m, fl, refresh=(s == 0))
            S.ibm_substep(x, v, m, fs, refresh=(s == 0))
            assert rel(fs, fl) <= tol, (c, s, rel(fs, fl))
    FL = [a[1:-1, 1:-1, 1:-1] for a in L.get_force_field()]
    for c, a in enumerate(S.get_force_field()):
        assert rel(a, FL[c]) <= tol, (c, rel(a, FL[c]))
    L.lbm_step(g)
    S.lbm_step(g)
    assert rel(S.get_populations(), L.get_populations()[:, 1:-1, 1:-1, 1:-1]) <= tol
    L.close()
    S.close()


def _rank_ibm(rank, world, port, window, prefix, out):
    """One rank of the gloo test below: a RankSlab on cuda:0, its own
    markers, the same cycles as the whole lattice."""
    import datetime
    import os
    import torch.distributed as dist
    from couplb_b200.slabs import RankSlab, owner_slabs, partition
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n, f0, kw, ibm, x, v, m, g = _rank_case(world)
        S = RankSlab(dist, *n, device=0, **kw)
        S.L.set_option("ibm_window", window)
        S.set_populations(f0)
        S.set_ibm_params(**ibm)
        parts = partition(n[2], world)
        forces = []
        for c in range(3):
            S.lbm_step(g)
            for s in range(2):
                x = np.ascontiguousarray(np.mod(x + 0.5 * v, np.array(n, float)))
                mine = np.nonzero(owner_slabs(x[:, 2], parts) == rank)[0]
                f = np.zeros((mine.size, 3))
                S.ibm_substep(np.ascontiguousarray(x[mine]), np.ascontiguousarray(v[mine]),
                              np.ascontiguousarray(m[mine]), f, refresh=(s == 0))
                forces.append((mine, f))
        F = S.get_force_field()
        S.lbm_step(g)
        pops = S.get_populations()
        prof = S.y_profile()
        # a per-rank checkpoint restores this slab bit for bit
        S.write_checkpoint(prefix, 7)
        S2 = RankSlab(dist, *n, device=0, **kw)
        restored = S2.read_checkpoint(prefix) == 7 and np.array_equal(S2.get_populations(), pops)
        S2.close()
        out[rank] = (forces, F, pops, prof, restored)
        S.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _rank_case(world):
    n = (20, 14, 19)
    f0 = cases.initial_populations(3, n, 5)
    kw = dict(tau=0.75, wall=(0, 0, 1, 2, 0, 0), wall_vel=(0.01, 0.0, 0.0), body_force=True,
              precision="fp64")
    ibm = dict(delta="peskin4", md_per_lb=2, xi_ibm=0.8)
    x, v, m = _slab_markers(n, world)
    return n, f0, kw, ibm, x, v, m, (1e-5, 0.0, 2e-6)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("window", [0, 1])
def test_rank_slabs_over_gloo_match_the_whole_lattice(cuda_lib, tmp_path, world, window):
    """RankSlab end to end with one process per slab, all on this GPU, the
    halos (populations, IBM moments, folded forces) moved by gloo through the
    host (no kernel waits on another process): per-atom forces, force field,
    populations and y profile of the whole lattice, FP64 within 1e-12, and
    per-rank checkpoints that restore each slab bit for bit."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    prefix = str(tmp_path / "slab")
    mp.start_processes(_rank_ibm, args=(world, port, window, prefix, out), nprocs=world, start_method="spawn")
    n, f0, kw, ibm, x, v, m, g = _rank_case(world)
    L = Lattice(3, *n, **kw)
    L.set_option("ibm_window", window)
    L.set_populations(f0)
    L.set_ibm_params(**ibm)
    k = 0
    for c in range(3):
        L.lbm_step(g)
        for s in range(2):
            x = np.ascontiguousarray(np.mod(x + 0.5 * v, np.array(n, float)))
            fl = np.zeros_like(x)
            L.ibm_substep(x, v, m, fl, refresh=(s == 0))
            fr = np.zeros_like(x)
            for r in range(world):
                mine, f = out[r][0][k]
                fr[mine] = f
            assert rel(fr, fl) <= 1e-12, (c, s, rel(fr, fl))
            k += 1
    FL = [a[1:-1, 1:-1, 1:-1] for a in L.get_force_field()]
    for c in range(3):
        got = np.concatenate([out[r][1][c] for r in range(world)], axis=0)
        assert rel(got, FL[c]) <= 1e-12, (c, rel(got, FL[c]))
    L.lbm_step(g)
    pops = np.concatenate([out[r][2] for r in range(world)], axis=1)
    assert rel(pops, L.get_populations()[:, 1:-1, 1:-1, 1:-1]) <= 1e-12
    # the y profile of the whole lattice (sums over every rank), and the
    # per-rank checkpoints
    L.macroscopic()
    ux, uy, rho = L.y_profile()
    c = float(n[0] * n[2])
    for r in range(world):
        for got, want in zip(out[r][3], (rho / c, ux / c, uy / c)):
            assert rel(got, want) <= 1e-12
        assert out[r][4]
    L.close()
