"""Slab decomposition along z (couplb_b200/slabs.py): the plan and the halo
exchange between ranks, on the CPU with gloo.

Every rank holds the same seeded post-collision state of a global lattice
(19 populations on nz planes), packs the planes that leave its slab the way
couplb_halo_pack does (the crossing populations of its boundary plane, in
halo-slot order), exchanges them with slabs.exchange, and checks that what
arrived is what the pull at its faces reads in the undecomposed lattice:
the neighbour planes z0 - 1 and z0 + nz_local, wrapped on a periodic z
(Streaming::exchange_dim, couplb_streaming.h:176-194)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from couplb_b200 import slabs  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_and_neighbours():
    assert slabs.partition(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slabs.partition(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        slabs.partition(2, 3)
    assert slabs.neighbours(0, 3, True) == (2, 1)
    assert slabs.neighbours(2, 3, True) == (1, 0)
    assert slabs.neighbours(0, 3, False) == (None, 1)
    assert slabs.neighbours(2, 3, False) == (1, None)
    assert slabs.neighbours(0, 1, True) == (None, None)
    assert slabs.slab_walls((0, 0, 1, 1, 2, 3), 0, 3) == (0, 0, 1, 1, 2, 0)
    assert slabs.slab_walls((0, 0, 1, 1, 2, 3), 1, 3) == (0, 0, 1, 1, 0, 0)
    assert slabs.slab_walls((0, 0, 1, 1, 2, 3), 2, 3) == (0, 0, 1, 1, 0, 3)


def test_ibm_halo_planes_match_the_whole_lattice_window():
    """One plane below a bound face, two above; at the face that wraps the
    periodic box a clipped window (0) keeps one, as the whole lattice's
    window stops at its ghost layer; faces at a wall are not bound."""
    assert [slabs.ibm_halo_planes(s, 3, True, 1) for s in range(3)] == [(1, 2)] * 3
    assert [slabs.ibm_halo_planes(s, 3, True, 0) for s in range(3)] == [(1, 2), (1, 2), (1, 1)]
    assert [slabs.ibm_halo_planes(s, 3, False, 0) for s in range(3)] == [(0, 2), (1, 2), (1, 0)]
    assert slabs.ibm_halo_planes(0, 1, True, 0) == (0, 0)
    # a bound face has a halo on both sides of it: one plane above the face
    # for the slab above, one or two below it for the slab below
    for world in (2, 3, 4):
        for periodic in (True, False):
            for window in (0, 1):
                for s in range(world):
                    below, above = slabs.neighbours(s, world, periodic)
                    lo, hi = slabs.ibm_halo_planes(s, world, periodic, window)
                    assert (lo > 0) == (below is not None) and (hi > 0) == (above is not None)
                    if above is not None:
                        assert slabs.ibm_halo_planes(above, world, periodic, window)[0] == 1


def test_crossing_populations_are_the_d3q19_z_movers():
    up, down = slabs.crossing(1), slabs.crossing(-1)
    assert up == [5, 11, 14, 15, 18] and down == [6, 12, 13, 16, 17]
    # every mover has its opposite in the other list
    opp = [0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17]
    assert sorted(opp[q] for q in up) == down


def _rank(rank, world, port, periodic, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        nx, ny, nz = 5, 4, 11
        P = np.random.default_rng(7).standard_normal((19, nz, ny, nx))
        z0, nzl = slabs.partition(nz, world)[rank]
        up, down = slabs.crossing(1), slabs.crossing(-1)
        send_hi = torch.from_numpy(np.ascontiguousarray(P[up, z0 + nzl - 1]).reshape(-1))
        send_lo = torch.from_numpy(np.ascontiguousarray(P[down, z0]).reshape(-1))
        recv_lo = torch.full_like(send_hi, np.nan)
        recv_hi = torch.full_like(send_lo, np.nan)
        slabs.exchange(dist, rank, world, periodic, send_lo, send_hi, recv_lo, recv_hi)
        below, above = slabs.neighbours(rank, world, periodic)
        ok = True
        if below is not None:
            want = P[up, (z0 - 1) % nz].reshape(-1)
            ok &= bool(np.array_equal(recv_lo.numpy(), want))
        else:
            ok &= bool(np.isnan(recv_lo.numpy()).all())
        if above is not None:
            want = P[down, (z0 + nzl) % nz].reshape(-1)
            ok &= bool(np.array_equal(recv_hi.numpy(), want))
        else:
            ok &= bool(np.isnan(recv_hi.numpy()).all())
        out[rank] = ok
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_halo_exchange_delivers_the_neighbour_planes(world, periodic):
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, _free_port(), periodic, out), nprocs=world, start_method="spawn")
    assert dict(out) == {r: True for r in range(world)}


def test_clbk_round_trip_and_header_checks(tmp_path):
    """A slab's checkpoint file: the .clbk header of IO::write_checkpoint
    (couplb_io.h:669-719) with the slab's dims and z offset, f after it; a
    reader for another slab refuses it."""
    import struct
    f = np.random.default_rng(3).standard_normal((19, 7, 6, 5))
    path = str(tmp_path / "ck.1.clbk")
    slabs.write_clbk(path, 42, f, (0, 0, 10), (3, 4, 20))
    raw = open(path, "rb").read()
    assert struct.unpack("<Iiqii", raw[:24]) == (0x434C424B, 1, 42, 3, 19)
    assert struct.unpack("<9i", raw[24:60]) == (3, 4, 5, 0, 0, 10, 3, 4, 20)
    assert len(raw) == 60 + f.size * 8
    step, g = slabs.read_clbk(path, f.shape, (0, 0, 10), (3, 4, 20))
    assert step == 42 and np.array_equal(g, f)
    with pytest.raises(ValueError):
        slabs.read_clbk(path, f.shape, (0, 0, 5), (3, 4, 20))
    with pytest.raises(ValueError):
        slabs.read_clbk(path, (19, 8, 6, 5), (0, 0, 10), (3, 4, 20))


def test_owner_slabs_by_cell():
    """A marker belongs to the slab whose planes hold its cell; cells below
    or above the box go to the first or last slab."""
    parts = slabs.partition(10, 3)          # (0,4) (4,3) (7,3)
    z = np.array([0.0, 3.999, 4.0, 6.5, 7.0, 9.99, -0.5, 10.2])
    assert slabs.owner_slabs(z, parts).tolist() == [0, 0, 1, 1, 2, 2, 0, 2]
    # lattice units from MD units: z = lo + dx * cell
    assert slabs.owner_slabs(z * 0.5 - 1.0, parts, lo=-1.0, dx=0.5).tolist() == [0, 0, 1, 1, 2, 2, 0, 2]
