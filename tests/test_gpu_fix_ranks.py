"""The fix core on several ranks along z (couplb_fix_set_comm): one fix per
rank, each running its z slab of the lattice, the halos moved by the host
code's communicator -- here threads of this process on one GPU, exchanging
through host memory (each rank synchronises its own stream and copies; no
kernel waits on another rank).  The run matches one fix over the whole box:
atom forces at every step, populations and the reduced diagnostics, FP64
within 1e-12, and rank 0's profile file; checkpoints are written per rank
and a restart from them continues bit for bit."""
import ctypes as C
import threading
import struct

import numpy as np
import pytest

import cases
from couplb_b200 import md
from couplb_b200.fix import FixCoupLB

pytestmark = pytest.mark.gpu

N = (16, 14, 12)
BOX = ((0.0, 0.0, 0.0), (16.0, 14.0, 12.0))


def _cudart():
    import torch
    torch.zeros(1, device="cuda")        # the runtime torch loaded
    lib = C.CDLL("libcudart.so.12")
    lib.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return lib


class ThreadComm:
    """sendrecv / allreduce between the ranks of this process (threads)."""

    def __init__(self, nprocs):
        self.n = nprocs
        self.bar = threading.Barrier(nprocs, timeout=60)
        self.box = [[None, None] for _ in range(nprocs)]
        self.red = [None] * nprocs
        self.rt = _cudart()

    def sendrecv(self, rank, side, d_send, sb, d_recv, rb):
        msg = None
        if d_send:
            msg = (C.c_char * sb)()
            assert self.rt.cudaMemcpy(C.addressof(msg), d_send, sb, 2) == 0
        self.box[rank][side] = msg
        self.bar.wait()
        if d_recv:
            # sending across `side`, receiving from the rank across the other face
            src = (rank - 1) % self.n if side == 1 else (rank + 1) % self.n
            got = self.box[src][side]
            assert got is not None and len(got) == rb, (rank, side, rb)
            assert self.rt.cudaMemcpy(d_recv, C.addressof(got), rb, 1) == 0
        self.bar.wait()

    def allreduce(self, rank, a, op):
        self.red[rank] = a.copy()
        self.bar.wait()
        r = np.max(self.red, axis=0) if op == 1 else np.sum(self.red, axis=0)
        self.bar.wait()
        a[:] = r


def _cfg(wall, profile=""):
    return cases.make_cfg(Nx=N[0], Ny=N[1], Nz=N[2], nu=0.1, rho=1.0, md_per_lb=2, delta=1,
                          gravity=(3e-5, 0, 0), wall=wall, check_every=5, dimension=3,
                          output_every=6 if profile else 0, output_file=profile)


def _profile(path):
    return np.array([[float(w) for w in line.split()] for line in open(path)
                     if line.strip() and not line.startswith("#")])


def _markers():
    rng = np.random.default_rng(43)
    x = rng.uniform(0.5, 1.0, (40, 3)) * np.array(BOX[1])
    x[:, 1] = rng.uniform(3.0, 11.0, 40)        # away from the y walls
    x[:12, 2] = rng.uniform(-1.5, 1.5, 12) % N[2]   # across the periodic z face
    x[12:24, 2] = 6.0 + rng.uniform(-1.5, 1.5, 12)  # across the middle
    return x, 0.01 * rng.standard_normal(x.shape)


def _run(fix, x, v, steps=12):
    at = md.Atoms(x, v, integrate=False)
    forces, diags = [], []

    def on_step(step):
        forces.append(at.f.copy())
        if step % 5 == 0:
            d = fix.last_diag()
            diags.append([d.umax, d.mass, d.mom[0], d.mom[1], d.mom[2]])
    md.run(fix, at, steps, 0.5, on_step=on_step)
    return np.stack(forces), np.array(diags)


@pytest.mark.parametrize("nprocs", [2, 3])
@pytest.mark.parametrize("wall", [(0, 0, 1, 1, 0, 0), (0, 0, 1, 1, 1, 1)])
def test_z_slab_ranks_match_one_rank(cuda_lib, tmp_path, nprocs, wall):
    from couplb_b200.slabs import owner_slabs, partition
    x, v = _markers()
    one = FixCoupLB(_cfg(wall, str(tmp_path / "one.dat")), dimension=3)
    one.init(*BOX, 0.5)
    f1, d1 = _run(one, x, v)
    p1 = cases.interior(one.lattice.get_populations(), 3)
    one.close()

    parts = partition(N[2], nprocs)
    own = owner_slabs(x[:, 2], parts)
    comm = ThreadComm(nprocs)
    out = [None] * nprocs
    errors = []

    def rank_main(r):
        try:
            fx = FixCoupLB(_cfg(wall, str(tmp_path / f"ranks{r}.dat")), dimension=3)
            fx.set_comm(nprocs, r, lambda *a: comm.sendrecv(r, *a), lambda a, op: comm.allreduce(r, a, op))
            z0, nzl = parts[r]
            fx.init(*BOX, 0.5, sublo=(0.0, 0.0, float(z0)), subhi=(16.0, 14.0, float(z0 + nzl)))
            idx = np.nonzero(own == r)[0]
            f, d = _run(fx, x[idx], v[idx])
            out[r] = (idx, f, d, cases.interior(fx.lattice.get_populations(), 3))
            fx.close()
        except Exception as e:      # noqa: BLE001 -- reported by the main thread
            errors.append(repr(e))
            comm.bar.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(nprocs)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(120)
    assert not errors, errors
    fr = np.zeros_like(f1)
    for idx, f, _, _ in out:
        fr[:, idx] = f
    rel = lambda a, b: np.abs(a - b).max() / np.abs(b).max()   # noqa: E731
    assert rel(fr, f1) <= 1e-12, rel(fr, f1)
    pr = np.concatenate([o[3] for o in out], axis=1)
    assert rel(pr, p1) <= 1e-12, rel(pr, p1)
    for o in out:   # every rank holds the reduced diagnostics
        assert np.abs(o[2] - d1).max() <= 1e-12 * np.abs(d1).max()
    # rank 0 writes the profile of the whole lattice (sums over the ranks)
    a, b = _profile(tmp_path / "ranks0.dat"), _profile(tmp_path / "one.dat")
    assert a.shape == b.shape and np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    assert not any((tmp_path / f"ranks{r}.dat").exists() for r in range(1, nprocs))


def _in_threads(nprocs, body):
    """body(rank, comm) on `nprocs` threads; their results in rank order."""
    comm = ThreadComm(nprocs)
    out, errors = [None] * nprocs, []

    def main(r):
        try:
            out[r] = body(r, comm)
        except Exception as e:      # noqa: BLE001 -- reported by the main thread
            errors.append(repr(e))
            comm.bar.abort()

    threads = [threading.Thread(target=main, args=(r,)) for r in range(nprocs)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(120)
    assert not errors, errors
    return out


@pytest.mark.parametrize("nprocs", [2, 3])
def test_z_slab_checkpoint_restart(cuda_lib, tmp_path, nprocs):
    """A channel on z slabs writes prefix.<rank>.clbk with the slab's local
    grid and offset (couplb_io.h:669-719); fixes restarted from those files
    continue bit for bit, and the slabs match one fix over the whole box."""
    from couplb_b200.slabs import partition
    n = (6, 5, 9)
    box = ((0.0, 0.0, 0.0), (6.0, 5.0, 9.0))
    args = "f all couplb 6 5 9 0.1 1.0 wall_y 1 2 wall_vel 0.01 0 0 gravity 1e-5 0 2e-6".split()
    one = FixCoupLB(args, dimension=3)
    one.init(*box, 1.0)
    md.run(one, md.empty_atoms(), 17, 1.0)
    f17 = cases.interior(one.lattice.get_populations(), 3)
    one.close()
    parts = partition(n[2], nprocs)
    pre = str(tmp_path / "ck")

    def sub(r):
        z0, nzl = parts[r]
        return dict(sublo=(0.0, 0.0, float(z0)), subhi=(6.0, 5.0, float(z0 + nzl)))

    def first(r, comm):
        fx = FixCoupLB(args + ["checkpoint", "10", pre], dimension=3)
        fx.set_comm(nprocs, r, lambda *a: comm.sendrecv(r, *a), lambda a, op: comm.allreduce(r, a, op))
        fx.init(*box, 1.0, **sub(r))
        md.run(fx, md.empty_atoms(), 17, 1.0)
        f = cases.interior(fx.lattice.get_populations(), 3)
        fx.close()
        return f

    def again(r, comm):
        fx = FixCoupLB(args + ["restart", pre], dimension=3)
        fx.set_comm(nprocs, r, lambda *a: comm.sendrecv(r, *a), lambda a, op: comm.allreduce(r, a, op))
        fx.init(*box, 1.0, ntimestep=10, **sub(r))
        md.run(fx, md.empty_atoms(), 7, 1.0, start_step=10)
        f = cases.interior(fx.lattice.get_populations(), 3)
        fx.close()
        return f

    cont = _in_threads(nprocs, first)
    np.testing.assert_array_equal(np.concatenate(cont, axis=1), f17)
    for r in range(nprocs):
        raw = open(f"{pre}.{r}.clbk", "rb").read()
        step = struct.unpack_from("<q", raw, 8)[0]
        dims = struct.unpack_from("<9i", raw, 24)
        z0, nzl = parts[r]
        assert step == 10 and dims == (6, 5, nzl, 0, 0, z0, 6, 5, 9)
    rest = _in_threads(nprocs, again)
    for a, b in zip(rest, cont):
        np.testing.assert_array_equal(a, b)
