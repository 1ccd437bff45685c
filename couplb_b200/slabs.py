"""Slab decomposition of a D3Q19 lattice along z.

The reference decomposes the grid over MPI ranks and exchanges the ghost
planes of the populations every LB step (Streaming::exchange_dim,
couplb_streaming.h:176-194).  Here each slab is one lattice handle whose
z faces toward other slabs carry a halo (couplb_halo_attach): before every LB
step the halo holds the five populations that cross the face, packed by the
neighbour slab from its boundary plane after its last LB step
(couplb_halo_pack).  Only those 5 of 19 populations of the interior face
travel (the reference sends all 19 of the ghost-inclusive face).

- ``partition`` / ``neighbours`` / ``crossing`` are the plan (pure functions,
  tested on the CPU);
- ``exchange`` moves the packed planes between ranks with torch.distributed
  (NCCL for device tensors, gloo for host tensors);
- ``SlabLattice`` runs all slabs of a lattice in one process (on one device
  or several), moving the planes with device copies; its results are those
  of the whole lattice, bit for bit;
- ``RankSlab`` is the slab of one rank of a process group (one GPU per rank),
  exchanging with ``exchange``.

The immersed-boundary coupling is decomposed too (``SlabLattice``, single
pass): a marker belongs to the slab whose planes hold its cell; its window
reaches one plane below the slab and two above, whose moments the neighbours
compute after every LB step (couplb_ibm_halo_moments) and whose spread forces
they add to their own fields before the next one (couplb_ibm_halo_fold) -- the
velocity exchange and the reverse force exchange of the reference
(couplb_streaming.h:196-245), with the window the whole lattice uses.
"""
import numpy as np

from .lattice import Lattice

# D3Q19 velocities in the reference's q order (couplb_lattice.h:44-75)
EZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1)


def crossing(ez):
    """Populations that cross a z face moving in direction ez (+1 / -1), in
    the slot order of a packed halo."""
    return [q for q in range(19) if EZ[q] == ez]


def partition(nz, nslab):
    """(z0, nz_local) of each slab: nz planes split as evenly as possible."""
    if nslab < 1 or nslab > nz:
        raise ValueError(f"cannot split {nz} planes into {nslab} slabs")
    base, extra = divmod(nz, nslab)
    out, z0 = [], 0
    for s in range(nslab):
        n = base + (1 if s < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


def neighbours(slab, nslab, periodic_z):
    """(below, above): the slab across the low and the high z face, or None
    at a wall (non-periodic global z) or when one slab wraps onto itself."""
    if nslab == 1:
        return None, None
    below = slab - 1 if slab > 0 else (nslab - 1 if periodic_z else None)
    above = slab + 1 if slab < nslab - 1 else (0 if periodic_z else None)
    return below, above


CLBK_MAGIC, CLBK_VERSION = 0x434C424B, 1   # "CLBK" (couplb_io.h:21)


def write_clbk(path, step, f, offset, glob):
    """One rank's checkpoint in the .clbk layout (couplb_io.h:669-719):
    magic, version, step, D, Q, local dims, offset, global dims, then f
    (Q x ghost-inclusive nodes, FP64)."""
    import struct
    Q, gz, gy, gx = f.shape
    with open(path, "wb") as fp:
        fp.write(struct.pack("<Iiqii", CLBK_MAGIC, CLBK_VERSION, int(step), 3, Q))
        fp.write(struct.pack("<3i", gx - 2, gy - 2, gz - 2))
        fp.write(struct.pack("<3i", *offset))
        fp.write(struct.pack("<3i", *glob))
        fp.write(np.ascontiguousarray(f, dtype=np.float64).tobytes())


def read_clbk(path, shape, offset, glob):
    """(step, f) of a .clbk file whose header matches this slab's D, Q, local
    dims, offset and global dims (ValueError otherwise)."""
    import struct
    Q, gz, gy, gx = shape
    with open(path, "rb") as fp:
        head = fp.read(24 + 36)
        if len(head) != 60:
            raise ValueError(f"{path}: truncated header")
        magic, version, step, D, q = struct.unpack("<Iiqii", head[:24])
        dims, offs, gl = (struct.unpack("<3i", head[24 + 12 * i:36 + 12 * i]) for i in range(3))
        if magic != CLBK_MAGIC or version != CLBK_VERSION:
            raise ValueError(f"{path}: not a version {CLBK_VERSION} .clbk file")
        if (D, q) != (3, Q) or dims != (gx - 2, gy - 2, gz - 2) or offs != tuple(offset) or gl != tuple(glob):
            raise ValueError(f"{path}: written for another lattice or slab")
        f = np.frombuffer(fp.read(), dtype=np.float64)
    if f.size != Q * gz * gy * gx:
        raise ValueError(f"{path}: short read")
    return step, f.reshape(shape).copy()


def owner_slabs(z, parts, lo=0.0, dx=1.0):
    """Slab of every marker z coordinate: the one whose planes hold its cell
    (cells below / above the box go to the first / last slab)."""
    cell = np.floor((np.asarray(z, dtype=np.float64) - lo) / dx).astype(np.int64)
    starts = np.array([z0 for z0, _ in parts])
    return np.clip(np.searchsorted(starts, cell, side="right") - 1, 0, len(parts) - 1)


def ibm_halo_planes(slab, nslab, periodic_z, window):
    """(below, above): window planes a slab's markers reach beyond its low and
    high faces (0 where the face is not bound to a neighbour): 1 below; 2
    above, except where the high face wraps the global periodic box and the
    window is clipped (window 0), where the whole lattice drops the plane
    beyond its ghost layer."""
    below, above = neighbours(slab, nslab, periodic_z)
    lo = 0 if below is None else 1
    hi = 0 if above is None else (1 if (periodic_z and slab == nslab - 1 and window == 0) else 2)
    return lo, hi


def slab_walls(wall, slab, nslab):
    """Wall types of a slab: the global x and y faces; a z face is the
    global wall at the ends of a non-periodic z and periodic (a halo or,
    for a single slab, the self wrap) elsewhere."""
    w = list(wall)
    if slab > 0:
        w[4] = 0
    if slab < nslab - 1:
        w[5] = 0
    return tuple(w)


def exchange(dist, rank, world, periodic_z, send_lo, send_hi, recv_lo, recv_hi):
    """One halo exchange of a rank's slab over torch.distributed: send_hi
    (the planes leaving through the high face) goes to the slab above, whose
    recv_lo receives it; send_lo to the slab below, into its recv_hi.  Any
    argument for a face without a neighbour is ignored.  Every rank calls it
    at the same point of every step."""
    below, above = neighbours(rank, world, periodic_z)
    # gloo moves host tensors: device buffers are staged through the host
    host = dist.get_backend() == "gloo"
    stage = (lambda t: t.cpu() if (host and t.is_cuda) else t)   # noqa: E731
    s_lo, s_hi, r_lo, r_hi = stage(send_lo), stage(send_hi), stage(recv_lo), stage(recv_hi)
    # upward flow first, then downward, on every rank: with two ranks on a
    # periodic z the neighbour above is also the one below, and messages of
    # one pair match in the order they are posted (tags 0 / 1 for backends
    # that use them)
    ops = []
    if above is not None:
        ops.append(dist.P2POp(dist.isend, s_hi, above, tag=0))
    if below is not None:
        ops.append(dist.P2POp(dist.irecv, r_lo, below, tag=0))
    if below is not None:
        ops.append(dist.P2POp(dist.isend, s_lo, below, tag=1))
    if above is not None:
        ops.append(dist.P2POp(dist.irecv, r_hi, above, tag=1))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    if below is not None and r_lo is not recv_lo:
        recv_lo.copy_(r_lo)
    if above is not None and r_hi is not recv_hi:
        recv_hi.copy_(r_hi)


def _gravity(g_lb):
    return None if g_lb is None else tuple(g_lb)


class SlabLattice:
    """A D3Q19 lattice of nz planes run as `nslab` z slabs in one process.

    devices: one CUDA device per slab (default: all on device 0); with several
    devices the planes move by peer copies.  All slabs of one device share
    that device's current torch stream, so the packs of a step are ordered
    after every slab's LB step and before the next step."""

    def __init__(self, nx, ny, nz, nslab, tau=0.8, rho0=1.0, wall=(0,) * 6, wall_vel=(0.0, 0.0, 0.0),
                 body_force=False, precision="fp64", devices=None):
        import torch
        self.torch = torch
        self.n = (nx, ny, nz)
        self.nslab = nslab
        self.periodic_z = wall[4] == 0 and wall[5] == 0
        self.parts = partition(nz, nslab)
        self.devices = list(devices) if devices is not None else [0] * nslab
        self.slabs, self.recv = [], []
        for s, (z0, nzl) in enumerate(self.parts):
            dev = self.devices[s]
            L = Lattice(3, nx, ny, nzl, tau=tau, rho0=rho0, wall=slab_walls(wall, s, nslab),
                        wall_vel=wall_vel, body_force=body_force, precision=precision, device=dev)
            with torch.cuda.device(dev):
                L.set_stream(torch.cuda.current_stream().cuda_stream)
            self.slabs.append(L)
        nb = int(self.slabs[0].L.couplb_halo_bytes(self.slabs[0].h))
        for s, L in enumerate(self.slabs):
            below, above = neighbours(s, nslab, self.periodic_z)
            bufs = [None, None]
            for side, nbr in ((0, below), (1, above)):
                if nbr is None:
                    continue
                bufs[side] = torch.zeros(nb, dtype=torch.uint8, device=f"cuda:{self.devices[s]}")
                L._ck(L.L.couplb_halo_attach(L.h, side, bufs[side].data_ptr()))
            self.recv.append(bufs)
        self.stage = [torch.empty(nb, dtype=torch.uint8, device=f"cuda:{d}") for d in self.devices]

    def close(self):
        for L in self.slabs:
            L.close()
        self.slabs = []

    def set_option(self, name, value):
        for L in self.slabs:
            L.set_option(name, value)
        if name == "ibm_window" and getattr(self, "ibm", None):
            self._attach_ibm()

    # ---- immersed boundary -------------------------------------------------
    def _high_planes(self, s):
        return ibm_halo_planes(s, self.nslab, self.periodic_z, self.slabs[s].get_option("ibm_window"))[1]

    def _attach_ibm(self):
        torch = self.torch
        self.ih = []
        for s, L in enumerate(self.slabs):
            below, above = neighbours(s, self.nslab, self.periodic_z)
            dev = f"cuda:{self.devices[s]}"
            bufs = {}
            for side, nbr in ((0, below), (1, above)):
                if nbr is None:
                    continue
                planes = 1 if side == 0 else self._high_planes(s)
                nb = int(L.L.couplb_ibm_halo_bytes(L.h, planes))
                vel = torch.zeros(nb, dtype=torch.uint8, device=dev)
                frc = torch.zeros(nb, dtype=torch.uint8, device=dev)
                L._ck(L.L.couplb_ibm_halo_attach(L.h, side, planes, vel.data_ptr(), frc.data_ptr()))
                bufs[side] = (planes, vel, frc)
            self.ih.append(bufs)
        self._fold_pending = False
        self._ibm_moments()

    def set_ibm_params(self, domain_lo=(0.0, 0.0, 0.0), dx=1.0, **kw):
        """IBM constants of every slab (offset z0: global positions map to the
        slab's own planes) and the IBM halos of its bound faces."""
        self.ibm = dict(domain_lo=tuple(domain_lo), dx=float(dx))
        for (z0, _), L in zip(self.parts, self.slabs):
            L.set_ibm_params(domain_lo=domain_lo, dx=dx, offset=(0, 0, z0), **kw)
        self._attach_ibm()

    def _ibm_moments(self):
        """After the population exchange: every slab's halo moments from its
        neighbours' boundary planes."""
        for s, L in enumerate(self.slabs):
            below, above = neighbours(s, self.nslab, self.periodic_z)
            for side, nbr in ((0, below), (1, above)):
                if side not in self.ih[s]:
                    continue
                planes, vel, _ = self.ih[s][side]
                N = self.slabs[nbr]
                if self.devices[nbr] == self.devices[s]:
                    N._ck(N.L.couplb_ibm_halo_moments(N.h, 1 - side, planes, vel.data_ptr()))
                else:
                    st = self.torch.empty_like(vel, device=f"cuda:{self.devices[nbr]}")
                    N._ck(N.L.couplb_ibm_halo_moments(N.h, 1 - side, planes, st.data_ptr()))
                    self.torch.cuda.current_stream(self.devices[nbr]).synchronize()
                    vel.copy_(st)

    def fold_forces(self):
        """Add the forces every slab spread beyond its faces to its neighbours'
        fields and clear them (before the next LB step)."""
        if not getattr(self, "_fold_pending", False):
            return
        for s, L in enumerate(self.slabs):
            below, above = neighbours(s, self.nslab, self.periodic_z)
            for side, nbr in ((0, below), (1, above)):
                if side not in self.ih[s]:
                    continue
                planes, _, frc = self.ih[s][side]
                N = self.slabs[nbr]
                src = frc
                if self.devices[nbr] != self.devices[s]:
                    self.torch.cuda.current_stream(self.devices[s]).synchronize()
                    src = frc.to(f"cuda:{self.devices[nbr]}")
                N._ck(N.L.couplb_ibm_halo_fold(N.h, 1 - side, planes, src.data_ptr()))
                if src is not frc:
                    self.torch.cuda.current_stream(self.devices[nbr]).synchronize()
                frc.zero_()
        self._fold_pending = False

    def owners(self, x):
        """Slab of every marker: the one whose planes hold its cell (cells
        below / above the box go to the first / last slab)."""
        return owner_slabs(np.asarray(x)[:, 2], self.parts, self.ibm["domain_lo"][2], self.ibm["dx"])

    def _idle_substep(self, s, refresh):
        """The sub-step of a slab without coupled markers while the group has
        some elsewhere: the refresh still happens on every subdomain (the
        group count is global, fix_couplb.cpp:743-760), so the slab runs the
        sub-step of one marker outside the group."""
        torch = self.torch
        L = self.slabs[s]
        dev = f"cuda:{self.devices[s]}"
        z = self.ibm["domain_lo"][2] + (self.parts[s][0] + 0.5) * self.ibm["dx"]
        x = torch.tensor([[0.0, 0.0, z]], dtype=torch.float64, device=dev)
        zero = torch.zeros((1, 3), dtype=torch.float64, device=dev)
        one = torch.ones(1, dtype=torch.float64, device=dev)
        off = torch.zeros(1, dtype=torch.int32, device=dev)
        L.ibm_substep_device(1, x.data_ptr(), zero.data_ptr(), one.data_ptr(), zero.data_ptr(),
                             off.data_ptr(), refresh=refresh)
        torch.cuda.current_stream(self.devices[s]).synchronize()

    def ibm_substep(self, x, v, mass, f_add, active=None, refresh=True):
        """Single-pass IBM sub-step of host markers (f_add incremented in
        place), each marker on its slab.  Returns the markers in the group."""
        own = self.owners(x)
        coupled = np.ones(x.shape[0], bool) if active is None else np.asarray(active) != 0
        total = int(coupled.sum())
        nc = 0
        for s, L in enumerate(self.slabs):
            idx = np.nonzero(own == s)[0]
            if total > 0 and not coupled[idx].any():
                self._idle_substep(s, refresh)
                continue
            xs = np.ascontiguousarray(x[idx])
            fs = np.zeros_like(xs)
            act = None if active is None else np.ascontiguousarray(active[idx], dtype=np.int32)
            nc += L.ibm_substep(xs, np.ascontiguousarray(v[idx]), np.ascontiguousarray(mass[idx]), fs,
                                active=act, refresh=refresh)
            f_add[idx] += fs
        self._fold_pending = True
        return nc

    def get_force_field(self):
        """Interior force field (3 arrays nz, ny, nx) after the pending folds."""
        self.fold_forces()
        parts = [[a[1:-1, 1:-1, 1:-1] for a in L.get_force_field()] for L in self.slabs]
        return [np.concatenate([p[c] for p in parts], axis=0) for c in range(3)]

    def _exchange(self):
        """Pack every slab's leaving planes into its neighbours' halos."""
        torch = self.torch
        for s, L in enumerate(self.slabs):
            below, above = neighbours(s, self.nslab, self.periodic_z)
            for side, nbr in ((1, above), (0, below)):
                if nbr is None:
                    continue
                dst = self.recv[nbr][1 - side]
                if self.devices[nbr] == self.devices[s]:
                    L._ck(L.L.couplb_halo_pack(L.h, side, dst.data_ptr()))
                else:
                    L._ck(L.L.couplb_halo_pack(L.h, side, self.stage[s].data_ptr()))
                    torch.cuda.current_stream(self.devices[s]).synchronize()
                    dst.copy_(self.stage[s])
        if len(set(self.devices)) > 1:
            for d in set(self.devices):
                torch.cuda.current_stream(d).synchronize()

    def lbm_step(self, g_lb=None):
        if getattr(self, "ibm", None):
            self.fold_forces()
        for L in self.slabs:
            L.lbm_step(_gravity(g_lb))
        self._exchange()
        if getattr(self, "ibm", None):
            self._ibm_moments()

    def set_populations(self, f):
        """f: global (19, nz+2, ny+2, nx+2) reference layout."""
        for (z0, nzl), L in zip(self.parts, self.slabs):
            L.set_populations(np.ascontiguousarray(f[:, z0:z0 + nzl + 2]))
        if getattr(self, "ibm", None):
            self._ibm_moments()

    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        for L in self.slabs:
            L.init_equilibrium(rho, ux, uy, uz)
        if getattr(self, "ibm", None):
            self._ibm_moments()

    def get_populations(self):
        """Interior populations (19, nz, ny, nx) of the whole lattice."""
        return np.concatenate([L.get_populations()[:, 1:-1, 1:-1, 1:-1] for L in self.slabs], axis=1)

    def get_macroscopic(self):
        """Interior rho, ux, uy, uz (nz, ny, nx) after a moment pass."""
        parts = []
        for L in self.slabs:
            L.macroscopic()
            parts.append([a[1:-1, 1:-1, 1:-1] for a in L.get_macroscopic()])
        return [np.concatenate([p[c] for p in parts], axis=0) for c in range(4)]

    def diagnostics(self):
        """(umax, mass, momentum[3]) of the whole lattice: FP64 sums of the
        slabs' FP64 reductions, the largest speed."""
        ds = []
        for L in self.slabs:
            L.macroscopic()
            ds.append(L.diagnostics())
        return (max(d.umax for d in ds), sum(d.mass for d in ds),
                [sum(d.mom[c] for d in ds) for c in range(3)])


class RankSlab:
    """The slab of this rank in a process group (one GPU per rank): a D3Q19
    lattice of nz global planes, split over the group's ranks along z.  The
    halos move with ``exchange`` (NCCL device tensors) after every LB step;
    diagnostics reduce over the group in FP64."""

    def __init__(self, dist, nx, ny, nz, tau=0.8, rho0=1.0, wall=(0,) * 6, wall_vel=(0.0, 0.0, 0.0),
                 body_force=False, precision="fp64", device=0):
        import torch
        self.torch, self.dist = torch, dist
        self.device = device
        self.L_nx, self.L_ny, self.nz_global = nx, ny, nz
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.periodic_z = wall[4] == 0 and wall[5] == 0
        self.z0, nzl = partition(nz, self.world)[self.rank]
        self.L = Lattice(3, nx, ny, nzl, tau=tau, rho0=rho0, wall=slab_walls(wall, self.rank, self.world),
                         wall_vel=wall_vel, body_force=body_force, precision=precision, device=device)
        torch.cuda.set_device(device)
        self.L.set_stream(torch.cuda.current_stream().cuda_stream)
        nb = int(self.L.L.couplb_halo_bytes(self.L.h))
        mk = lambda: torch.zeros(nb, dtype=torch.uint8, device=f"cuda:{device}")  # noqa: E731
        self.send = [mk(), mk()]
        self.recv = [mk(), mk()]
        below, above = neighbours(self.rank, self.world, self.periodic_z)
        for side, nbr in ((0, below), (1, above)):
            if nbr is not None:
                self.L._ck(self.L.L.couplb_halo_attach(self.L.h, side, self.recv[side].data_ptr()))
        self.nbrs = (below, above)

    def lbm_step(self, g_lb=None):
        L = self.L
        if getattr(self, "ibm", None):
            self.fold_forces()
        L.lbm_step(_gravity(g_lb))
        for side in (0, 1):
            if self.nbrs[side] is not None:
                L._ck(L.L.couplb_halo_pack(L.h, side, self.send[side].data_ptr()))
        exchange(self.dist, self.rank, self.world, self.periodic_z, self.send[0], self.send[1],
                 self.recv[0], self.recv[1])
        if getattr(self, "ibm", None):
            self._ibm_moments()

    # ---- immersed boundary (single pass; this rank's markers) --------------
    def set_ibm_params(self, domain_lo=(0.0, 0.0, 0.0), dx=1.0, **kw):
        """IBM constants (offset z0) and the IBM halos: the moments of the
        planes beyond each bound face (received after every LB step) and the
        forces spread onto them (sent before the next)."""
        torch, L = self.torch, self.L
        self.ibm = dict(domain_lo=tuple(domain_lo), dx=float(dx))
        L.set_ibm_params(domain_lo=domain_lo, dx=dx, offset=(0, 0, self.z0), **kw)
        window = L.get_option("ibm_window")
        own = ibm_halo_planes(self.rank, self.world, self.periodic_z, window)
        below, above = self.nbrs
        # planes of the neighbours' halos that face this slab
        self.ih_planes = own
        self.ih_nbr = (0 if below is None else ibm_halo_planes(below, self.world, self.periodic_z, window)[1],
                       0 if above is None else ibm_halo_planes(above, self.world, self.periodic_z, window)[0])
        mk = lambda p: torch.zeros(int(L.L.couplb_ibm_halo_bytes(L.h, p)) if p else 1,  # noqa: E731
                                   dtype=torch.uint8, device=f"cuda:{self.device}")
        self.vel = [mk(own[0]), mk(own[1])]        # received moments
        self.frc = [mk(own[0]), mk(own[1])]        # forces spread beyond the faces
        self.msend = [mk(self.ih_nbr[0]), mk(self.ih_nbr[1])]   # moments for the neighbours
        self.frecv = [mk(self.ih_nbr[0]), mk(self.ih_nbr[1])]   # their forces on this slab
        for side in (0, 1):
            if own[side]:
                L._ck(L.L.couplb_ibm_halo_attach(L.h, side, own[side], self.vel[side].data_ptr(),
                                                 self.frc[side].data_ptr()))
        self._fold_pending = False
        self._ibm_moments()

    def _ibm_moments(self):
        L = self.L
        for side in (0, 1):
            if self.ih_nbr[side]:
                L._ck(L.L.couplb_ibm_halo_moments(L.h, side, self.ih_nbr[side], self.msend[side].data_ptr()))
        # msend[1] (our top plane) goes up into the neighbour's vel[0];
        # msend[0] (our lowest planes) down into its vel[1]
        exchange(self.dist, self.rank, self.world, self.periodic_z, self.msend[0], self.msend[1],
                 self.vel[0], self.vel[1])

    def fold_forces(self):
        """Send the forces spread beyond each face to the neighbour there, add
        the neighbours' forces on this slab, clear the halos.  Every rank
        calls it at the same point (lbm_step does)."""
        L = self.L
        exchange(self.dist, self.rank, self.world, self.periodic_z, self.frc[0], self.frc[1],
                 self.frecv[0], self.frecv[1])
        for side in (0, 1):
            if self.ih_nbr[side]:
                L._ck(L.L.couplb_ibm_halo_fold(L.h, side, self.ih_nbr[side], self.frecv[side].data_ptr()))
        for b in self.frc:
            b.zero_()
        self._fold_pending = False

    def ibm_substep(self, x, v, mass, f_add, active=None, refresh=True):
        """Single-pass sub-step of this rank's markers (host arrays, global
        positions within this slab's planes); the group count is global, so a
        rank without coupled markers still refreshes while others have some."""
        torch = self.torch
        mine = x.shape[0] if active is None else int(np.count_nonzero(active))
        tot = torch.tensor([mine], dtype=torch.int64, device=self._rdev())
        self.dist.all_reduce(tot)
        nc = 0
        if mine == 0 and int(tot.item()) > 0:
            z = self.ibm["domain_lo"][2] + (self.z0 + 0.5) * self.ibm["dx"]
            xd = torch.tensor([[0.0, 0.0, z]], dtype=torch.float64, device="cuda")
            zero = torch.zeros((1, 3), dtype=torch.float64, device="cuda")
            one = torch.ones(1, dtype=torch.float64, device="cuda")
            off = torch.zeros(1, dtype=torch.int32, device="cuda")
            self.L.ibm_substep_device(1, xd.data_ptr(), zero.data_ptr(), one.data_ptr(), zero.data_ptr(),
                                      off.data_ptr(), refresh=refresh)
            torch.cuda.synchronize()
        elif mine > 0:
            nc = self.L.ibm_substep(x, v, mass, f_add, active=active, refresh=refresh)
        self._fold_pending = True
        return nc

    def _rdev(self):
        """Device of reduction tensors: the host for gloo, this GPU for NCCL."""
        return "cpu" if self.dist.get_backend() == "gloo" else f"cuda:{self.device}"

    def diagnostics(self):
        torch = self.torch
        self.L.macroscopic()
        d = self.L.diagnostics()
        t = torch.tensor([d.mass, d.mom[0], d.mom[1], d.mom[2]], dtype=torch.float64, device=self._rdev())
        self.dist.all_reduce(t)
        u = torch.tensor([d.umax], dtype=torch.float64, device=self._rdev())
        self.dist.all_reduce(u, op=self.dist.ReduceOp.MAX)
        return float(u.item()), float(t[0].item()), [float(x) for x in t[1:].tolist()]

    def y_profile(self):
        """(rho, ux, uy) per j, means over i and k of the whole lattice: the
        profile of FixCoupLB::write_profile with every rank's sums reduced
        (fix_couplb.cpp:903-979), lattice units.  A collective."""
        torch = self.torch
        self.L.macroscopic()
        ux, uy, rho = self.L.y_profile()
        t = torch.tensor(np.concatenate([rho, ux, uy]), dtype=torch.float64, device=self._rdev())
        self.dist.all_reduce(t)
        ny = rho.shape[0]
        a = t.cpu().numpy() / float(self.L_nx * self.nz_global)
        return a[:ny], a[ny:2 * ny], a[2 * ny:]

    def write_checkpoint(self, prefix, step):
        """prefix.<rank>.clbk in the layout of IO::write_checkpoint
        (couplb_io.h:669-719): this rank's planes with their z offset."""
        write_clbk(f"{prefix}.{self.rank}.clbk", step, self.L.get_populations(),
                   (0, 0, self.z0), (self.L_nx, self.L_ny, self.nz_global))

    def read_checkpoint(self, prefix):
        """Restore this rank's planes from prefix.<rank>.clbk (header checked
        against this slab); returns the step."""
        step, f = read_clbk(f"{prefix}.{self.rank}.clbk", self.L.get_populations().shape, (0, 0, self.z0),
                            (self.L_nx, self.L_ny, self.nz_global))
        self.L.set_populations(f)
        if getattr(self, "ibm", None):
            self._ibm_moments()
        return step

    def set_populations(self, f):
        """f: the global (19, nz+2, ny+2, nx+2) reference layout; this rank
        takes its planes."""
        z0 = self.z0
        nzl = partition(f.shape[1] - 2, self.world)[self.rank][1]
        self.L.set_populations(np.ascontiguousarray(f[:, z0:z0 + nzl + 2]))
        if getattr(self, "ibm", None):
            self._ibm_moments()

    def get_populations(self):
        """This rank's interior populations (19, nz_local, ny, nx)."""
        return self.L.get_populations()[:, 1:-1, 1:-1, 1:-1]

    def get_force_field(self):
        """This rank's interior force field after the pending folds (a
        collective: every rank calls it)."""
        if getattr(self, "ibm", None):
            self.fold_forces()
        return [a[1:-1, 1:-1, 1:-1] for a in self.L.get_force_field()]

    def close(self):
        self.L.close()
