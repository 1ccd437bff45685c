"""FixCoupLB: the `fix couplb` command on the GPU (layer 2 of the C ABI).

Mirrors the LAMMPS fix (CoupLB/fix_couplb.h:22-30): construct from the
command's words, then call init / setup / post_force / end_of_step in the
order LAMMPS does.  Errors raise CoupLBError with the reference's message.

    fix = FixCoupLB("flow all couplb 8 32 1 0.1 1.0 wall_y 1 1 gravity 5e-6 0 0".split(),
                    dimension=2)
    fix.init(boxlo=(0, 0, -0.5), boxhi=(8, 32, 0.5), dt=1.0)
"""
import ctypes as C

import numpy as np

from . import abi
from .lattice import Lattice
from .lib import CoupLBError, GRAVITY_FN, LOG_FN, check, load


def parse_args(args, dimension=3):
    """couplb_fix_parse: words of the fix command (ID group couplb ...) -> FixConfig."""
    lib = load()
    words = [a.encode() if isinstance(a, str) else a for a in args]
    argv = (C.c_char_p * len(words))(*words)
    cfg = abi.FixConfig()
    err = C.create_string_buffer(512)
    rc = lib.couplb_fix_parse(len(words), argv, dimension, C.byref(cfg), err, 512)
    if rc:
        raise CoupLBError(rc, err.value.decode())
    return cfg


class _LatticeView(Lattice):
    """Lattice methods on a handle owned by a fix."""

    def __init__(self, handle, dim, nx, ny, nz):
        self.L = load()
        self.h = handle
        self.dim = dim
        self.Q = 19 if dim == 3 else 9
        self.nx, self.ny, self.nz = nx, ny, nz if dim == 3 else 1
        self.gx, self.gy = nx + 2, ny + 2
        self.gz = self.nz + 2 if dim == 3 else 1
        self.G = int(self.L.couplb_ghost_nodes(handle))

    def close(self):
        self.h = None


class FixCoupLB:
    def __init__(self, args, dimension=3, device=0, log=None):
        self.L = load()
        self.cfg = args if isinstance(args, abi.FixConfig) else parse_args(args, dimension)
        self.dimension = dimension
        h = C.c_void_p()
        check(self.L.couplb_fix_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        check(self.L.couplb_fix_set_device(h, device), fix=h)
        self._log_cb = None
        self._grav_cb = None
        self.messages = []
        self.set_log(log)
        self.lattice = None

    def _ck(self, rc):
        return check(rc, fix=self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.couplb_fix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setmask(self):
        return self.L.couplb_fix_setmask()

    def set_log(self, fn=None):
        def sink(_ctx, line):
            s = line.decode(errors="replace")
            self.messages.append(s)
            if fn is not None:
                fn(s)
        self._log_cb = LOG_FN(sink)
        self._ck(self.L.couplb_fix_set_log_callback(self.h, C.cast(self._log_cb, C.c_void_p), None))

    def set_gravity_callback(self, fn):
        """fn(component) -> acceleration (MD units) for v_ gravity components."""
        def cb(_ctx, comp, out):
            try:
                out[0] = float(fn(comp))
                return 0
            except Exception:
                return 1
        self._grav_cb = GRAVITY_FN(cb)
        self._ck(self.L.couplb_fix_set_gravity_callback(self.h, C.cast(self._grav_cb, C.c_void_p), None))

    def set_gravity_values(self, g):
        arr = np.asarray(g, dtype=np.float64)
        self._ck(self.L.couplb_fix_set_gravity_values(self.h, abi.dptr(arr)))

    # -- hooks (fix_couplb.h:26-30) ------------------------------------------
    def set_comm(self, nprocs, rank, sendrecv, allreduce):
        """Several ranks along z (couplb_fix_set_comm): sendrecv(side, d_send,
        send_bytes, d_recv, recv_bytes) and allreduce(numpy array, op) (op 0
        sum, 1 max, in place) move this rank's slab halos and reductions; the
        pointers are raw device addresses (0 where there is no neighbour)."""
        def sr(_ctx, side, d_send, sb, d_recv, rb):
            try:
                sendrecv(side, d_send or 0, sb, d_recv or 0, rb)
                return 0
            except Exception:
                return 1

        def ar(_ctx, buf, n, op):
            try:
                a = np.ctypeslib.as_array(buf, shape=(n,))
                allreduce(a, op)
                return 0
            except Exception:
                return 1
        self._comm_cbs = (abi.SENDRECV_FN(sr), abi.ALLREDUCE_FN(ar))
        self._comm = abi.FixComm(nprocs, rank, self._comm_cbs[0], self._comm_cbs[1], None)
        self._ck(self.L.couplb_fix_set_comm(self.h, C.byref(self._comm)))

    def init(self, boxlo, boxhi, dt, ntimestep=0, periodicity=(1, 1, 1), sublo=None, subhi=None):
        self.domain = abi.make_domain(self.dimension, boxlo, boxhi, dt, periodicity, ntimestep, sublo, subhi)
        self._ck(self.L.couplb_fix_init(self.h, C.byref(self.domain)))
        c = self.cfg
        nz = c.Nz
        if sublo is not None and self.dimension == 3:
            nz = int(round((subhi[2] - sublo[2]) / self.scales()["dx"]))
        self.lattice = _LatticeView(self.L.couplb_fix_handle(self.h), self.dimension, c.Nx, c.Ny, nz)
        return self

    def setup(self, atoms, ntimestep=0):
        self._ck(self.L.couplb_fix_setup(self.h, C.byref(atoms), ntimestep))

    def post_force(self, atoms, ntimestep):
        self._ck(self.L.couplb_fix_post_force(self.h, C.byref(atoms), ntimestep))

    def end_of_step(self, ntimestep):
        self._ck(self.L.couplb_fix_end_of_step(self.h, ntimestep))

    def write_solid(self, atoms, ntimestep):
        """vtk_solid output of the step end_of_step just handled (no-op on
        other steps)."""
        self._ck(self.L.couplb_fix_write_solid(self.h, C.byref(atoms), ntimestep))

    # -- accessors ----------------------------------------------------------
    def scales(self):
        out = np.empty(6)
        self._ck(self.L.couplb_fix_scales(self.h, abi.dptr(out)))
        return dict(zip(["dx", "dt_lbm", "vel_scale", "force_scale", "nu_lb", "tau"], out))

    def last_diag(self):
        d = abi.Diag()
        self._ck(self.L.couplb_fix_last_diag(self.h, C.byref(d)))
        return d

    def lbm_steps(self):
        return int(self.L.couplb_fix_lbm_steps(self.h))
