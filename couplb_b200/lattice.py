"""Python handle on one GPU lattice (layer 1 of the C ABI).

Arrays exchanged with the host use the reference layout: ghost-inclusive
(gz, gy, gx) node arrays, populations as (Q, gz, gy, gx) float64
(CoupLB/couplb_lattice.h:82-129).
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import check, load

PREC = abi.PRECISIONS


class Lattice:
    def __init__(self, dim, nx, ny, nz=1, tau=0.8, rho0=1.0, wall=(0,) * 6,
                 wall_vel=(0.0, 0.0, 0.0), body_force=False, precision="fp64", device=0):
        self.L = load()
        p = abi.LatticeParams()
        p.dim, p.nx, p.ny, p.nz = dim, nx, ny, (nz if dim == 3 else 1)
        p.tau, p.rho0 = tau, rho0
        for i in range(6):
            p.wall[i] = wall[i]
        for i in range(3):
            p.wall_vel[i] = wall_vel[i]
        p.body_force = int(bool(body_force))
        p.precision = PREC[precision] if isinstance(precision, str) else int(precision)
        p.device = device
        self.params = p
        h = C.c_void_p()
        check(self.L.couplb_create(C.byref(p), C.byref(h)), None)
        self.h = h
        self.dim = dim
        self.Q = 19 if dim == 3 else 9
        self.nx, self.ny, self.nz = nx, ny, p.nz
        self.gx, self.gy = nx + 2, ny + 2
        self.gz = p.nz + 2 if dim == 3 else 1
        self.G = int(self.L.couplb_ghost_nodes(h))

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.couplb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        return check(rc, self.h)

    @property
    def shape(self):
        return (self.gz, self.gy, self.gx)

    # -- state ------------------------------------------------------------
    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self._ck(self.L.couplb_init_equilibrium(self.h, rho, ux, uy, uz))

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        assert f.size == self.Q * self.G
        self._ck(self.L.couplb_set_populations(self.h, abi.dptr(f)))

    def get_populations(self):
        f = np.empty(self.Q * self.G)
        self._ck(self.L.couplb_get_populations(self.h, abi.dptr(f)))
        return f.reshape((self.Q,) + self.shape)

    def set_force_field(self, fx, fy, fz):
        a = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (fx, fy, fz)]
        self._ck(self.L.couplb_set_force_field(self.h, *[abi.dptr(x) for x in a]))

    def get_force_field(self):
        out = [np.empty(self.G) for _ in range(3)]
        self._ck(self.L.couplb_get_force_field(self.h, *[abi.dptr(x) for x in out]))
        return [x.reshape(self.shape) for x in out]

    # -- stepping ---------------------------------------------------------
    def lbm_step(self, g_lb=None):
        if g_lb is None:
            self._ck(self.L.couplb_lbm_step(self.h, C.POINTER(C.c_double)()))
        else:
            g = (C.c_double * 3)(*g_lb)
            self._ck(self.L.couplb_lbm_step(self.h, C.cast(g, C.POINTER(C.c_double))))

    def macroscopic(self):
        self._ck(self.L.couplb_macroscopic(self.h))

    def get_macroscopic(self):
        out = [np.empty(self.G) for _ in range(4)]
        self._ck(self.L.couplb_get_macroscopic(self.h, *[abi.dptr(x) for x in out]))
        return [x.reshape(self.shape) for x in out]

    def diagnostics(self):
        d = abi.Diag()
        self._ck(self.L.couplb_diagnostics(self.h, C.byref(d)))
        return d

    def y_profile(self):
        out = [np.empty(self.ny) for _ in range(3)]
        self._ck(self.L.couplb_y_profile(self.h, *[abi.dptr(x) for x in out]))
        return out

    def read_status(self, reset=False):
        a, b = C.c_int(0), C.c_int(0)
        self._ck(self.L.couplb_read_status(self.h, C.byref(a), C.byref(b), int(reset)))
        return a.value, b.value

    def status_post(self):
        """Enqueue a copy of the status word (pipelined per-step check)."""
        self._ck(self.L.couplb_status_post(self.h))

    def status_last(self):
        """(clamps, nonfinite) of the post before the latest one."""
        c, nf = C.c_int(0), C.c_int(0)
        self._ck(self.L.couplb_status_last(self.h, C.byref(c), C.byref(nf)))
        return c.value, nf.value

    def synchronize(self):
        self._ck(self.L.couplb_synchronize(self.h))

    def set_stream(self, stream_ptr):
        self._ck(self.L.couplb_set_stream(self.h, C.c_void_p(stream_ptr)))

    def device_bytes(self):
        return int(self.L.couplb_device_bytes(self.h))

    def set_option(self, name, value):
        self._ck(self.L.couplb_set_option(self.h, name.encode(), int(value)))

    def get_option(self, name):
        v = C.c_longlong(0)
        self._ck(self.L.couplb_get_option(self.h, name.encode(), C.byref(v)))
        return v.value

    # -- IBM ----------------------------------------------------------------
    def set_ibm_params(self, delta="roma", md_per_lb=1, xi_ibm=1.0, dt_lbm=1.0, dx=1.0,
                       vel_scale=1.0, force_scale=1.0, domain_lo=(0.0, 0.0, 0.0),
                       offset=(0, 0, 0)):
        ip = abi.IbmParams()
        ip.delta = {"roma": abi.DELTA_ROMA, "peskin4": abi.DELTA_PESKIN4}[delta] \
            if isinstance(delta, str) else int(delta)
        ip.md_per_lb, ip.xi_ibm, ip.dt_lbm, ip.dx = md_per_lb, xi_ibm, dt_lbm, dx
        ip.vel_scale, ip.force_scale = vel_scale, force_scale
        for i in range(3):
            ip.domain_lo[i] = domain_lo[i]
            ip.offset[i] = offset[i]
        self._ck(self.L.couplb_set_ibm_params(self.h, C.byref(ip)))
        self.ibm_params = ip
        return ip

    def ibm_substep(self, x, v, mass, f_add, active=None, refresh=True):
        """Host-array IBM sub-step; f_add (n,3) is incremented in place."""
        n = int(x.shape[0])
        nc = C.c_int(0)
        self._ck(self.L.couplb_ibm_substep(self.h, n, abi.dptr(x), abi.dptr(v), abi.dptr(mass),
                                           abi.iptr(active), abi.dptr(f_add), int(refresh),
                                           C.byref(nc)))
        return nc.value

    @staticmethod
    def _gptr(g_lb):
        if g_lb is None:
            return C.POINTER(C.c_double)()
        return C.cast((C.c_double * 3)(*g_lb), C.POINTER(C.c_double))

    def lbm_step_ibm(self, x, v, mass, f_add, g_lb=None, active=None):
        """LB step + the refresh IBM sub-step of its cycle (host arrays);
        f_add (n,3) is incremented in place.  Same results as lbm_step then
        ibm_substep(refresh=True)."""
        n = int(x.shape[0])
        nc = C.c_int(0)
        g = self._gptr(g_lb)
        self._ck(self.L.couplb_lbm_step_ibm(self.h, g, n, abi.dptr(x), abi.dptr(v), abi.dptr(mass),
                                            abi.iptr(active), abi.dptr(f_add), C.byref(nc)))
        return nc.value

    def lbm_step_ibm_device(self, n, x_ptr, v_ptr, m_ptr, f_ptr, active_ptr=0, g_lb=None):
        """LB step + the refresh IBM sub-step of its cycle (device pointers)."""
        g = self._gptr(g_lb)
        self._ck(self.L.couplb_lbm_step_ibm_device(self.h, g, n, C.c_void_p(x_ptr), C.c_void_p(v_ptr),
                                                   C.c_void_p(m_ptr), C.c_void_p(active_ptr or None),
                                                   C.c_void_p(f_ptr)))

    def ibm_substep_device(self, n, x_ptr, v_ptr, m_ptr, f_ptr, active_ptr=0, refresh=True):
        """Device-array IBM sub-step (raw device pointers, e.g. tensor.data_ptr())."""
        self._ck(self.L.couplb_ibm_substep_device(self.h, n, C.c_void_p(x_ptr), C.c_void_p(v_ptr),
                                                  C.c_void_p(m_ptr), C.c_void_p(active_ptr or None),
                                                  C.c_void_p(f_ptr), int(refresh)))

    def set_ibm_method(self, method="single", passes=1, slip_tol=0.0, model=None):
        """IBM forcing method: "single" (the reference's pass), "iterative"
        (passes-1 correction passes) or "learned" (network correction with the
        iterative fallback above slip_tol); model: a CorrectionNet."""
        m = abi.IbmMethod()
        m.method = abi.IBM_METHODS[method] if isinstance(method, str) else int(method)
        m.passes, m.slip_tol = int(passes), float(slip_tol)
        m.model = model.h if model is not None else None
        self._ck(self.L.couplb_set_ibm_method(self.h, C.byref(m)))
        self._model = model

    def ibm_slip(self, reset=False):
        """dict of the last slip measurement (synchronises)."""
        out = np.zeros(8)
        self._ck(self.L.couplb_ibm_slip(self.h, abi.dptr(out), int(reset)))
        keys = ["rms", "max", "check_rms", "check_max", "markers", "fell_back", "checks",
                "fallbacks"]
        return dict(zip(keys, out.tolist()))

    def ibm_record(self, rows_ptr, capacity):
        """Capture training rows into device memory (pointer, rows); 0 stops."""
        self._ck(self.L.couplb_ibm_record(self.h, C.c_void_p(rows_ptr or None), int(capacity)))

    def ibm_record_count(self):
        v = C.c_longlong(0)
        self._ck(self.L.couplb_ibm_record_count(self.h, C.byref(v)))
        return v.value

    def ibm_total_force(self, reset=False):
        out = np.zeros(3)
        self._ck(self.L.couplb_ibm_total_force(self.h, abi.dptr(out), int(reset)))
        return out
