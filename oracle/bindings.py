"""ctypes bindings of the CPU oracles (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline to check
or time the CUDA path; the product never imports this module.

    kind="port" -> oracle/libcouplb_oracle.so   (plain-C restatement)
    kind="ref"  -> oracle/_ref/libcouplb_ref.so (reference headers, parity build)
    kind="ref_fast" -> oracle/_ref/libcouplb_ref_fast.so (-O3, timed baseline)
"""
import ctypes as C
import os
import subprocess

import numpy as np

from couplb_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {
    "port": ("libcouplb_oracle.so", "orc_"),
    "ref": (os.path.join("_ref", "libcouplb_ref.so"), "ref_"),
    "ref_fast": (os.path.join("_ref", "libcouplb_ref_fast.so"), "ref_"),
}
_cache = {}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_V = C.c_void_p


def available(kind):
    return os.path.exists(os.path.join(HERE, _LIBS[kind][0]))


def build_port():
    """Compile the plain-C oracle (needs only gcc)."""
    subprocess.run(["make", "-s", "libcouplb_oracle.so"], cwd=HERE, check=True,
                   env={**os.environ, "CC": "gcc"})


def load(kind="port"):
    if kind in _cache:
        return _cache[kind]
    path, pre = _LIBS[kind]
    full = os.path.join(HERE, path)
    if not os.path.exists(full):
        if kind == "port":
            build_port()
        else:
            raise FileNotFoundError(f"{full} not built (needs the reference sources)")
    lib = C.CDLL(full)
    sig = {
        "grid_create": (_V, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _I, _D]),
        "grid_destroy": (None, [_V]),
        "grid_ntotal": (C.c_long, [_V]),
        "grid_init_equilibrium": (None, [_V, C.c_double, C.c_double, C.c_double, C.c_double]),
        "grid_set_f": (None, [_V, _D]),
        "grid_get_f": (None, [_V, _D]),
        "grid_get_macro": (None, [_V, _D, _D, _D, _D]),
        "grid_set_force": (None, [_V, _D, _D, _D]),
        "grid_get_force": (None, [_V, _D, _D, _D]),
        "grid_lbm_step": (None, [_V, _D]),
        "grid_macroscopic": (None, [_V, C.c_int]),
        "grid_exchange_velocity": (None, [_V]),
        "grid_fold_forces": (None, [_V]),
        "grid_diagnostics": (None, [_V, _D, _I]),
        "grid_ibm_substep": (C.c_int, [_V, C.POINTER(abi.IbmParams), C.c_int, _D, _D, _D, _I, _D,
                                       C.c_int, C.c_int]),
        "fix_create": (_V, [C.POINTER(abi.FixConfig), C.POINTER(abi.Domain), C.c_char_p, C.c_int]),
        "fix_destroy": (None, [_V]),
        "fix_setup": (C.c_int, [_V, C.POINTER(abi.Atoms), C.c_longlong]),
        "fix_post_force": (C.c_int, [_V, C.POINTER(abi.Atoms), C.c_longlong]),
        "fix_end_of_step": (C.c_int, [_V, C.c_longlong]),
        "fix_set_gravity": (None, [_V, _D]),
        "fix_grid": (_V, [_V]),
        "fix_last_diag": (None, [_V, _D, _I]),
        "fix_scales": (None, [_V, _D]),
        "fix_last_error": (C.c_char_p, [_V]),
    }
    if kind == "port":
        # project definitions without a reference counterpart
        sig.update({
            "grid_ibm_substep_method": (C.c_int, [_V, C.POINTER(abi.IbmParams), C.c_int, _D, _D, _D,
                                                  _I, _D, C.c_int, C.c_int, C.c_int, C.c_int,
                                                  C.c_double, _D, C.c_double, C.c_double, _D, _D,
                                                  _D]),
            "mlp_forward": (None, [_D, C.c_double, C.c_double, C.c_int, _D, C.c_int, _D]),
            "grid_set_ibm_wrap": (None, [_V, C.c_int]),
            "mlp_loss_grad": (C.c_double, [_D, C.c_double, C.c_double, C.c_int, _D, _D]),
        })
    fns = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, pre + name)
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    _cache[kind] = fns
    return fns


def _d(a):
    return abi.dptr(a)


class OracleGrid:
    """One subdomain on the CPU oracle, reference (ghost-inclusive) layout."""

    def __init__(self, dim, nx, ny, nz, tau, rho0=1.0, wall=(0,) * 6, wall_vel=(0.0,) * 3,
                 kind="port", handle=None, owner=None):
        self.L = load(kind)
        self.dim, self.nx, self.ny = dim, nx, ny
        self.nz = nz if dim == 3 else 1
        self.Q = 19 if dim == 3 else 9
        self.gx, self.gy = nx + 2, ny + 2
        self.gz = self.nz + 2 if dim == 3 else 1
        self._owner = owner
        if handle is None:
            w = (C.c_int * 6)(*wall)
            v = (C.c_double * 3)(*wall_vel)
            self.h = self.L["grid_create"](dim, nx, ny, self.nz, tau, rho0,
                                           C.cast(w, _I), C.cast(v, _D))
            self._own = True
        else:
            self.h = handle
            self._own = False
        self.G = int(self.L["grid_ntotal"](self.h))

    def close(self):
        if self._own and self.h:
            self.L["grid_destroy"](self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self):
        return (self.gz, self.gy, self.gx)

    def init_equilibrium(self, rho, ux=0.0, uy=0.0, uz=0.0):
        self.L["grid_init_equilibrium"](self.h, rho, ux, uy, uz)

    def set_f(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(self.Q * self.G)
        self.L["grid_set_f"](self.h, _d(f))

    def get_f(self):
        f = np.empty(self.Q * self.G)
        self.L["grid_get_f"](self.h, _d(f))
        return f.reshape(self.Q, self.gz, self.gy, self.gx)

    def get_macro(self):
        out = [np.empty(self.G) for _ in range(4)]
        self.L["grid_get_macro"](self.h, *[_d(a) for a in out])
        return [a.reshape(self.shape()) for a in out]

    def set_force(self, fx, fy, fz):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(self.G) for a in (fx, fy, fz)]
        self.L["grid_set_force"](self.h, *[_d(a) for a in arrs])

    def get_force(self):
        out = [np.empty(self.G) for _ in range(3)]
        self.L["grid_get_force"](self.h, *[_d(a) for a in out])
        return [a.reshape(self.shape()) for a in out]

    def lbm_step(self, g_lb=None):
        if g_lb is None:
            self.L["grid_lbm_step"](self.h, _D())
        else:
            g = np.asarray(g_lb, dtype=np.float64)
            self.L["grid_lbm_step"](self.h, _d(g))

    def macroscopic(self, guo=False):
        self.L["grid_macroscopic"](self.h, int(guo))

    def diagnostics(self):
        out = np.empty(5)
        cl = C.c_int(0)
        self.L["grid_diagnostics"](self.h, _d(out), C.byref(cl))
        return out, cl.value

    def set_ibm_wrap(self, mask):
        """Periodic wrap of the IBM window along the axes of bit mask
        (port oracle only; the reference clips)."""
        self.L["grid_set_ibm_wrap"](self.h, int(mask))

    def ibm_substep(self, ip, x, v, mass, f_add, active=None, refresh=True, fold=True):
        n = x.shape[0]
        return self.L["grid_ibm_substep"](self.h, C.byref(ip), n, _d(x), _d(v), _d(mass),
                                          abi.iptr(active), _d(f_add), int(refresh), int(fold))


    def ibm_substep_method(self, ip, x, v, mass, f_add, method, passes, slip_tol=0.0,
                           mlp=None, g_lb=(0.0, 0.0, 0.0), active=None, refresh=True, fold=True,
                           rows=False):
        """One sub-step with a forcing method (1 iterative, 2 learned; port
        oracle only).  mlp: (weights float64[MLP_NPARAM], s_in, s_out).
        Returns (coupled, stats[6], rows or None)."""
        n = x.shape[0]
        st = np.zeros(6)
        rw = np.zeros((n, MLP_ROW)) if rows else None
        w, s_in, s_out = mlp if mlp is not None else (None, 1.0, 1.0)
        wv = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        gl = np.asarray(g_lb, dtype=np.float64)
        nc = self.L["grid_ibm_substep_method"](
            self.h, C.byref(ip), n, _d(x), _d(v), _d(mass), abi.iptr(active), _d(f_add),
            int(refresh), int(fold), int(method), int(passes), float(slip_tol),
            _D() if wv is None else _d(wv), float(s_in), float(s_out), _d(gl), _d(st),
            _D() if rw is None else _d(rw))
        return nc, st, rw


MLP_IN, MLP_HID, MLP_OUT, MLP_ROW = 84, 64, 3, 88
MLP_NPARAM = MLP_HID * MLP_IN + MLP_HID + MLP_HID * MLP_HID + MLP_HID + MLP_OUT * MLP_HID + MLP_OUT


def mlp_forward(w, s_in, s_out, x):
    """FP64 network output for inputs x (n x 84, or rows n x 88)."""
    L = load("port")
    x = np.ascontiguousarray(x, dtype=np.float64)
    n, stride = x.shape
    y = np.empty((n, MLP_OUT))
    L["mlp_forward"](_d(np.ascontiguousarray(w, dtype=np.float64)), s_in, s_out, n, _d(x),
                     stride, _d(y))
    return y


def mlp_loss_grad(w, s_in, s_out, rows):
    """FP64 loss and gradient over sample rows (n x 88)."""
    L = load("port")
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    g = np.empty(MLP_NPARAM)
    loss = L["mlp_loss_grad"](_d(np.ascontiguousarray(w, dtype=np.float64)), s_in, s_out,
                              rows.shape[0], _d(rows), _d(g))
    return loss, g


class OracleFix:
    """FixCoupLB hooks on the CPU oracle."""

    def __init__(self, cfg, domain, kind="port"):
        self.L = load(kind)
        err = C.create_string_buffer(256)
        self.h = self.L["fix_create"](C.byref(cfg), C.byref(domain), err, 256)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.cfg = cfg
        dim = domain.dimension
        sc = self.scales()
        g = self.L["fix_grid"](self.h)
        self.grid = OracleGrid(dim, 1, 1, 1, 1.0, kind=kind, handle=g, owner=self)
        # fix the grid geometry from the config (single rank)
        self.grid.nx, self.grid.ny = cfg.Nx, cfg.Ny
        self.grid.nz = cfg.Nz if dim == 3 else 1
        self.grid.gx, self.grid.gy = cfg.Nx + 2, cfg.Ny + 2
        self.grid.gz = self.grid.nz + 2 if dim == 3 else 1
        self.grid.G = int(self.L["grid_ntotal"](g))
        self._scales = sc

    def scales(self):
        out = np.empty(6)
        self.L["fix_scales"](self.h, _d(out))
        return dict(zip(["dx", "dt_lbm", "vel_scale", "force_scale", "nu_lb", "tau"], out))

    def set_gravity(self, g):
        self.L["fix_set_gravity"](self.h, _d(np.asarray(g, dtype=np.float64)))

    def setup(self, atoms, step=0):
        return self.L["fix_setup"](self.h, C.byref(atoms), step)

    def post_force(self, atoms, step):
        return self.L["fix_post_force"](self.h, C.byref(atoms), step)

    def end_of_step(self, step):
        return self.L["fix_end_of_step"](self.h, step)

    def last_diag(self):
        out = np.empty(5)
        cl = C.c_int(0)
        self.L["fix_last_diag"](self.h, _d(out), C.byref(cl))
        return out, cl.value

    def close(self):
        if self.h:
            self.L["fix_destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
