"""Sphere drag with the IBM forcing methods: a rigid sphere of Fibonacci
markers (held fixed, v = 0, m = 1, xi = 1, Roma kernel, md_per_lb = 1) in a
periodic D3Q19 box driven by a uniform body force.  Runs the single penalty
pass, the multi-pass iterative correction and the learned correction on the
GPU, generates training rows from iterative runs and trains the network on
them with the library's own kernels.

Quantities, per LB step after the forcing: slip = RMS over markers of
|U - v| with U the interpolated velocity the next collision sees; drag = sum
over markers of the x force the fluid exerts on them.
"""
import numpy as np

from .lattice import Lattice
from .markers import fibonacci_sphere
from .mlp import CorrectionNet
from . import abi


class SphereCase:
    def __init__(self, n=192, radius=12.0, offset=(0.0, 0.0, 0.0), g=2e-6, tau=0.8,
                 precision="fp32", device=0):
        import torch
        self.torch = torch
        self.n, self.g = n, (float(g), 0.0, 0.0)
        self.L = Lattice(3, n, n, n, tau=tau, body_force=True, precision=precision, device=device)
        self.stream = torch.cuda.current_stream(device)
        self.L.set_stream(self.stream.cuda_stream)
        self.L.init_equilibrium(1.0)
        self.L.set_ibm_params(delta="roma", md_per_lb=1, xi_ibm=1.0, dt_lbm=1.0, dx=1.0)
        c = np.full(3, n / 2.0) + np.asarray(offset, dtype=np.float64)
        x = fibonacci_sphere(radius, c)
        dev = f"cuda:{device}"
        self.nm = x.shape[0]
        self.x = torch.from_numpy(x).to(dev)
        self.v = torch.zeros_like(self.x)
        self.m = torch.ones(self.nm, dtype=torch.float64, device=dev)
        self.f = torch.zeros_like(self.x)
        self.drag = torch.zeros((), dtype=torch.float64, device=dev)

    def set_method(self, method, passes=5, slip_tol=0.0, net=None):
        self.L.set_ibm_method(method, passes=passes, slip_tol=slip_tol, model=net)

    def force(self):
        self.f.zero_()
        self.L.ibm_substep_device(self.nm, self.x.data_ptr(), self.v.data_ptr(), self.m.data_ptr(),
                                  self.f.data_ptr(), 0, refresh=True)

    def step(self):
        self.force()
        self.L.lbm_step(self.g)

    def run(self, steps, slip_from=None):
        """steps LB steps; from step slip_from on, read the slip after every
        forcing (synchronises).  Returns (slip list, final drag)."""
        slips = []
        for s in range(steps):
            self.force()
            if slip_from is not None and s >= slip_from:
                slips.append(self.L.ibm_slip()["rms"])
            self.L.lbm_step(self.g)
        drag = float(self.f[:, 0].sum())
        return slips, drag

    def time_forcing(self, steps):
        """Mean device time (ms) of the IBM call and of the whole LB step.
        The timed calls run without the slip statistics of the forcing
        methods (handle option ibm_slip 0), which only diagnostics read."""
        torch = self.torch
        self.L.set_option("ibm_slip", 0)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
               torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b, c in ev:
            self.f.zero_()
            a.record(self.stream)
            self.L.ibm_substep_device(self.nm, self.x.data_ptr(), self.v.data_ptr(),
                                      self.m.data_ptr(), self.f.data_ptr(), 0, refresh=True)
            b.record(self.stream)
            self.L.lbm_step(self.g)
            c.record(self.stream)
        torch.cuda.synchronize()
        self.L.set_option("ibm_slip", 1)
        ibm = sum(a.elapsed_time(b) for a, b, _ in ev) / steps
        tot = sum(a.elapsed_time(c) for a, _, c in ev) / steps
        return ibm, tot

    def close(self):
        self.L.close()


def generate_rows(runs, steps, every, n=192, radius=12.0, passes=5, seed=11, precision="fp32",
                  device=0):
    """Training rows from iterative runs: `runs` spheres at random sub-cell
    offsets and body forces 1e-6..3e-6, `steps` LB steps each, rows captured
    every `every` steps.  Returns a device tensor (rows x COUPLB_MLP_ROW)."""
    import torch
    rng = np.random.default_rng(seed)
    per = fibonacci_sphere(radius, (0.0, 0.0, 0.0)).shape[0]
    cap = runs * (steps // every + 1) * per
    rows = torch.zeros((cap, abi.MLP_ROW), dtype=torch.float32, device=f"cuda:{device}")
    used = 0
    for r in range(runs):
        case = SphereCase(n=n, radius=radius, offset=rng.random(3), g=1e-6 + 2e-6 * rng.random(),
                          precision=precision, device=device)
        case.set_method("iterative", passes=passes)
        for s in range(steps):
            rec = s % every == 0
            if rec:
                case.L.ibm_record(rows.data_ptr() + 4 * abi.MLP_ROW * used, cap - used)
            case.step()
            if rec:
                used += case.L.ibm_record_count()
                case.L.ibm_record(0, 0)
        case.close()
    torch.cuda.synchronize()
    return rows[:used]


def train_net(rows, epochs=30, batch=4096, lr=2e-3, lr_final=2e-5, val_frac=0.05, seed=1,
              device=0):
    net = CorrectionNet(device, seed=seed)
    n = rows.shape[0]
    net.fit_scales(rows.data_ptr(), n)
    tl, vl = net.train(rows.data_ptr(), n, epochs=epochs, batch=batch, lr=lr, lr_final=lr_final,
                       n_val=int(val_frac * n), seed=seed + 100)
    return net, tl, vl
