"""The no-slip correction network (84-64-64-3, BF16 weights) and its
GPU training, through the couplb_mlp_* C ABI.

Rows are COUPLB_MLP_ROW = 88 floats in device memory: 84 inputs (u0 at the 27
nodes round(l)-1..round(l)+1 of a marker, then v / vel_scale), 3 targets (the correction beyond
the penalty pass over m xi vel_scale / dt), 1 unused.
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import CoupLBError, load


class CorrectionNet:
    def __init__(self, device=0, seed=1):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.couplb_mlp_create(int(device), int(seed), C.byref(h))
        if rc:
            raise CoupLBError(rc, "couplb_mlp_create failed")
        self.h = h
        self.device = device

    def _ck(self, rc):
        if rc:
            raise CoupLBError(rc, (self.L.couplb_mlp_last_error(self.h) or b"").decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.couplb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._ck(self.L.couplb_mlp_set_stream(self.h, C.c_void_p(stream_ptr or None)))

    def set_weights(self, w, s_in, s_out):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == abi.MLP_NPARAM
        self._ck(self.L.couplb_mlp_set_weights(self.h, w.ctypes.data, float(s_in), float(s_out)))

    def get_weights(self):
        w = np.empty(abi.MLP_NPARAM, dtype=np.float32)
        si, so = C.c_double(0), C.c_double(0)
        self._ck(self.L.couplb_mlp_get_weights(self.h, w.ctypes.data, C.byref(si), C.byref(so)))
        return w, si.value, so.value

    def fit_scales(self, rows_ptr, n):
        self._ck(self.L.couplb_mlp_fit_scales(self.h, C.c_void_p(rows_ptr), int(n)))

    def forward(self, rows_ptr, n, out_ptr):
        self._ck(self.L.couplb_mlp_forward(self.h, C.c_void_p(rows_ptr), int(n), C.c_void_p(out_ptr)))

    def loss_grad(self, rows_ptr, n):
        g = np.empty(abi.MLP_NPARAM, dtype=np.float32)
        loss = C.c_double(0)
        self._ck(self.L.couplb_mlp_loss_grad(self.h, C.c_void_p(rows_ptr), int(n), C.byref(loss),
                                             g.ctypes.data))
        return loss.value, g

    def train(self, rows_ptr, n, epochs=20, batch=4096, lr=2e-3, lr_final=5e-5, beta1=0.9,
              beta2=0.999, eps=1e-8, seed=7, n_val=0):
        tp = abi.MlpTrainParams()
        tp.epochs, tp.batch, tp.lr, tp.lr_final = int(epochs), int(batch), lr, lr_final
        tp.beta1, tp.beta2, tp.eps, tp.seed, tp.n_val = beta1, beta2, eps, int(seed), int(n_val)
        tl, vl = C.c_double(0), C.c_double(0)
        self._ck(self.L.couplb_mlp_train(self.h, C.c_void_p(rows_ptr), int(n), C.byref(tp),
                                         C.byref(tl), C.byref(vl)))
        return tl.value, vl.value

    def save(self, path):
        self._ck(self.L.couplb_mlp_save(self.h, str(path).encode()))

    def load(self, path):
        self._ck(self.L.couplb_mlp_load(self.h, str(path).encode()))
