"""Loader of libcouplb_b200.so, the CUDA library behind the C ABI.

There is no CPU fallback: when the library is missing or cannot be loaded,
load() raises.  The library is built in-tree by couplb_b200.build.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcouplb_b200.so")

_lib = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_H = C.c_void_p

# name -> (restype, argtypes); the exported symbols of include/couplb_b200.h
SIGNATURES = {
    "couplb_version": (C.c_int, []),
    "couplb_struct_size": (C.c_size_t, [C.c_int]),
    "couplb_last_error": (C.c_char_p, [_H]),
    "couplb_create": (C.c_int, [C.POINTER(abi.LatticeParams), C.POINTER(_H)]),
    "couplb_destroy": (C.c_int, [_H]),
    "couplb_set_stream": (C.c_int, [_H, C.c_void_p]),
    "couplb_synchronize": (C.c_int, [_H]),
    "couplb_init_equilibrium": (C.c_int, [_H, C.c_double, C.c_double, C.c_double, C.c_double]),
    "couplb_set_populations": (C.c_int, [_H, _D]),
    "couplb_get_populations": (C.c_int, [_H, _D]),
    "couplb_ghost_nodes": (C.c_size_t, [_H]),
    "couplb_lbm_step": (C.c_int, [_H, _D]),
    "couplb_macroscopic": (C.c_int, [_H]),
    "couplb_halo_attach": (C.c_int, [_H, C.c_int, C.c_void_p]),
    "couplb_halo_bytes": (C.c_size_t, [_H]),
    "couplb_halo_pack": (C.c_int, [_H, C.c_int, C.c_void_p]),
    "couplb_ibm_halo_bytes": (C.c_size_t, [_H, C.c_int]),
    "couplb_ibm_halo_attach": (C.c_int, [_H, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "couplb_ibm_halo_moments": (C.c_int, [_H, C.c_int, C.c_int, C.c_void_p]),
    "couplb_ibm_halo_fold": (C.c_int, [_H, C.c_int, C.c_int, C.c_void_p]),
    "couplb_get_macroscopic": (C.c_int, [_H, _D, _D, _D, _D]),
    "couplb_get_force_field": (C.c_int, [_H, _D, _D, _D]),
    "couplb_set_force_field": (C.c_int, [_H, _D, _D, _D]),
    "couplb_diagnostics": (C.c_int, [_H, C.POINTER(abi.Diag)]),
    "couplb_y_profile": (C.c_int, [_H, _D, _D, _D]),
    "couplb_diagnostics_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_longlong, C.c_int, C.c_double, C.c_void_p,
                                             C.c_void_p]),
    "couplb_set_ibm_params": (C.c_int, [_H, C.POINTER(abi.IbmParams)]),
    "couplb_ibm_substep": (C.c_int, [_H, C.c_int, _D, _D, _D, _I, _D, C.c_int, _I]),
    "couplb_ibm_substep_device": (C.c_int, [_H, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_int]),
    "couplb_ibm_total_force": (C.c_int, [_H, _D, C.c_int]),
    "couplb_lbm_step_ibm": (C.c_int, [_H, _D, C.c_int, _D, _D, _D, _I, _D, _I]),
    "couplb_lbm_step_ibm_device": (C.c_int, [_H, _D, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p]),
    "couplb_read_status": (C.c_int, [_H, _I, _I, C.c_int]),
    "couplb_status_post": (C.c_int, [_H]),
    "couplb_status_last": (C.c_int, [_H, _I, _I]),
    "couplb_set_ibm_method": (C.c_int, [_H, C.POINTER(abi.IbmMethod)]),
    "couplb_ibm_slip": (C.c_int, [_H, _D, C.c_int]),
    "couplb_ibm_record": (C.c_int, [_H, C.c_void_p, C.c_longlong]),
    "couplb_ibm_record_count": (C.c_int, [_H, C.POINTER(C.c_longlong)]),
    "couplb_mlp_create": (C.c_int, [C.c_int, C.c_ulonglong, C.POINTER(_H)]),
    "couplb_mlp_destroy": (C.c_int, [_H]),
    "couplb_mlp_last_error": (C.c_char_p, [_H]),
    "couplb_mlp_set_stream": (C.c_int, [_H, C.c_void_p]),
    "couplb_mlp_set_weights": (C.c_int, [_H, C.c_void_p, C.c_double, C.c_double]),
    "couplb_mlp_get_weights": (C.c_int, [_H, C.c_void_p, _D, _D]),
    "couplb_mlp_fit_scales": (C.c_int, [_H, C.c_void_p, C.c_longlong]),
    "couplb_mlp_forward": (C.c_int, [_H, C.c_void_p, C.c_longlong, C.c_void_p]),
    "couplb_mlp_loss_grad": (C.c_int, [_H, C.c_void_p, C.c_longlong, _D, C.c_void_p]),
    "couplb_mlp_train": (C.c_int, [_H, C.c_void_p, C.c_longlong, C.POINTER(abi.MlpTrainParams),
                                   _D, _D]),
    "couplb_mlp_save": (C.c_int, [_H, C.c_char_p]),
    "couplb_mlp_load": (C.c_int, [_H, C.c_char_p]),
    "couplb_device_bytes": (C.c_size_t, [_H]),
    "couplb_set_option": (C.c_int, [_H, C.c_char_p, C.c_longlong]),
    "couplb_get_option": (C.c_int, [_H, C.c_char_p, C.POINTER(C.c_longlong)]),
    "couplb_fix_parse": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.c_int,
                                   C.POINTER(abi.FixConfig), C.c_char_p, C.c_int]),
    "couplb_fix_create": (C.c_int, [C.POINTER(abi.FixConfig), C.POINTER(_H)]),
    "couplb_fix_destroy": (C.c_int, [_H]),
    "couplb_fix_last_error": (C.c_char_p, [_H]),
    "couplb_fix_set_gravity_callback": (C.c_int, [_H, C.c_void_p, C.c_void_p]),
    "couplb_fix_set_log_callback": (C.c_int, [_H, C.c_void_p, C.c_void_p]),
    "couplb_fix_set_gravity_values": (C.c_int, [_H, _D]),
    "couplb_fix_set_device": (C.c_int, [_H, C.c_int]),
    "couplb_fix_set_comm": (C.c_int, [_H, C.c_void_p]),
    "couplb_fix_setmask": (C.c_int, []),
    "couplb_fix_init": (C.c_int, [_H, C.POINTER(abi.Domain)]),
    "couplb_fix_setup": (C.c_int, [_H, C.POINTER(abi.Atoms), C.c_longlong]),
    "couplb_fix_post_force": (C.c_int, [_H, C.POINTER(abi.Atoms), C.c_longlong]),
    "couplb_fix_end_of_step": (C.c_int, [_H, C.c_longlong]),
    "couplb_fix_write_solid": (C.c_int, [_H, C.POINTER(abi.Atoms), C.c_longlong]),
    "couplb_fix_handle": (_H, [_H]),
    "couplb_fix_scales": (C.c_int, [_H, _D]),
    "couplb_fix_last_diag": (C.c_int, [_H, C.POINTER(abi.Diag)]),
    "couplb_fix_lbm_steps": (C.c_longlong, [_H]),
}

GRAVITY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double))
LOG_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_char_p)


class CoupLBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


def load(path=LIB_PATH):
    """Load the CUDA library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m couplb_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, handle=None, fix=None):
    if rc != 0:
        lib = load()
        if fix is not None:
            msg = lib.couplb_fix_last_error(fix)
        else:
            msg = lib.couplb_last_error(handle)
        raise CoupLBError(rc, (msg or b"").decode(errors="replace"))
    return rc
