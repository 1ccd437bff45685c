"""The C-ABI library loads without a GPU and exports every entry point that
include/couplb_b200.h declares, with struct layouts matching the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess

import pytest

from couplb_b200 import abi, build, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "couplb_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(couplb_[a-z0-9_]+)\s*\(", src)
    return sorted(set(n for n in names if not n.endswith("_fn")))


def test_library_builds_and_loads(cuda_lib):
    assert os.path.exists(lib.LIB_PATH)
    assert cuda_lib.couplb_version() == 1


def test_every_declared_symbol_is_exported(cuda_lib):
    names = declared_functions()
    assert len(names) > 30
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the Python bindings know every one of them
    assert not [n for n in names if n not in lib.SIGNATURES], [n for n in names if n not in lib.SIGNATURES]


@pytest.mark.parametrize("which,cls", [(0, abi.LatticeParams), (1, abi.IbmParams), (2, abi.Diag),
                                       (3, abi.FixConfig), (4, abi.Domain), (5, abi.Atoms),
                                       (6, abi.IbmMethod), (7, abi.MlpTrainParams)])
def test_struct_layouts(cuda_lib, which, cls):
    assert cuda_lib.couplb_struct_size(which) == C.sizeof(cls)


def test_create_fails_cleanly_without_gpu_or_bad_args(cuda_lib):
    p = abi.LatticeParams()
    p.dim, p.nx, p.ny, p.nz, p.tau, p.rho0 = 3, 4, 4, 4, 0.4, 1.0   # tau <= 0.5
    h = C.c_void_p()
    rc = cuda_lib.couplb_create(C.byref(p), C.byref(h))
    assert rc == abi.ERR_ARG
    assert b"tau" in cuda_lib.couplb_last_error(None)


def test_build_is_sm100a():
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS
