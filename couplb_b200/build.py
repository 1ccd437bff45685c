"""Build of the CUDA library libcouplb_b200.so (sm_100a), in-tree.

    python -m couplb_b200.build          # build if sources changed
    python -m couplb_b200.build --force  # always rebuild
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libcouplb_b200.so")
SOURCES = ["engine.cu", "engine_ibm.cu", "engine_methods_f64.cu", "engine_methods_f32.cu",
           "engine_methods_f16.cu", "fix_core.cpp", "noalloc.cu", "mlp.cu", "vtk_io.cpp"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-shared",
]


def _inputs():
    files = [os.path.join(INCLUDE, "couplb_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".cpp", ".h")):
            files.append(os.path.join(CSRC, f))
    return files


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force=False, verbose=False):
    """Compile every source to an object in parallel (couplb_b200/_build),
    then link the shared library."""
    if not force and not needs_build():
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmd = [nvcc()] + compile_flags + ["-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, cwd=CSRC, env=env)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC, env=env)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
