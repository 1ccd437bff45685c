"""ctypes mirror of the structs in include/couplb_b200.h.

The layouts here must match the C header field for field; tests/test_abi.py
checks the sizes against the compiled library.
"""
import ctypes as C

PATH_MAX = 256
VTK_MAX_ATTR = 32

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_STATE = -3
ERR_NUMERIC = -4
ERR_IO = -5
ERR_PARSE = -6
ERR_UNSUPPORTED = -7
ERR_TOO_LARGE = -8

FP64 = 0
FP32_SHIFTED = 1
FP16_SHIFTED = 2
PRECISIONS = {"fp64": FP64, "fp32": FP32_SHIFTED, "fp16": FP16_SHIFTED}

DELTA_ROMA = 0
DELTA_PESKIN4 = 1

IBM_SINGLE = 0
IBM_ITERATIVE = 1
IBM_LEARNED = 2
IBM_METHODS = {"single": IBM_SINGLE, "iterative": IBM_ITERATIVE, "learned": IBM_LEARNED}

MLP_IN, MLP_HID, MLP_OUT, MLP_ROW, MLP_NPARAM = 84, 64, 3, 88, 9795

G_NONE = 0
G_CONSTANT = 1
G_EQUAL = 2


class LatticeParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("tau", C.c_double),
        ("rho0", C.c_double),
        ("wall", C.c_int * 6),
        ("wall_vel", C.c_double * 3),
        ("body_force", C.c_int),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class IbmParams(C.Structure):
    _fields_ = [
        ("delta", C.c_int),
        ("md_per_lb", C.c_int),
        ("xi_ibm", C.c_double),
        ("dt_lbm", C.c_double),
        ("dx", C.c_double),
        ("vel_scale", C.c_double),
        ("force_scale", C.c_double),
        ("domain_lo", C.c_double * 3),
        ("offset", C.c_int * 3),
    ]


class IbmMethod(C.Structure):
    _fields_ = [
        ("method", C.c_int),
        ("passes", C.c_int),
        ("slip_tol", C.c_double),
        ("model", C.c_void_p),
    ]


class MlpTrainParams(C.Structure):
    _fields_ = [
        ("epochs", C.c_int),
        ("batch", C.c_int),
        ("lr", C.c_double),
        ("lr_final", C.c_double),
        ("beta1", C.c_double),
        ("beta2", C.c_double),
        ("eps", C.c_double),
        ("seed", C.c_ulonglong),
        ("n_val", C.c_longlong),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("umax", C.c_double),
        ("mass", C.c_double),
        ("mom", C.c_double * 3),
        ("clamps", C.c_int),
        ("nonfinite", C.c_int),
    ]


class FixConfig(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
        ("nu", C.c_double), ("rho", C.c_double),
        ("md_per_lb", C.c_int),
        ("xi_ibm", C.c_double),
        ("gstyle", C.c_int * 3),
        ("gconst", C.c_double * 3),
        ("gvar", (C.c_char * 64) * 3),
        ("wall", C.c_int * 6),
        ("wall_vel", C.c_double * 3),
        ("output_every", C.c_int),
        ("output_file", C.c_char * PATH_MAX),
        ("check_every", C.c_int),
        ("delta", C.c_int),
        ("vtk_every", C.c_int),
        ("vtk_prefix", C.c_char * PATH_MAX),
        ("has_vtk_region", C.c_int),
        ("vtk_region_n", C.c_int),
        ("vtk_rlo", C.c_double * 3),
        ("vtk_rhi", C.c_double * 3),
        ("vtk_solid_nattr", C.c_int),
        ("checkpoint_every", C.c_int),
        ("checkpoint_prefix", C.c_char * PATH_MAX),
        ("do_restart", C.c_int),
        ("restart_prefix", C.c_char * PATH_MAX),
        ("precision", C.c_int),
        ("dimension", C.c_int),
        ("ibm_method", C.c_int),
        ("ibm_passes", C.c_int),
        ("slip_tol", C.c_double),
        ("mlp_model", C.c_char * PATH_MAX),
        ("vtk_solid_attr", (C.c_char * 16) * VTK_MAX_ATTR),
        ("ibm_window", C.c_int),
    ]


class Domain(C.Structure):
    _fields_ = [
        ("dimension", C.c_int),
        ("boxlo", C.c_double * 3), ("boxhi", C.c_double * 3),
        ("sublo", C.c_double * 3), ("subhi", C.c_double * 3),
        ("periodicity", C.c_int * 3),
        ("dt", C.c_double),
        ("ntimestep", C.c_longlong),
    ]


class Atoms(C.Structure):
    _fields_ = [
        ("nlocal", C.c_int),
        ("x", C.POINTER(C.c_double)),
        ("v", C.POINTER(C.c_double)),
        ("f", C.POINTER(C.c_double)),
        ("mask", C.POINTER(C.c_int)),
        ("groupbit", C.c_int),
        ("rmass", C.POINTER(C.c_double)),
        ("mass", C.POINTER(C.c_double)),
        ("type", C.POINTER(C.c_int)),
        ("tag", C.POINTER(C.c_longlong)),
        ("molecule", C.POINTER(C.c_longlong)),
        ("radius", C.POINTER(C.c_double)),
        ("mu", C.POINTER(C.c_double)),
        ("omega", C.POINTER(C.c_double)),
        ("torque", C.POINTER(C.c_double)),
    ]


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or NULL for None)."""
    if a is None:
        return C.POINTER(C.c_double)()
    assert a.dtype.name == "float64" and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    """int* of a C-contiguous int32 numpy array (or NULL for None)."""
    if a is None:
        return C.POINTER(C.c_int)()
    assert a.dtype.name == "int32" and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def make_atoms(x, v, f, mask=None, groupbit=1, rmass=None, mass=None, type_=None):
    """Atoms struct over numpy arrays (x, v, f: (n,3) float64)."""
    at = Atoms()
    at.nlocal = 0 if x is None else int(x.shape[0])
    at.x, at.v, at.f = dptr(x), dptr(v), dptr(f)
    at.mask = iptr(mask)
    at.groupbit = groupbit
    at.rmass = dptr(rmass)
    at.mass = dptr(mass)
    at.type = iptr(type_)
    return at


def make_domain(dimension, boxlo, boxhi, dt, periodicity=(1, 1, 1), ntimestep=0, sublo=None, subhi=None):
    d = Domain()
    d.dimension = dimension
    for k in range(3):
        d.boxlo[k] = boxlo[k]
        d.boxhi[k] = boxhi[k]
        d.sublo[k] = boxlo[k] if sublo is None else sublo[k]
        d.subhi[k] = boxhi[k] if subhi is None else subhi[k]
        d.periodicity[k] = periodicity[k]
    d.dt = dt
    d.ntimestep = ntimestep
    return d


# couplb_fix_comm (several ranks along z)
SENDRECV_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int)


class FixComm(C.Structure):
    _fields_ = [("nprocs", C.c_int), ("rank", C.c_int), ("sendrecv", SENDRECV_FN),
                ("allreduce", ALLREDUCE_FN), ("ctx", C.c_void_p)]
