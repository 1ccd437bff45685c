"""`fix couplb` argument parsing (fix_couplb.cpp:71-238): values, defaults and
the reference's error messages.  Host-only: needs no GPU."""
import pytest

from couplb_b200 import abi
from couplb_b200.fix import parse_args
from couplb_b200.lib import CoupLBError


def P(cmd, dim=3):
    return parse_args(cmd.split(), dimension=dim)


def test_defaults(cuda_lib):
    c = P("f all couplb 8 32 4 0.1 1.0")
    assert (c.Nx, c.Ny, c.Nz, c.nu, c.rho) == (8, 32, 4, 0.1, 1.0)
    assert c.md_per_lb == 1 and c.xi_ibm == 1.0 and c.delta == abi.DELTA_ROMA
    assert list(c.wall) == [0] * 6 and list(c.gstyle) == [0, 0, 0]
    assert c.output_file == b"couplb_profile.dat" and c.checkpoint_prefix == b"couplb_ckpt"
    assert c.precision == abi.FP64


def test_all_keywords(cuda_lib):
    c = P("f all couplb 64 48 32 0.1 1.26 md_per_lb 10 xi_ibm 0.1 wall_y 1 1 wall_z 2 3 "
          "wall_vel 0.1 0 0 gravity v_Gx 0.0 -2e-3 kernel peskin4 vtk 5000 flow_vtk "
          "vtk_region 0 10 0 5 0 3 vtk_solid x v checkpoint 10000 ckpt/fluid check_every 1000 "
          "output 100 prof.dat restart old precision fp32")
    assert c.md_per_lb == 10 and c.xi_ibm == 0.1
    assert list(c.wall) == [0, 0, 1, 1, 2, 3]
    assert list(c.wall_vel) == [0.1, 0, 0]
    assert list(c.gstyle) == [abi.G_EQUAL, abi.G_CONSTANT, abi.G_CONSTANT]
    assert c.gvar[0].value == b"Gx" and c.gconst[2] == -2e-3
    assert c.delta == abi.DELTA_PESKIN4
    assert c.vtk_every == 5000 and c.vtk_prefix == b"flow_vtk"
    assert c.has_vtk_region == 1 and c.vtk_region_n == 6 and list(c.vtk_rhi) == [10, 5, 3]
    assert c.vtk_solid_nattr == 2
    assert c.checkpoint_every == 10000 and c.checkpoint_prefix == b"ckpt/fluid"
    assert c.check_every == 1000 and c.output_every == 100 and c.output_file == b"prof.dat"
    assert c.do_restart == 1 and c.restart_prefix == b"old"
    assert c.precision == abi.FP32_SHIFTED


@pytest.mark.parametrize("cmd,dim,msg", [
    ("f all couplb 8 32 1 0.1", 2, "Illegal fix couplb command: need Nx Ny Nz nu rho"),
    ("f all couplb 0 32 1 0.1 1.0", 2, "fix couplb: Nx, Ny, and Nz must be positive"),
    ("f all couplb 8 32 1 -0.1 1.0", 2, "fix couplb: viscosity must be positive and finite"),
    ("f all couplb 8 32 1 0.1 0", 2, "fix couplb: density must be positive and finite"),
    ("f all couplb 8 32 1 0.1 1.0 bogus 1", 2, "Unknown fix couplb keyword: bogus"),
    ("f all couplb 8 32 1 0.1 1.0 md_per_lb 0", 2, "fix couplb: md_per_lb must be >= 1"),
    ("f all couplb 8 32 1 0.1 1.0 md_per_lb", 2, "fix couplb md_per_lb: need 1 value"),
    ("f all couplb 8 32 1 0.1 1.0 xi_ibm 5.0", 2, "fix couplb: xi_ibm must satisfy 0 < xi_ibm <= 1"),
    ("f all couplb 8 32 1 0.1 1.0 gravity 1 2", 2, "fix couplb gravity: need 3 values"),
    ("f all couplb 8 32 1 0.1 1.0 wall_y 1 5", 2, "fix couplb: wall_y types must be in [0,4]"),
    ("f all couplb 8 32 1 0.1 1.0 wall_x 1", 2, "fix couplb wall_x: need 2 values"),
    ("f all couplb 8 32 1 0.1 1.0 output -1 a", 2, "fix couplb: output frequency cannot be negative"),
    ("f all couplb 8 32 1 0.1 1.0 check_every -2", 2, "fix couplb: check_every cannot be negative"),
    ("f all couplb 8 32 1 0.1 1.0 kernel cubic", 2, "fix couplb kernel: use roma or peskin4"),
    ("f all couplb 8 32 1 0.1 1.0 vtk_region 0 1 2", 2,
     "fix couplb vtk_region: need 4 values (2D: xlo xhi ylo yhi) or 6 values (3D: xlo xhi ylo yhi zlo zhi)"),
    ("f all couplb 8 32 1 0.1 1.0 vtk_solid", 2, "fix couplb vtk_solid: need at least one attribute"),
    ("f all couplb 8 32 1 0.1 1.0 vtk_solid x vtk_solid v", 2,
     "fix couplb vtk_solid: keyword specified more than once"),
    ("f all couplb 8 32 1 0.1 1.0 checkpoint -5 p", 2, "fix couplb: checkpoint frequency cannot be negative"),
    ("f all couplb 8 32 1 0.1 1.0 restart", 2, "fix couplb restart: need prefix"),
    ("f all couplb 8 32 2 0.1 1.0", 2, "fix couplb: Nz must be 1 for 2D"),
    ("f all couplb 8 32 2 0.1 1.0 precision fp8", 3, "fix couplb precision: use fp64, fp32 or fp16"),
])
def test_errors(cuda_lib, cmd, dim, msg):
    with pytest.raises(CoupLBError) as e:
        P(cmd, dim)
    assert e.value.msg == msg
    assert e.value.code == abi.ERR_PARSE


def test_swimmer_deck_is_rejected_like_the_reference(cuda_lib):
    """examples/swimming/in.swim:49 passes `xi_ibm 5.0`, which the reference
    parser rejects (fix_couplb.cpp:119-120)."""
    with pytest.raises(CoupLBError):
        P("lb all couplb 64 64 1 0.1 1.0 xi_ibm 5.0", 2)


def test_ibm_method_keywords(cuda_lib):
    c = P("f all couplb 8 8 8 0.1 1.0")
    assert c.ibm_method == abi.IBM_SINGLE and c.ibm_passes == 5 and c.slip_tol == 0.0
    c = P("f all couplb 8 8 8 0.1 1.0 ibm_method learned ibm_passes 4 slip_tol 2e-4 mlp_model net.bin")
    assert c.ibm_method == abi.IBM_LEARNED and c.ibm_passes == 4 and c.slip_tol == 2e-4
    assert c.mlp_model == b"net.bin"
    assert P("f all couplb 8 8 8 0.1 1.0 ibm_method iterative").ibm_method == abi.IBM_ITERATIVE


@pytest.mark.parametrize("tail,msg", [
    ("ibm_method fancy", "ibm_method: use single, iterative or learned"),
    ("ibm_passes 0", "ibm_passes must be 1..64"),
    ("slip_tol -1", "slip_tol must be >= 0"),
    ("ibm_method", "ibm_method: need 1 value"),
])
def test_ibm_method_errors(cuda_lib, tail, msg):
    with pytest.raises(CoupLBError) as e:
        P("f all couplb 8 8 8 0.1 1.0 " + tail)
    assert msg in e.value.msg


def test_vtk_solid_attribute_names(cuda_lib):
    c = P("f all couplb 8 8 8 0.1 1.0 vtk 10 out vtk_solid x y z vx id md_per_lb 2")
    assert c.vtk_solid_nattr == 5 and c.md_per_lb == 2
    assert [c.vtk_solid_attr[i].value for i in range(5)] == [b"x", b"y", b"z", b"vx", b"id"]
    with pytest.raises(CoupLBError) as e:
        P("f all couplb 8 8 8 0.1 1.0 vtk_solid " + " ".join(["x"] * 40))
    assert "too many attributes" in e.value.msg


@pytest.mark.parametrize("axis,dim", [(0, 3), (1, 3), (2, 3), (0, 2)])
def test_init_refuses_a_sub_box_smaller_than_the_box(cuda_lib, axis, dim):
    """Under a domain decomposition each rank's sub-box is part of the box
    (fix_couplb.cpp:494-500).  One lattice per fix cannot exchange ghost
    layers with other ranks, so init refuses such a sub-box instead of
    simulating a periodic slab; no device work happens before the check."""
    import ctypes as C
    from couplb_b200.fix import FixCoupLB
    nz = 8 if dim == 3 else 1
    fx = FixCoupLB(f"f all couplb 16 8 {nz} 0.1 1.0".split(), dimension=dim)
    hi = (16.0, 8.0, float(nz))
    d = abi.make_domain(dim, (0.0, 0.0, 0.0), hi, 0.1)
    d.subhi[axis] = hi[axis] / 2
    rc = fx.L.couplb_fix_init(fx.h, C.byref(d))
    assert rc == abi.ERR_UNSUPPORTED
    msg = fx.L.couplb_fix_last_error(fx.h).decode()
    assert "one rank" in msg and "xyz"[axis] in msg
    fx.close()


def _comm_fix(words, rank=0, nprocs=2):
    from couplb_b200.fix import FixCoupLB
    fx = FixCoupLB(words.split(), dimension=3)
    fx.set_comm(nprocs, rank, lambda *a: None, lambda a, op: None)
    return fx


@pytest.mark.parametrize("axis,why", [(0, "split along z only"), (1, "split along z only")])
def test_comm_refuses_x_and_y_splits(cuda_lib, axis, why):
    """With a communicator the sub-boxes may split z only."""
    import ctypes as C
    fx = _comm_fix("f all couplb 16 8 8 0.1 1.0")
    d = abi.make_domain(3, (0.0, 0.0, 0.0), (16.0, 8.0, 8.0), 0.1)
    d.subhi[axis] /= 2
    assert fx.L.couplb_fix_init(fx.h, C.byref(d)) == abi.ERR_UNSUPPORTED
    assert why in fx.L.couplb_fix_last_error(fx.h).decode()
    fx.close()


def test_comm_slab_rules(cuda_lib):
    """A z slab has at least 2 planes; VTK output and the correction methods
    are refused with several ranks; a communicator of several ranks needs
    both callbacks."""
    import ctypes as C
    fx = _comm_fix("f all couplb 8 8 8 0.1 1.0")
    d = abi.make_domain(3, (0.0, 0.0, 0.0), (8.0, 8.0, 8.0), 0.1)
    d.subhi[2] = 1.0
    assert fx.L.couplb_fix_init(fx.h, C.byref(d)) == abi.ERR_UNSUPPORTED
    assert "at least 2 planes" in fx.L.couplb_fix_last_error(fx.h).decode()
    fx.close()
    fx = _comm_fix("f all couplb 8 8 8 0.1 1.0 vtk 10 out")
    d.subhi[2] = 4.0
    assert fx.L.couplb_fix_init(fx.h, C.byref(d)) == abi.ERR_UNSUPPORTED
    assert "vtk" in fx.L.couplb_fix_last_error(fx.h).decode()
    fx.close()
    fx = _comm_fix("f all couplb 8 8 8 0.1 1.0 ibm_method iterative")
    assert fx.L.couplb_fix_init(fx.h, C.byref(d)) == abi.ERR_UNSUPPORTED
    assert "iterative with several ranks" in fx.L.couplb_fix_last_error(fx.h).decode()
    fx.close()
    from couplb_b200.fix import FixCoupLB
    fx = FixCoupLB("f all couplb 8 8 8 0.1 1.0".split(), dimension=3)
    comm = abi.FixComm(2, 0, abi.SENDRECV_FN(), abi.ALLREDUCE_FN(), None)
    assert fx.L.couplb_fix_set_comm(fx.h, C.byref(comm)) == abi.ERR_ARG
    comm = abi.FixComm(2, 2, abi.SENDRECV_FN(), abi.ALLREDUCE_FN(), None)
    assert fx.L.couplb_fix_set_comm(fx.h, C.byref(comm)) == abi.ERR_ARG
    fx.close()


def test_ibm_window_keyword(cuda_lib):
    assert P("f all couplb 8 8 8 0.1 1.0").ibm_window == 0
    assert P("f all couplb 8 8 8 0.1 1.0 ibm_window wrap").ibm_window == 1
    assert P("f all couplb 8 8 8 0.1 1.0 ibm_window clip").ibm_window == 0
    with pytest.raises(CoupLBError) as e:
        P("f all couplb 8 8 8 0.1 1.0 ibm_window torus")
    assert e.value.msg == "fix couplb ibm_window: use clip or wrap"
