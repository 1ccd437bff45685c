"""`vtk N prefix`, `vtk_region` and `vtk_solid` output of the fix
(IO::write_vtk / write_solid_vtk / write_pvd, couplb_io.h:42-614): the files
are read back with a small parser of VTK XML appended binary data and compared
with the fields and atoms they were written from."""
import re

import numpy as np
import pytest

from couplb_b200 import md
from couplb_b200.fix import FixCoupLB

pytestmark = pytest.mark.gpu


def read_vtk(path):
    """{name: (ncomp, array)} plus the XML header of a VTK file with raw
    appended data and UInt64 length headers."""
    raw = open(path, "rb").read()
    start = raw.index(b"<AppendedData encoding=\"raw\">")
    head = raw[:start].decode()
    blob = raw[raw.index(b"_", start) + 1:]
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="(\d)")? '
                         r'format="appended" offset="(\d+)"/>', head):
        typ, name, nc, off = m.group(1), m.group(2) or "Points", int(m.group(3) or 1), int(m.group(4))
        nbytes = int(np.frombuffer(blob[off:off + 8], dtype="<u8")[0])
        dt = "<f8" if typ == "Float64" else "<i4"
        out[name] = (nc, np.frombuffer(blob[off + 8:off + 8 + nbytes], dtype=dt))
    return head, out


def run_fix(tmp_path, extra, natoms=6, steps=10):
    prefix = str(tmp_path / "flow")
    cmd = ("f all couplb 12 10 8 0.1 1.0 wall_y 1 1 gravity 1e-4 0 0 md_per_lb 2 "
           f"vtk 5 {prefix} " + extra).split()
    fix = FixCoupLB(cmd, dimension=3)
    fix.init((0, 0, 0), (12, 10, 8), 0.5)
    rng = np.random.default_rng(4)
    x = np.array([2, 2, 2]) + rng.random((natoms, 3)) * np.array([8, 6, 4])
    at = md.Atoms(x, 0.01 * rng.standard_normal((natoms, 3)), mass=rng.uniform(1, 2, natoms),
                  tag=np.arange(1, natoms + 1), type_=np.ones(natoms, dtype=np.int32))
    md.run(fix, at, steps, 0.5)
    return fix, at, prefix


def test_field_output_matches_the_fields(cuda_lib, tmp_path):
    fix, at, prefix = run_fix(tmp_path, "")
    sc = fix.scales()
    head, arr = read_vtk(prefix + "_000010.vti")
    assert 'WholeExtent="0 12 0 10 0 8"' in head
    rho, ux, uy, uz = fix.lattice.get_macroscopic()
    fx, fy, fz = fix.lattice.get_force_field()
    inner = (slice(1, -1),) * 3
    flat = lambda a: a[inner].reshape(-1)   # x fastest, like the cells
    np.testing.assert_allclose(arr["rho"][1], flat(rho) * 1.0, rtol=1e-15, atol=0)
    vel = arr["velocity_phys"][1].reshape(-1, 3)
    np.testing.assert_allclose(vel[:, 0], flat(ux) * sc["vel_scale"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(vel[:, 2], flat(uz) * sc["vel_scale"], rtol=1e-15, atol=0)
    force = arr["force_phys"][1].reshape(-1, 3)
    np.testing.assert_allclose(force[:, 1], flat(fy) * sc["force_scale"], rtol=1e-15, atol=0)
    assert not arr["type"][1].any()
    pvd = open(prefix + ".pvd").read()
    assert 'file="flow_000005.vti"' in pvd and 'file="flow_000010.vti"' in pvd
    assert 'timestep="5.00000000e+00"' in pvd      # step 10 x dt 0.5
    fix.close()


def test_region_and_solid_output(cuda_lib, tmp_path):
    fix, at, prefix = run_fix(tmp_path, "vtk_region 2 9 1 8 2 6 vtk_solid id type mass x y z vx vy vz fx fz")
    head, arr = read_vtk(prefix + "_000005.vti")
    assert 'WholeExtent="0 7 0 7 0 4"' in head
    assert 'Origin="2.00000000e+00 1.00000000e+00 2.00000000e+00"' in head
    assert arr["rho"][1].size == 7 * 7 * 4
    head, arr = read_vtk(prefix + "_solid_000010.vtp")
    inside = np.all((at.x >= [2, 1, 2]) & (at.x < [9, 8, 6]), axis=1)
    pts = arr["Points"][1].reshape(-1, 3)
    np.testing.assert_array_equal(pts, at.x[inside])
    np.testing.assert_array_equal(arr["id"][1], at.tag[inside].astype(float))
    np.testing.assert_array_equal(arr["mass"][1], at.rmass[inside])
    np.testing.assert_array_equal(arr["velocity"][1].reshape(-1, 3), at.v[inside])
    # fx and fz without fy: two scalars, not a vector group
    np.testing.assert_array_equal(arr["fx"][1], at.f[inside][:, 0])
    np.testing.assert_array_equal(arr["fz"][1], at.f[inside][:, 2])
    assert "force" not in arr
    np.testing.assert_array_equal(arr["connectivity"][1], np.arange(inside.sum()))
    assert 'file="flow_solid_000010.vtp"' in open(prefix + "_solid.pvd").read()
    fix.close()


def test_unknown_and_unavailable_attributes(cuda_lib, tmp_path):
    from couplb_b200.lib import CoupLBError
    with pytest.raises(CoupLBError) as e:
        run_fix(tmp_path, "vtk_solid x y z charge")
    assert "unknown attribute 'charge'" in e.value.msg
    with pytest.raises(CoupLBError) as e:
        run_fix(tmp_path, "vtk_solid x diameter")
    assert "'diameter' is not available" in e.value.msg
