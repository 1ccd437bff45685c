"""Slab decomposition along z on the GPU: a lattice run as 2 or 3 z slabs
(halo faces packed and attached after every LB step, couplb_halo_pack /
couplb_halo_attach) steps exactly like the whole lattice -- the same
arithmetic per node, only the source of the crossing populations differs --
so populations and moments agree bit for bit, FP64 and FP32-shifted, with a
periodic z or walls on the z faces, moving walls and a body force."""
import numpy as np
import pytest

import cases
from couplb_b200.lattice import Lattice
from couplb_b200.lib import CoupLBError
from couplb_b200.slabs import SlabLattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("nslab", [2, 3])
@pytest.mark.parametrize("wall", [(0, 0, 1, 1, 0, 0), (0, 0, 1, 2, 3, 1), (0,) * 6])
def test_slabs_step_like_the_whole_lattice(cuda_lib, prec, nslab, wall):
    n = (24, 14, 19)
    f0 = cases.initial_populations(3, n, 17)
    kw = dict(tau=0.7, wall=wall, wall_vel=(0.02, 0.0, 0.01), body_force=True, precision=prec)
    L = Lattice(3, *n, **kw)
    L.set_populations(f0)
    S = SlabLattice(*n, nslab, **kw)
    S.set_populations(f0)
    g = (1e-5, -2e-6, 3e-6)
    for _ in range(12):
        L.lbm_step(g)
        S.lbm_step(g)
    np.testing.assert_array_equal(S.get_populations(), L.get_populations()[:, 1:-1, 1:-1, 1:-1])
    L.macroscopic()
    want = [a[1:-1, 1:-1, 1:-1] for a in L.get_macroscopic()]
    for got, ref in zip(S.get_macroscopic(), want):
        np.testing.assert_array_equal(got, ref)
    d = L.diagnostics()
    umax, mass, mom = S.diagnostics()
    assert umax == d.umax
    assert abs(mass - d.mass) <= 1e-12 * d.mass
    L.close()
    S.close()


def test_halo_face_rules(cuda_lib):
    L = Lattice(3, 8, 6, 5, tau=0.8, wall=(0, 0, 0, 0, 1, 0))
    import torch
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(CoupLBError):     # the z-low face is a wall
        L._ck(L.L.couplb_halo_attach(L.h, 0, dummy.data_ptr()))
    buf = torch.zeros(int(L.L.couplb_halo_bytes(L.h)), dtype=torch.uint8, device="cuda")
    assert buf.numel() == 5 * 8 * 6 * 8
    with pytest.raises(CoupLBError):     # post-stream state: nothing to pack yet
        L._ck(L.L.couplb_halo_pack(L.h, 1, buf.data_ptr()))
    L._ck(L.L.couplb_halo_attach(L.h, 1, buf.data_ptr()))
    L.set_ibm_params(delta="peskin4")
    x = np.array([[4.0, 3.0, 2.5]])
    with pytest.raises(CoupLBError):     # IBM is not decomposed
        L.ibm_substep(x, np.zeros_like(x), np.ones(1), np.zeros_like(x))
    L.close()
