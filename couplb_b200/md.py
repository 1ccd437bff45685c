"""Minimal MD driver for running `fix couplb` without LAMMPS.

It reproduces the call order of LAMMPS' Verlet integrator with `fix nve` for
the parts the fix sees: at setup the forces are cleared and fix setup() runs;
every step increments the timestep, half-kicks and drifts the integrated atoms,
clears forces (plus optional constant external forces), calls post_force(),
half-kicks again and calls end_of_step().  Any object with setup /
post_force / end_of_step taking an Atoms struct works (the GPU FixCoupLB or
the CPU oracle).
"""
import ctypes as C

import numpy as np

from . import abi


class Atoms:
    """Per-atom arrays in LAMMPS layout ((n,3) x, v, f; masses; group mask)."""

    def __init__(self, x, v=None, mass=None, mask=None, groupbit=1, integrate=True, tag=None,
                 type_=None):
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        n = self.x.shape[0]
        self.v = np.zeros((n, 3)) if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self.f = np.zeros((n, 3))
        self.rmass = np.ones(n) if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        self.mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
        self.groupbit = groupbit
        self.integrate = integrate
        self.fext = None   # constant external force (fix addforce), (n,3) or None
        self.tag = None if tag is None else np.ascontiguousarray(tag, dtype=np.int64)
        self.type = None if type_ is None else np.ascontiguousarray(type_, dtype=np.int32)

    @property
    def n(self):
        return self.x.shape[0]

    def struct(self):
        if self.n == 0:
            return abi.make_atoms(None, None, None)
        at = abi.make_atoms(self.x, self.v, self.f, mask=self.mask, groupbit=self.groupbit,
                            rmass=self.rmass, type_=self.type)
        if self.tag is not None:
            at.tag = self.tag.ctypes.data_as(C.POINTER(C.c_longlong))
        return at


def empty_atoms():
    return Atoms(np.zeros((0, 3)))


def run(fix, atoms, nsteps, dt, start_step=0, setup=True, box=None, on_step=None):
    """Advance `nsteps` MD steps; returns the final timestep."""
    at = atoms.struct()
    if setup:
        atoms.f[:] = 0.0 if atoms.fext is None else atoms.fext
        fix.setup(at, start_step)
    step = start_step
    minv = None if atoms.n == 0 else (1.0 / atoms.rmass)[:, None]
    for _ in range(nsteps):
        step += 1
        if atoms.n and atoms.integrate:
            atoms.v += 0.5 * dt * atoms.f * minv
            atoms.x += dt * atoms.v
            if box is not None:
                lo, hi = np.asarray(box[0]), np.asarray(box[1])
                atoms.x[:] = lo + np.mod(atoms.x - lo, hi - lo)
        atoms.f[:] = 0.0 if atoms.fext is None else atoms.fext
        fix.post_force(at, step)
        if atoms.n and atoms.integrate:
            atoms.v += 0.5 * dt * atoms.f * minv
        fix.end_of_step(step)
        if hasattr(fix, "write_solid"):
            fix.write_solid(at, step)
        if on_step is not None:
            on_step(step)
    return step
