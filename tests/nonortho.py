"""A box with a general lower-triangular cell for the tests (the reference's
triclinic water case, tests/golden/wat_nonortho_rc8.npz)."""

import os

import numpy as np

from sponge_b200 import systems

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "wat_nonortho_rc8.npz")


class TriclinicSystem(systems.System):
    """A periodic box of cell {a11, a21, a22, a31, a32, a33} (`cell6`) and its
    inverse (`rcell6`); `lengths` = (a11, a22, a33), the brick the lattice
    tiles and the lengths the PME grid is sized from."""

    def cell(self):
        return np.array(self.cell6, np.float32)

    def rcell(self):
        return np.array(self.rcell6, np.float32)

    @classmethod
    def make(cls, crd, charge, lj_type, lj_A, lj_B, mass, excl_start, excl_numbers,
             excl_list, n_types, cell6, rcell6):
        s = cls(crd=np.ascontiguousarray(crd, np.float32),
                vel=np.zeros_like(crd, np.float32),
                charge=np.ascontiguousarray(charge, np.float32),
                lj_type=np.ascontiguousarray(lj_type, np.int32),
                lj_A=np.ascontiguousarray(lj_A, np.float32),
                lj_B=np.ascontiguousarray(lj_B, np.float32),
                mass=np.ascontiguousarray(mass, np.float32),
                excl_start=np.ascontiguousarray(excl_start, np.int32),
                excl_numbers=np.ascontiguousarray(excl_numbers, np.int32),
                excl_list=np.ascontiguousarray(excl_list, np.int32),
                bonds=np.zeros((0, 2), np.int32), angles=np.zeros((0, 3), np.int32),
                box=float(cell6[0]), n_types=int(n_types))
        s.cell6 = np.array(cell6, np.float32)
        s.rcell6 = np.array(rcell6, np.float32)
        s.lengths = [float(cell6[0]), float(cell6[2]), float(cell6[5])]
        return s


def load():
    """(system, fixture arrays) of the reference's triclinic water case."""
    z = np.load(FIXTURE)
    s = TriclinicSystem.make(z["crd"], z["charge"], z["lj_type"], z["lj_A"], z["lj_B"],
                             z["mass"], z["excl_start"], z["excl_numbers"], z["excl_list"],
                             int(z["n_types"]), z["cell"], z["rcell"])
    return s, z
