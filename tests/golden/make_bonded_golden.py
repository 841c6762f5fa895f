"""Golden vectors for the harmonic bond and angle modules from the reference.

Runs the reference's own BOND and ANGLE (bond/bond.cpp, angle/angle.cpp,
compiled from its sources into oracle/_ref by `make -C oracle ref`, CPU
build) on three cases and stores inputs and outputs:

  * bonded_amber_alanine_dipeptide.npz: the bonds (solute and the waters'
    three rigid-geometry bonds) and angles of the reference's Amber
    comparison case, read from tests/golden/amber_alanine_dipeptide_tip4pew_iter1.npz
    (the frame perturbed by 0.02 A, so every term is off its minimum);
  * bonded_wat_nonortho.npz: the reference's triclinic water case, its
    bond_in_file (WAT_bond.txt) read by the reference's own loader, in its
    skewed cell (tests/golden/wat_nonortho_rc8.npz);
  * bonded_water_box.npz: 300 waters with O-H bonds and H-O-H angles, every
    atom displaced by up to 0.1 A (seeded).

Needs the reference checkout, named by SPONGE_REFERENCE:

    SPONGE_REFERENCE=<reference checkout> python tests/golden/make_bonded_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def save(name, crd, cell, bonds, angles, ref):
    b, a = ref.bonded(crd, cell, bonds, angles)
    out = os.path.join(HERE, name)
    np.savez_compressed(
        out, crd=np.asarray(crd, np.float32), cell=np.asarray(cell, np.float32),
        bond_a=np.asarray(bonds[0], np.int32), bond_b=np.asarray(bonds[1], np.int32),
        bond_k=np.asarray(bonds[2], np.float32), bond_r0=np.asarray(bonds[3], np.float32),
        angle_a=np.asarray(angles[0], np.int32), angle_b=np.asarray(angles[1], np.int32),
        angle_c=np.asarray(angles[2], np.int32), angle_k=np.asarray(angles[3], np.float32),
        angle_theta0=np.asarray(angles[4], np.float32),
        bond_frc=b["frc"], bond_atom_energy=b["atom_energy"], bond_virial=b["virial"],
        bond_energy=np.float64(b["energy"]), angle_frc=a["frc"],
        angle_atom_energy=a["atom_energy"], angle_virial=a["virial"],
        angle_energy=np.float64(a["energy"]))
    print(out, len(bonds[0]), "bonds", len(angles[0]), "angles", b["energy"], a["energy"])


def main():
    root = os.environ.get("SPONGE_REFERENCE", "")
    if not root:
        raise SystemExit("set SPONGE_REFERENCE to the reference checkout's root")
    from oracle.oracle import ReferenceCPU, build_oracle
    from sponge_b200 import systems
    build_oracle(with_reference=True)
    ref = ReferenceCPU(exact=False)

    z = np.load(os.path.join(HERE, "amber_alanine_dipeptide_tip4pew_iter1.npz"))
    # parm7 tables: atom fields are 3 x the atom index, types count from 1
    bt, at = np.abs(z["bonds"]), np.abs(z["angles"])
    tb, ta = bt[:, 2] - 1, at[:, 3] - 1
    bonds = (bt[:, 0] // 3, bt[:, 1] // 3, z["bond_k"][tb].astype(np.float32),
             z["bond_r0"][tb].astype(np.float32))
    angles = (at[:, 0] // 3, at[:, 1] // 3, at[:, 2] // 3,
              z["angle_k"][ta].astype(np.float32), z["angle_t0"][ta].astype(np.float32))
    L = np.asarray(z["box"], np.float32)
    save("bonded_amber_alanine_dipeptide.npz", z["crd"],
         np.array([L[0], 0, L[1], 0, 0, L[2]], np.float32), bonds, angles, ref)

    w = np.load(os.path.join(HERE, "wat_nonortho_rc8.npz"))
    case = os.path.join(root, "benchmarks", "performance", "nonortho", "statics",
                        "WAT_nonortho")
    ref.native_load({"bond_in_file": os.path.join(case, "WAT_bond.txt")})
    bonds = (ref.native_get("bond_a", np.int32), ref.native_get("bond_b", np.int32),
             ref.native_get("bond_k"), ref.native_get("bond_r0"))
    empty = (np.zeros(0, np.int32),) * 3 + (np.zeros(0, np.float32),) * 2
    save("bonded_wat_nonortho.npz", w["crd"], w["cell"], bonds, empty, ref)

    s = systems.water_box(300, seed=4)
    rng = np.random.default_rng(12)
    crd = (s.crd + rng.uniform(-0.1, 0.1, s.crd.shape)).astype(np.float32)
    nb, na = len(s.bonds), len(s.angles)
    bonds = (s.bonds[:, 0], s.bonds[:, 1], np.full(nb, systems.BOND_K, np.float32),
             np.full(nb, systems.BOND_R0, np.float32))
    angles = (s.angles[:, 0], s.angles[:, 1], s.angles[:, 2],
              np.full(na, systems.ANGLE_K, np.float32),
              np.full(na, systems.ANGLE_T0, np.float32))
    save("bonded_water_box.npz", crd, s.cell(), bonds, angles, ref)


if __name__ == "__main__":
    main()
