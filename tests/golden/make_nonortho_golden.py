"""Known answer for a skewed cell: the reference's own triclinic water case.

Reads benchmarks/performance/nonortho/statics/WAT_nonortho of the reference
checkout (1,081 TIP4P waters, 4,324 sites, a = 36.77, b = 37.77, c = 33.50 A,
alpha = beta = gamma = 60 degrees) through the reference's own native-file
loaders, turns the box into its lower-triangular cell as MD_core/pbc.hpp:61-81
does, and runs the reference's own CPU build of the hot path on it at the
case's cutoff (8 A, skin 2 A): the neighbor pair set (the build without fast
math, so the criterion is evaluated as written; stored as its size, the
SHA-256 of the sorted (i < j) pairs as int32 and the row sizes), and the LJ +
direct Coulomb, PME reciprocal and excluded-correction forces and energies.
The extra points (EPW) are charged sites at their positions in the file.

On this cell the reference's neighbour-grid table does not reach every pair
its own criterion accepts: the pairs that the all-pairs restatement of the
criterion (oracle/snb_oracle.c) lists and the reference does not are stored
too (pairs_missed_by_reference), so a test can show that the reference's set
is the complete set less exactly those.

Writes tests/golden/wat_nonortho_rc8.npz; the tests read only that file.
Needs the reference checkout, named by SPONGE_REFERENCE:

    SPONGE_REFERENCE=<reference checkout> python tests/golden/make_nonortho_golden.py
"""

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CUTOFF, SKIN = 8.0, 2.0
DEG_TO_RAD = np.float32(0.017453292519943295)  # common.h CONSTANT_DEG_TO_RAD


def read_coordinates(path):
    """Native coordinate file: "N time", N lines "x y z", then
    "a b c alpha beta gamma"."""
    with open(path) as f:
        n = int(f.readline().split()[0])
        crd = np.array([[float(v) for v in f.readline().split()[:3]] for _ in range(n)],
                       np.float32)
        box = np.array([float(v) for v in f.read().split()[:6]], np.float32)
    return crd, box


def lower_cell(box):
    """{a11, a21, a22, a31, a32, a33} of lengths a, b, c and angles
    alpha, beta, gamma (degrees), in float32 as pbc.hpp:61-81 forms it, with
    the near-orthogonal entries set to zero (Normalize_Near_Orthogonal_Cell)."""
    a, b, c = (np.float32(v) for v in box[:3])
    al, be, ga = (np.float32(v) * DEG_TO_RAD for v in box[3:6])
    ca, cb, cg = np.cos(al), np.cos(be), np.cos(ga)
    sg = np.sin(ga)
    one = np.float32(1.0)
    za = np.sqrt(one - ca * ca - cb * cb - cg * cg + np.float32(2.0) * ca * cb * cg)
    cell = np.array([a, b * cg, b * sg, c * cb, c / sg * (ca - cb * cg), c / sg * za],
                    np.float32)
    for k in (1, 3, 4):
        if abs(cell[k]) < np.float32(1e-3):
            cell[k] = np.float32(0.0)
    return cell


def lower_rcell(cell):
    """Invert_Lower_Triangular_Cell (utils/boundary.h:61-72) in float32."""
    a11, a21, a22, a31, a32, a33 = (np.float32(v) for v in cell)
    one = np.float32(1.0)
    return np.array([one / a11, -a21 / (a11 * a22), one / a22,
                     (a21 * a32 - a22 * a31) / (a11 * a22 * a33), -a32 / (a22 * a33),
                     one / a33], np.float32)


def main():
    root = os.environ.get("SPONGE_REFERENCE", "")
    if not root:
        raise SystemExit("set SPONGE_REFERENCE to the reference checkout's root")
    case = os.path.join(root, "benchmarks", "performance", "nonortho", "statics",
                        "WAT_nonortho")
    from oracle.oracle import ReferenceCPU, build_oracle
    from tests.nonortho import TriclinicSystem
    build_oracle(with_reference=True)
    loader = ReferenceCPU(exact=False)
    loader.native_load({"mass_in_file": os.path.join(case, "WAT_mass.txt"),
                        "charge_in_file": os.path.join(case, "WAT_charge.txt"),
                        "exclude_in_file": os.path.join(case, "WAT_exclude.txt"),
                        "LJ_in_file": os.path.join(case, "WAT_LJ.txt")})
    crd, box = read_coordinates(os.path.join(case, "WAT_coordinate.txt"))
    n = len(crd)
    charge = loader.native_get("charge")
    mass = loader.native_get("mass")
    lj_A, lj_B = loader.native_get("lj_A"), loader.native_get("lj_B")
    lj_type = loader.native_get("lj_type", np.int32)
    n_types = int(loader.lib.ref_native_get(b"lj_type_numbers", None))
    excl_numbers = loader.native_get("excl_numbers", np.int32)
    excl_list = loader.native_get("excl_list", np.int32)
    excl_start = np.zeros(n, np.int32)
    excl_start[1:] = np.cumsum(excl_numbers)[:-1]
    assert len(charge) == n and len(lj_type) == n
    cell = lower_cell(box)
    s = TriclinicSystem.make(crd, charge, lj_type, lj_A, lj_B, mass, excl_start,
                             excl_numbers, excl_list, n_types, cell, lower_rcell(cell))

    exact = ReferenceCPU(exact=True)
    exact.init(s, CUTOFF, SKIN)
    counts, serial, ov = exact.nl_update()
    assert not ov.any()
    i = np.repeat(np.arange(n), counts)
    pairs = np.stack([np.minimum(i, serial), np.maximum(i, serial)], 1).astype(np.int64)
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]

    # the pairs the reference's cell grid leaves out: its criterion holds for
    # them (the all-pairs restatement of it lists them), but no cell of its
    # neighbour-grid table reaches them
    from oracle.oracle import Oracle
    rs, cols = Oracle().nl_pairs_system(s, CUTOFF, SKIN)
    full = np.stack([np.repeat(np.arange(n), np.diff(rs)), cols.astype(np.int64)], 1)
    ref_set = set(map(tuple, pairs.tolist()))
    missed = np.array([p for p in map(tuple, full.tolist()) if p not in ref_set],
                      np.int32).reshape(-1, 2)
    assert len(full) == len(pairs) + len(missed)

    ref = ReferenceCPU(exact=False)
    beta = ref.init(s, CUTOFF, SKIN)
    ref.nl_update()
    lj = ref.lj_direct()
    pme = ref.pme_reciprocal()
    ex = ref.pme_excluded()
    out = os.path.join(HERE, "wat_nonortho_rc8.npz")
    np.savez_compressed(
        out, crd=crd, box=box, cell=cell, rcell=s.rcell(), charge=charge, mass=mass,
        lj_A=lj_A, lj_B=lj_B, lj_type=lj_type, n_types=np.int32(n_types),
        excl_start=excl_start, excl_numbers=excl_numbers, excl_list=excl_list,
        cutoff=np.float32(CUTOFF), skin=np.float32(SKIN), beta=np.float32(beta),
        grid=np.array(ref.grid, np.int32), pair_numbers=np.int64(len(pairs)),
        pairs_sha256=np.array(hashlib.sha256(pairs.astype(np.int32).tobytes()).hexdigest()),
        pair_row_counts=np.bincount(pairs[:, 0], minlength=n).astype(np.int32),
        pairs_missed_by_reference=missed,
        lj_frc=lj["frc"], lj_energy=lj["lj_energy"], coulomb_energy=lj["coulomb_energy"],
        lj_virial=lj["virial"], pme_frc=pme["frc"], pme_e_recip=np.float32(pme["e_recip"]),
        pme_e_self=np.float32(pme["e_self"]), pme_virial=pme["virial"],
        excl_frc=ex["frc"], excl_energy=ex["atom_energy"])
    print(out, n, "atoms,", len(pairs), "pairs, sha256",
          hashlib.sha256(pairs.astype(np.int32).tobytes()).hexdigest()[:16],
          "grid", ref.grid, "beta", beta, "missed by its grid", len(missed))


if __name__ == "__main__":
    main()
