"""Known-answer fixture from the reference's Amber comparison case
(benchmarks/comparison/reference/amber: alanine dipeptide in 790 TIP4P-Ew
waters, 2,398 sites, a 30.10 x 30.51 x 42.00 A box; sander forces and energy
of the minimised frame, cutoff 8 A).

Reads the case's system.parm7 and system_minimized.rst7 with the parser
below and stores what this project's path needs (coordinates, charges, LJ
tables in SPONGE's A' = 12 A, B' = 6 B triangular form, the exclusion CSR)
plus the bonded term lists and parameters the test evaluates in FP64, the
residue ranges, and Amber's forces (iter0.npy) and potential energy
(reference.json), for the case's three frames: the minimised one and two
made from it by the reference's own rigid-water perturbation (0.02 and
0.05 A).  Needs the reference checkout, named by SPONGE_REFERENCE:

    SPONGE_REFERENCE=<reference checkout> python tests/golden/make_amber_golden.py
"""

import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout's root, from the environment (required to regenerate)
REF_ROOT = os.environ.get("SPONGE_REFERENCE", "")
CASE = os.path.join(REF_ROOT, "benchmarks", "comparison", "reference", "amber")
NAME = "alanine_dipeptide_tip4pew"


def read_parm7(path):
    """{FLAG: list of values} of an Amber prmtop, by its %FORMAT widths."""
    out, flag, fmt = {}, None, None
    for line in open(path):
        if line.startswith("%FLAG"):
            flag = line.split()[1]
            out[flag] = []
            continue
        if line.startswith("%FORMAT"):
            m = re.match(r"%FORMAT\((\d+)([aIE])(\d+)", line)
            fmt = (int(m.group(1)), m.group(2), int(m.group(3)))
            continue
        if line.startswith("%") or flag is None:
            continue
        count, kind, width = fmt
        body = line.rstrip("\n")
        for k in range(0, len(body), width):
            tok = body[k:k + width]
            if not tok.strip():
                continue
            out[flag].append(tok.strip() if kind == "a" else
                             int(tok) if kind == "I" else float(tok))
    return out


def read_rst7(path):
    lines = open(path).read().split("\n")
    n = int(lines[1].split()[0])
    vals = []
    for ln in lines[2:]:
        for k in range(0, len(ln), 12):
            tok = ln[k:k + 12]
            if tok.strip():
                vals.append(float(tok))
    crd = np.array(vals[:3 * n]).reshape(n, 3)
    box = np.array(vals[-6:-3])
    return crd, box


def frame(iteration, perturbation):
    """Coordinates of one of the case's frames: the minimised one, perturbed
    by the reference's own rigid-water perturbation (seed 20260217 +
    2000 * iteration, as its comparison test calls it) for iterations > 0."""
    import pathlib
    import shutil
    import sys
    import tempfile
    src = os.path.join(CASE, "statics", NAME, "system_minimized.rst7")
    if perturbation == 0.0:
        return read_rst7(src)
    sys.path.insert(0, REF_ROOT)
    from benchmarks.comparison.tests.amber.tests.utils import (
        perturb_rst7_with_rigid_water_inplace)
    with tempfile.TemporaryDirectory() as d:
        dst = os.path.join(d, "system.rst7")
        shutil.copy(src, dst)
        perturb_rst7_with_rigid_water_inplace(
            pathlib.Path(dst), pathlib.Path(os.path.join(CASE, "statics", NAME, "system.parm7")),
            perturbation=perturbation, seed=20260217 + 2000 * iteration)
        return read_rst7(dst)


def main():
    for it, pert in ((0, 0.0), (1, 0.02), (2, 0.05)):
        make(it, pert)


def make(iteration, perturbation):
    p = read_parm7(os.path.join(CASE, "statics", NAME, "system.parm7"))
    crd, box = frame(iteration, perturbation)
    n = p["POINTERS"][0]
    ntypes = p["POINTERS"][1]
    assert crd.shape == (n, 3)
    typ = np.array(p["ATOM_TYPE_INDEX"], np.int32) - 1
    npi = np.array(p["NONBONDED_PARM_INDEX"], np.int64).reshape(ntypes, ntypes) - 1
    acoef = np.array(p["LENNARD_JONES_ACOEF"])
    bcoef = np.array(p["LENNARD_JONES_BCOEF"])
    # SPONGE's triangular pair tables, A' = 12 A and B' = 6 B
    tri = ntypes * (ntypes + 1) // 2
    lj_A, lj_B = np.zeros(tri, np.float32), np.zeros(tri, np.float32)
    for a in range(ntypes):
        for b in range(a + 1):
            k = a * (a + 1) // 2 + b
            lj_A[k] = np.float32(12.0 * acoef[npi[a, b]])
            lj_B[k] = np.float32(6.0 * bcoef[npi[a, b]])
    # exclusions: one-directional lists, a 0 entry marks an atom without any
    nex = p["NUMBER_EXCLUDED_ATOMS"]
    lst = p["EXCLUDED_ATOMS_LIST"]
    start, numbers, flat, pos = [], [], [], 0
    for i in range(n):
        row = lst[pos:pos + nex[i]]
        pos += nex[i]
        row = [j - 1 for j in row if j > 0]
        start.append(len(flat))
        numbers.append(len(row))
        flat.extend(row)

    def terms(key_h, key_nh, width):
        v = np.array(p[key_h] + p[key_nh], np.int64).reshape(-1, width)
        return v

    bonds = terms("BONDS_INC_HYDROGEN", "BONDS_WITHOUT_HYDROGEN", 3)
    angles = terms("ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN", 4)
    dihedrals = terms("DIHEDRALS_INC_HYDROGEN", "DIHEDRALS_WITHOUT_HYDROGEN", 5)
    ref = json.load(open(os.path.join(CASE, "reference.json")))
    entry = next(e for e in ref["entries"]
                 if e["case_name"] == NAME and e["iteration"] == iteration)
    assert abs(entry["perturbation"] - perturbation) < 1e-12
    forces = np.load(os.path.join(CASE, entry["forces_file"]))
    out = dict(
        crd=crd.astype(np.float32), crd64=crd, box=box,
        charge=np.array(p["CHARGE"], np.float32), lj_type=typ, n_types=np.int32(ntypes),
        lj_A=lj_A, lj_B=lj_B, acoef=acoef, bcoef=bcoef, nb_index=npi.astype(np.int32),
        excl_start=np.array(start, np.int32), excl_numbers=np.array(numbers, np.int32),
        excl_list=np.array(flat, np.int32), mass=np.array(p["MASS"], np.float32),
        bonds=bonds.astype(np.int32), bond_k=np.array(p["BOND_FORCE_CONSTANT"]),
        bond_r0=np.array(p["BOND_EQUIL_VALUE"]),
        angles=angles.astype(np.int32), angle_k=np.array(p["ANGLE_FORCE_CONSTANT"]),
        angle_t0=np.array(p["ANGLE_EQUIL_VALUE"]),
        dihedrals=dihedrals.astype(np.int32), dih_k=np.array(p["DIHEDRAL_FORCE_CONSTANT"]),
        dih_n=np.array(p["DIHEDRAL_PERIODICITY"]), dih_phase=np.array(p["DIHEDRAL_PHASE"]),
        scee=np.array(p["SCEE_SCALE_FACTOR"]), scnb=np.array(p["SCNB_SCALE_FACTOR"]),
        residue_label=np.array(p["RESIDUE_LABEL"]),
        residue_pointer=np.array(p["RESIDUE_POINTER"], np.int32) - 1,
        amber_forces=forces, amber_epot=np.float64(entry["energy_epot"]),
        cutoff=np.float32(8.0),
    )
    path = os.path.join(HERE, f"amber_alanine_dipeptide_tip4pew_iter{iteration}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes;", n, "sites,", len(flat), "exclusions")


if __name__ == "__main__":
    if not os.path.isdir(CASE):
        raise SystemExit("set SPONGE_REFERENCE to the reference checkout's root")
    main()
