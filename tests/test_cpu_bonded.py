"""Harmonic bonds and angles: the FP64 oracle pinned to the reference's own
BOND and ANGLE (bond/bond.cpp, angle/angle.cpp built from its sources into
oracle/_ref), and the native bond / angle file readers against the
reference's loaders.

Fixtures (tests/golden/make_bonded_golden.py): the Amber alanine dipeptide
case's bonds and angles on its perturbed frame, the triclinic water case's
bond file in its skewed cell, and 300 waters displaced by up to 0.1 A.
Forces within relative RMS 5e-5 (the reference forms r - r0 in FP32 and the
Amber frame's bonds sit 0.02 A from their minimum, so the difference keeps
few significant bits: 2.2e-5 there, 2e-6 or less on the other cases), energies
within 1e-5 relative, per-atom energies and virial sums to FP32 accuracy.
"""

import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["bonded_amber_alanine_dipeptide.npz", "bonded_wat_nonortho.npz",
         "bonded_water_box.npz"]


def load(name):
    z = np.load(os.path.join(HERE, "golden", name))
    cell = z["cell"]
    a11, a21, a22, a31, a32, a33 = (np.float32(v) for v in cell)
    one = np.float32(1.0)
    rcell = np.array([one / a11, -a21 / (a11 * a22), one / a22,
                      (a21 * a32 - a22 * a31) / (a11 * a22 * a33), -a32 / (a22 * a33),
                      one / a33], np.float32)
    bonds = (z["bond_a"], z["bond_b"], z["bond_k"], z["bond_r0"])
    angles = (z["angle_a"], z["angle_b"], z["angle_c"], z["angle_k"], z["angle_theta0"])
    return z, rcell, bonds, angles


def rel_rms(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", CASES)
def test_oracle_bonded_matches_reference(oracle, name):
    z, rcell, bonds, angles = load(name)
    b, a = oracle.bonded_f64(z["crd"], z["cell"], rcell, bonds, angles)
    for fam, got in (("bond", b), ("angle", a)):
        if len(z[f"{fam}_k"]) == 0:
            continue
        assert rel_rms(z[f"{fam}_frc"], got["frc"]) < 5e-5, fam
        assert got["energy"] == pytest.approx(float(z[f"{fam}_energy"]), rel=1e-5), fam
        ae = z[f"{fam}_atom_energy"].astype(np.float64)
        assert np.abs(ae - got["atom_energy"]).max() <= 1e-5 * np.abs(ae).max() + 1e-6, fam
        vs = z[f"{fam}_virial"].astype(np.float64).sum(0)
        assert np.all(np.abs(vs - got["virial"].sum(0)) <= 1e-5 * np.abs(vs).max() + 1e-4), fam


def _write_terms(path, rows):
    with open(path, "w") as f:
        f.write(f"{len(rows)}\n")
        for r in rows:
            f.write(" ".join(r) + "\n")


def test_bond_angle_readers_match_reference_loaders(tmp_path):
    from oracle import oracle as om
    from sponge_b200 import capi
    if not os.path.exists(om.REF_SO):
        pytest.skip("oracle/_ref not built here")
    z, _, bonds, angles = load("bonded_water_box.npz")
    bp, ap = str(tmp_path / "bond.txt"), str(tmp_path / "angle.txt")
    _write_terms(bp, [(str(int(a)), str(int(b)), f"{k:.9g}", f"{r:.9g}")
                      for a, b, k, r in zip(*bonds)])
    _write_terms(ap, [(str(int(a)), str(int(b)), str(int(c)), f"{k:.9g}", f"{t:.9g}")
                      for a, b, c, k, t in zip(*angles)])
    lib = capi.load()
    m = ctypes.c_int(0)
    capi.check(lib.snb_read_bond_in_file(bp.encode(), ctypes.byref(m), None, None, None,
                                         None), "read_bond")
    ba, bb = np.zeros(m.value, np.int32), np.zeros(m.value, np.int32)
    bk, br = np.zeros(m.value, np.float32), np.zeros(m.value, np.float32)
    capi.check(lib.snb_read_bond_in_file(bp.encode(), ctypes.byref(m), ba.ctypes.data,
                                         bb.ctypes.data, bk.ctypes.data, br.ctypes.data),
               "read_bond")
    capi.check(lib.snb_read_angle_in_file(ap.encode(), ctypes.byref(m), None, None, None,
                                          None, None), "read_angle")
    aa, ab, ac = (np.zeros(m.value, np.int32) for _ in range(3))
    ak, at = np.zeros(m.value, np.float32), np.zeros(m.value, np.float32)
    capi.check(lib.snb_read_angle_in_file(ap.encode(), ctypes.byref(m), aa.ctypes.data,
                                          ab.ctypes.data, ac.ctypes.data, ak.ctypes.data,
                                          at.ctypes.data), "read_angle")
    ref = om.ReferenceCPU(exact=False)
    ref.native_load({"bond_in_file": bp, "angle_in_file": ap})
    assert np.array_equal(ba, ref.native_get("bond_a", np.int32))
    assert np.array_equal(bb, ref.native_get("bond_b", np.int32))
    assert np.array_equal(bk, ref.native_get("bond_k"))
    assert np.array_equal(br, ref.native_get("bond_r0"))
    assert np.array_equal(aa, ref.native_get("angle_a", np.int32))
    assert np.array_equal(ac, ref.native_get("angle_c", np.int32))
    assert np.array_equal(ak, ref.native_get("angle_k"))
    assert np.array_equal(at, ref.native_get("angle_theta0"))
    # a short row is the reference's format error
    with open(bp, "a") as f:
        f.write("1 2 3.0\n")
    with open(bp) as f:
        lines = f.read().splitlines()
    lines[0] = str(len(lines) - 1)
    with open(bp, "w") as f:
        f.write("\n".join(lines) + "\n")
    rc = lib.snb_read_bond_in_file(bp.encode(), ctypes.byref(m), ba.ctypes.data,
                                   bb.ctypes.data, bk.ctypes.data, br.ctypes.data)
    assert rc != 0 and b"bond_in_file" in lib.snb_last_error()
