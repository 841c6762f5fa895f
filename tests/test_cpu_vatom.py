"""Virtual atoms: the FP64 oracle pinned to the reference's own position and
force formulas (virtual_atoms/virtual_atom_math.h through oracle/_ref), and
the native virtual_atom_in_file reader against the reference's loader.

Fixtures (tests/golden/make_vatom_golden.py): the triclinic TIP4P water
case's type-2 sites in its skewed cell, and 200 atoms with sites of all four
types and a second layer of sites built from sites.  Positions within 2e-5 A
(the reference computes in FP32), redistributed forces within relative RMS
1e-6.
"""

import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["vatom_wat_nonortho.npz", "vatom_mixed.npz"]


def load(name):
    z = np.load(os.path.join(HERE, "golden", name))
    a11, a21, a22, a31, a32, a33 = (np.float32(v) for v in z["cell"])
    one = np.float32(1.0)
    rcell = np.array([one / a11, -a21 / (a11 * a22), one / a22,
                      (a21 * a32 - a22 * a31) / (a11 * a22 * a33), -a32 / (a22 * a33),
                      one / a33], np.float32)
    records = (z["type"], z["virtual_atom"], z["source"], z["parameter"])
    return z, rcell, records


@pytest.mark.parametrize("name", CASES)
def test_oracle_vatom_matches_reference(oracle, name):
    z, rcell, records = load(name)
    x, f, bad = oracle.vatom_f64(records, z["cell"], rcell, z["crd_in"], z["frc_in"])
    assert bad == 0
    assert np.abs(x - z["crd_out"]).max() <= 2e-5
    want = z["frc_out"].astype(np.float64)
    assert np.linalg.norm(f - want) / np.linalg.norm(want) <= 1e-6
    assert not np.any(f[z["virtual_atom"]])


def _min_image(d, cell, rcell):
    c, r = np.asarray(cell, np.float64), np.asarray(rcell, np.float64)
    d = np.array(d, np.float64)
    fx = np.floor(d[:, 0] * r[0] + d[:, 1] * r[1] + d[:, 2] * r[3] + 0.5)
    fy = np.floor(d[:, 1] * r[2] + d[:, 2] * r[4] + 0.5)
    fz = np.floor(d[:, 2] * r[5] + 0.5)
    d[:, 0] -= fx * c[0] + fy * c[1] + fz * c[3]
    d[:, 1] -= fy * c[2] + fz * c[4]
    d[:, 2] -= fz * c[5]
    return d


def test_oracle_vatom_conserves_force_and_torque(oracle):
    """Moving a type-2 site's force onto its atoms keeps each water's force
    and torque (the weights sum to one and the site is their weighted mean):
    the invariants a rigid-water force scheme must keep."""
    z, rcell, records = load("vatom_wat_nonortho.npz")
    x, f, _ = oracle.vatom_f64(records, z["cell"], rcell, z["crd_in"], z["frc_in"])
    f_in = z["frc_in"].astype(np.float64)
    for t in range(0, len(records[0]), 97):
        v, (a, b, c) = records[1][t], records[2][t]
        atoms = [a, b, c, v]
        # the water's atoms relative to O, minimum image on the skewed cell
        r = _min_image(x[atoms] - x[a], z["cell"], rcell)
        assert np.allclose(f[atoms].sum(0), f_in[atoms].sum(0), atol=1e-9)
        tq_in = np.cross(r, f_in[atoms]).sum(0)
        tq = np.cross(r, f[atoms]).sum(0)
        assert np.allclose(tq, tq_in, atol=1e-6 * np.abs(tq_in).max() + 1e-9)


def _write_records(path, records, extra=()):
    ty, vi, fr, pa = records
    with open(path, "w") as f:
        f.write("# virtual atoms\n")
        for t, v, s, p in zip(ty, vi, fr, pa):
            if t == 0:
                f.write(f"0 {v} {s[0]} {p[0]:.9g}\n")
            elif t == 1:
                f.write(f"1 {v} {s[0]} {s[1]} {p[0]:.9g}\n")
            else:
                f.write(f"{t} {v} {s[0]} {s[1]} {s[2]} {p[0]:.9g} {p[1]:.9g}  # site\n")
        for line in extra:
            f.write(line + "\n")


def _read(path):
    from sponge_b200 import capi
    lib = capi.load()
    m = ctypes.c_int(0)
    rc = lib.snb_read_virtual_atom_in_file(path.encode(), ctypes.byref(m), None, None, None,
                                           None)
    if rc:
        return rc, None
    ty, vi = np.zeros(m.value, np.int32), np.zeros(m.value, np.int32)
    fr, pa = np.zeros(3 * m.value, np.int32), np.zeros(2 * m.value, np.float32)
    capi.check(lib.snb_read_virtual_atom_in_file(path.encode(), ctypes.byref(m),
                                                 ty.ctypes.data, vi.ctypes.data,
                                                 fr.ctypes.data, pa.ctypes.data), "read")
    return 0, (ty, vi, fr.reshape(-1, 3), pa.reshape(-1, 2))


def test_reader_matches_reference_loader(tmp_path):
    from oracle import oracle as om
    if not os.path.exists(om.REF_SO):
        pytest.skip("oracle/_ref not built here")
    _, _, records = load("vatom_mixed.npz")
    p = str(tmp_path / "vatom.txt")
    _write_records(p, records, extra=["", "not a record"])
    rc, got = _read(p)
    assert rc == 0
    ref = om.ReferenceCPU(exact=False)
    ref.native_load({"virtual_atom_in_file": p})
    m = len(got[0])
    assert np.array_equal(got[0], ref.native_get("vatom_type", np.int32))
    assert np.array_equal(got[1], ref.native_get("vatom_virtual", np.int32))
    assert np.array_equal(got[2].reshape(-1), ref.native_get("vatom_from", np.int32))
    assert np.array_equal(got[3].reshape(-1), ref.native_get("vatom_param"))
    assert m == len(records[0])


@pytest.mark.parametrize("line", ["4 7 1 2 3 0.5 0.5", "2 7 1 2 0.5", "1 7 1 2 0.5 junk"])
def test_reader_rejects_what_the_reference_rejects(tmp_path, line):
    p = str(tmp_path / "bad.txt")
    with open(p, "w") as f:
        f.write("0 5 1 2.0\n" + line + "\n")
    rc, _ = _read(p)
    assert rc != 0
