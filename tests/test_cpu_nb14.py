"""1-4 terms (NON_BOND_14, nb14/nb14.cpp:8-103) on the CPU: the FP64 oracle
against the golden vectors that the reference's own NON_BOND_14 made
(tests/golden/make_nb14_golden.py), the Amber case's 1-4 energies against
Amber's own formula with its SCNB / SCEE, and the nb14 native-file reader
(snb_read_nb14_in_file) against the reference's loader
(xponge/load/native/nb14.hpp:8-101), bit for bit.

Tolerances: forces and virials 1e-5 relative RMS, energies 1e-6 relative;
the reference computes in FP32, the oracle in FP64."""

import ctypes
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["nb14_alanine_dipeptide.npz", "nb14_water_box.npz"]


class Box:
    def __init__(self, z):
        self.crd, self.charge = z["crd"], z["charge"]
        self.n = len(self.crd)
        self._cell, self._rcell = z["cell"], z["rcell"]

    def cell(self):
        return self._cell

    def rcell(self):
        return self._rcell


def load(name):
    z = np.load(os.path.join(HERE, "golden", name))
    return Box(z), z


def rel_rms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(oracle, name):
    box, z = load(name)
    o = oracle.nb14_f64(box, z["atom_a"], z["atom_b"], z["A"], z["B"], z["cf"])
    assert rel_rms(o["frc"], z["ref_frc"]) <= 1e-5
    assert rel_rms(o["atom_energy"], z["ref_atom_energy"]) <= 1e-5
    assert rel_rms(o["virial"], z["ref_virial"]) <= 1e-5
    assert abs(o["lj"] - float(z["ref_lj"])) <= 1e-6 * abs(float(z["ref_lj"])) + 1e-6
    assert abs(o["ee"] - float(z["ref_ee"])) <= 1e-6 * abs(float(z["ref_ee"]))
    # the per-atom energies hold the same total, all on the first atom of each pair
    assert abs(o["atom_energy"].sum() - (o["lj"] + o["ee"])) <= 1e-9 * abs(o["ee"])
    assert not np.any(o["atom_energy"][np.setdiff1d(np.arange(box.n), z["atom_a"])])


def test_uncharged_atoms_take_the_charge_floor(oracle):
    """The water case leaves some atoms uncharged; the reference takes their
    charge as 1e-10, so their pairs keep a vanishing but nonzero Coulomb term
    and the LJ part alone sets the force."""
    box, z = load("nb14_water_box.npz")
    zero = np.nonzero(box.charge == 0)[0]
    hit = np.isin(z["atom_a"], zero) | np.isin(z["atom_b"], zero)
    assert hit.any()
    o = oracle.nb14_f64(box, z["atom_a"][hit], z["atom_b"][hit], z["A"][hit], z["B"][hit],
                        z["cf"][hit])
    assert o["ee"] != 0.0 and abs(o["ee"]) < 1e-6


def test_amber_one_four_energy_matches_amber_formula():
    """Amber's 1-4 energy of the Amber case (LJ / SCNB with its ACOEF, BCOEF;
    q q / r / SCEE) equals the reference's sums on SPONGE's 1-4 list."""
    z = np.load(os.path.join(HERE, "golden", "amber_alanine_dipeptide_tip4pew_iter0.npz"))
    g = np.load(os.path.join(HERE, "golden", "nb14_alanine_dipeptide.npz"))
    x = np.asarray(z["crd64"], np.float64)
    L = np.asarray(z["box"], np.float64)
    d = z["dihedrals"]
    d = d[d[:, 2] >= 0]
    i, l4, t = np.abs(d[:, 0]) // 3, np.abs(d[:, 3]) // 3, d[:, 4] - 1
    dr = x[i] - x[l4]
    dr -= np.round(dr / L) * L
    r = np.linalg.norm(dr, axis=1)
    ab = z["nb_index"][z["lj_type"][i], z["lj_type"][l4]]
    lj = ((z["acoef"][ab] / r ** 12 - z["bcoef"][ab] / r ** 6) / z["scnb"][t]).sum()
    q = z["charge"].astype(np.float64)
    ee = (q[i] * q[l4] / r / z["scee"][t]).sum()
    assert abs(lj - float(g["ref_lj"])) <= 1e-5 * abs(lj) + 1e-5
    assert abs(ee - float(g["ref_ee"])) <= 1e-5 * abs(ee)


# -- nb14_in_file / nb14_extra_in_file --------------------------------------

def _lib():
    from sponge_b200 import capi
    return capi, capi.load()


def _ref():
    from oracle import oracle as om
    if not os.path.exists(om.REF_SO):
        pytest.skip("oracle/_ref not built here")
    return om.ReferenceCPU(exact=False)


def read_nb14(path, extra, s):
    capi, lib = _lib()
    m = ctypes.c_int(0)
    typ = np.ascontiguousarray(s.lj_type, np.int32)
    A_t = np.ascontiguousarray(s.lj_A, np.float32)
    B_t = np.ascontiguousarray(s.lj_B, np.float32)
    args = (path.encode() if path else None, extra.encode() if extra else None, s.n,
            typ.ctypes.data, A_t.ctypes.data, B_t.ctypes.data, ctypes.byref(m))
    rc = lib.snb_read_nb14_in_file(*args, None, None, None, None, None)
    if rc != capi.SNB_OK:
        return rc, None
    k = m.value
    out = [np.zeros(k, np.int32), np.zeros(k, np.int32), np.zeros(k, np.float32),
           np.zeros(k, np.float32), np.zeros(k, np.float32)]
    rc = lib.snb_read_nb14_in_file(*args, *[a.ctypes.data for a in out])
    return rc, out


@pytest.fixture(scope="module")
def nb14_files(tmp_path_factory):
    from tests.test_cpu_native_io import write_lj
    from sponge_b200 import systems
    d = tmp_path_factory.mktemp("nb14")
    s = systems.water_box(200, seed=7)
    rng = np.random.default_rng(8)
    m, mx = 150, 40
    a, b = rng.integers(0, s.n, m), rng.integers(0, s.n, m)
    scale = rng.choice([0.5, 1.0 / 1.2, 1.0], m)
    cf = rng.choice([0.5, 1.0 / 1.2, 1.0], m)
    with open(d / "nb14.txt", "w") as f:
        f.write(f"{m}\n")
        for r in range(m):
            f.write(f"{a[r]} {b[r]} {scale[r]:.9g} {cf[r]:.9g}\n")
    ax, bx = rng.integers(0, s.n, mx), rng.integers(0, s.n, mx)
    Ax, Bx, cx = rng.uniform(1e4, 1e6, mx), rng.uniform(10, 1e3, mx), rng.uniform(0.5, 1, mx)
    with open(d / "nb14_extra.txt", "w") as f:
        f.write(f"{mx}\n")
        for r in range(mx):
            f.write(f"{ax[r]} {bx[r]} {Ax[r]:.9g} {Bx[r]:.9g} {cx[r]:.9g}\n")
    write_lj(d / "lj.txt", s)
    return s, {"LJ_in_file": str(d / "lj.txt"), "nb14_in_file": str(d / "nb14.txt"),
               "nb14_extra_in_file": str(d / "nb14_extra.txt")}


@pytest.mark.parametrize("which", ["both", "in_file", "extra"])
def test_nb14_reader_matches_reference_loader(nb14_files, which):
    s, paths = nb14_files
    capi, lib = _lib()
    ref = _ref()
    use = dict(paths)
    if which == "in_file":
        del use["nb14_extra_in_file"]
    if which == "extra":
        del use["nb14_in_file"]
    ref.native_load(use)
    # the reference takes the types and tables from its LJ loader: read them
    # back through this project's LJ reader so both sides use the same file
    from tests.test_cpu_native_io import read_lj
    t, A_t, B_t, typ = read_lj(paths["LJ_in_file"])

    class S:
        n, lj_type, lj_A, lj_B = s.n, typ, A_t, B_t
    rc, out = read_nb14(use.get("nb14_in_file"), use.get("nb14_extra_in_file"), S)
    assert rc == capi.SNB_OK
    for arr, key in zip(out, ("nb14_a", "nb14_b", "nb14_A", "nb14_B", "nb14_cf")):
        assert np.array_equal(arr, ref.native_get(key, arr.dtype)), key


def test_nb14_reader_rejects_bad_files(nb14_files, tmp_path):
    s, paths = nb14_files
    capi, lib = _lib()
    lines = open(paths["nb14_in_file"]).read().split("\n")
    bad = tmp_path / "nb14_bad.txt"
    bad.write_text("\n".join(lines[:10]))  # fewer rows than its count
    rc, _ = read_nb14(str(bad), None, s)
    assert rc == capi.SNB_ERR_BAD_INPUT
    assert b"nb14_in_file is not right" in lib.snb_last_error()
    oob = tmp_path / "nb14_oob.txt"
    oob.write_text(f"1\n0 {s.n} 1.0 1.0\n")  # atom index past the end
    rc, _ = read_nb14(str(oob), None, s)
    assert rc == capi.SNB_ERR_BAD_INPUT
    rc, _ = read_nb14(str(tmp_path / "missing.txt"), None, s)
    assert rc == capi.SNB_ERR_BAD_INPUT
