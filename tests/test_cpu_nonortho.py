"""The oracle pinned on a skewed cell: the reference's own triclinic water
case (benchmarks/performance/nonortho/statics/WAT_nonortho, 4,324 sites,
60-degree angles; tests/golden/wat_nonortho_rc8.npz from
tests/golden/make_nonortho_golden.py, which runs the reference's own CPU
build).  The oracle restatement holds every pair the reference's criterion
accepts (the minimum image and |dr|^2 < r_l^2 on the full lower-triangular
cell, evaluated for all pairs); the reference's own set is exactly that set
less the pairs its neighbour-grid table does not reach (478 here, 33 of them
inside the cutoff), which the fixture lists.  With the reference's pair set
the oracle reproduces its direct forces and energies, and its PME and
excluded forces and energies, to FP32 accuracy.
"""

import hashlib

import numpy as np
import pytest

from tests import nonortho


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    return nonortho.load()


def test_fixture_cell_is_skewed(case):
    s, z = case
    assert np.all(np.abs(z["cell"][[1, 3, 4]]) > 5.0)
    assert np.allclose(np.asarray(z["box"][3:]), 60.0)


def _reference_pairs(oracle, s, z):
    """The oracle's complete set less the pairs the reference's grid misses."""
    rs, cols = oracle.nl_pairs_system(s, float(z["cutoff"]), float(z["skin"]))
    i = np.repeat(np.arange(s.n), np.diff(rs))
    full = np.stack([i, cols.astype(np.int64)], 1)
    missed = z["pairs_missed_by_reference"].astype(np.int64)
    key = full[:, 0] * s.n + full[:, 1]
    keep = ~np.isin(key, missed[:, 0] * s.n + missed[:, 1])
    return full, full[keep]


def test_oracle_pair_set_is_reference_plus_missed(oracle, case):
    s, z = case
    full, ref = _reference_pairs(oracle, s, z)
    missed = z["pairs_missed_by_reference"]
    assert len(full) == int(z["pair_numbers"]) + len(missed)
    assert len(ref) == int(z["pair_numbers"])
    assert np.array_equal(np.bincount(ref[:, 0], minlength=s.n), z["pair_row_counts"])
    digest = hashlib.sha256(np.ascontiguousarray(ref, np.int32).tobytes()).hexdigest()
    assert digest == str(z["pairs_sha256"])


def test_missed_pairs_meet_the_reference_criterion(case):
    """Each pair the reference leaves out has |dr| < r_l under its own
    minimum image (evaluated here in FP64 from the same float inputs)."""
    s, z = case
    m = z["pairs_missed_by_reference"].astype(np.int64)
    assert len(m) > 0
    cell = s.cell().astype(np.float64)
    rc = s.rcell().astype(np.float64)
    d = s.crd[m[:, 0]].astype(np.float64) - s.crd[m[:, 1]]
    fx = np.floor(d[:, 0] * rc[0] + d[:, 1] * rc[1] + d[:, 2] * rc[3] + 0.5)
    fy = np.floor(d[:, 1] * rc[2] + d[:, 2] * rc[4] + 0.5)
    fz = np.floor(d[:, 2] * rc[5] + 0.5)
    d[:, 0] -= fx * cell[0] + fy * cell[1] + fz * cell[3]
    d[:, 1] -= fy * cell[2] + fz * cell[4]
    d[:, 2] -= fz * cell[5]
    r = np.linalg.norm(d, axis=1)
    rl = 0.5 * (float(z["cutoff"]) + float(z["skin"])) * 2.0
    assert np.all(r < rl + 1e-4)
    assert np.count_nonzero(r < float(z["cutoff"])) > 0


def test_oracle_beta(oracle, case):
    _, z = case
    assert oracle.get_beta(float(z["cutoff"]), 1e-5, 0) == float(z["beta"])


def test_oracle_direct_matches_reference(oracle, case):
    s, z = case
    cutoff, beta = float(z["cutoff"]), float(z["beta"])
    _, ref = _reference_pairs(oracle, s, z)
    rs = np.zeros(s.n + 1, np.int64)
    rs[1:] = np.cumsum(np.bincount(ref[:, 0], minlength=s.n))
    d = oracle.direct_f64(s, cutoff, beta, rs, ref[:, 1].astype(np.int32))
    assert rel_rms(z["lj_frc"], d["frc"]) < 5e-6
    assert abs(z["lj_energy"].astype(np.float64).sum() - d["lj_energy"].sum()) < \
        1e-5 * abs(d["lj_energy"].sum())
    assert abs(z["coulomb_energy"].astype(np.float64).sum() - d["coulomb_energy"].sum()) < \
        1e-5 * abs(d["coulomb_energy"].sum())
    vs = z["lj_virial"].astype(np.float64).sum(0)
    assert np.all(np.abs(vs - d["virial"].sum(0)) < 1e-5 * np.abs(vs).max() + 1e-3)


def test_oracle_pme_matches_reference(oracle, case):
    s, z = case
    p = oracle.pme_f64(s, tuple(int(k) for k in z["grid"]), float(z["beta"]))
    assert rel_rms(z["pme_frc"], p["frc"]) < 1e-5
    assert float(z["pme_e_recip"]) == pytest.approx(p["e_recip"], rel=2e-6)
    assert float(z["pme_e_self"]) == pytest.approx(p["e_self"], rel=1e-6)
    assert np.allclose(z["pme_virial"], p["virial"], rtol=1e-5,
                       atol=1e-5 * np.abs(p["virial"]).max())


def test_oracle_excluded_matches_reference(oracle, case):
    s, z = case
    e = oracle.excluded_f64(s, float(z["beta"]))
    assert rel_rms(z["excl_frc"], e["frc"]) < 5e-6
    assert np.abs(z["excl_energy"] - e["atom_energy"]).max() < 2e-3
