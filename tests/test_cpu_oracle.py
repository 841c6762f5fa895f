"""The oracle pinned against the reference's own outputs (CPU only).

The golden vectors in tests/golden/ were produced by the reference's own
neighbor_list / Lennard_Jones_force / PM_force CPU code (oracle/_ref, built
from its sources); tests/golden/make_golden.py regenerates them.  The oracle
restatement must reproduce them: the pair set exactly, forces and energies to
FP32 accuracy (the reference computes in FP32 with fast math).
"""

import hashlib
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
_FIXTURES = sorted(f for f in os.listdir(os.path.join(HERE, "golden")) if f.endswith(".npz"))
# the pair-set / force fixtures of make_golden.py are named for their water boxes
GOLDEN = [f for f in _FIXTURES if f.startswith("water")]
SOFT = [f for f in _FIXTURES if f.startswith("soft_")]
BOXCHANGE = [f for f in _FIXTURES if f.startswith("boxchange_")]


def load_case(name):
    from sponge_b200 import systems
    z = np.load(os.path.join(HERE, "golden", name))
    s = systems.System(
        crd=z["crd"], vel=np.zeros_like(z["crd"]), charge=z["charge"],
        lj_type=z["lj_type"], lj_A=z["lj_A"], lj_B=z["lj_B"],
        mass=np.ones(len(z["charge"]), np.float32), excl_start=z["excl_start"],
        excl_numbers=z["excl_numbers"], excl_list=z["excl_list"],
        bonds=np.zeros((0, 2), np.int32), angles=np.zeros((0, 3), np.int32),
        box=float(z["box"]))
    return s, z


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_pair_set_equals_reference(oracle, name):
    s, z = load_case(name)
    rs, cols = oracle.nl_pairs_system(s, float(z["cutoff"]), float(z["skin"]))
    assert np.array_equal(np.diff(rs).astype(np.int32), z["nl_counts"])
    i = np.repeat(np.arange(s.n), np.diff(rs))
    pairs = np.stack([i, cols.astype(np.int64)], 1)
    digest = hashlib.sha256(np.ascontiguousarray(pairs, np.int32).tobytes()).hexdigest()
    assert digest == str(z["nl_pair_sha256"])


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_beta_and_grid(oracle, name):
    from sponge_b200 import systems
    s, z = load_case(name)
    assert oracle.get_beta(float(z["cutoff"]), 1e-5, 0) == float(z["beta"])
    assert tuple(z["grid"]) == (systems.fft_size(s.box),) * 3


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_direct_matches_reference(oracle, name):
    s, z = load_case(name)
    cutoff, beta = float(z["cutoff"]), float(z["beta"])
    rs, cols = oracle.nl_pairs_system(s, cutoff, float(z["skin"]))
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    assert rel_rms(z["lj_frc"], d["frc"]) < 5e-6
    assert np.abs(z["lj_atom_energy"] - d["atom_energy"]).max() < 1e-3
    assert np.abs(z["lj_lj_energy"] - d["lj_energy"]).max() < 1e-3
    assert np.abs(z["lj_coulomb_energy"] - d["coulomb_energy"]).max() < 1e-3
    vs = z["lj_virial"].astype(np.float64).sum(0)
    assert np.all(np.abs(vs - d["virial"].sum(0)) < 1e-5 * np.abs(vs).max() + 1e-3)


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_pme_matches_reference(oracle, name):
    s, z = load_case(name)
    beta = float(z["beta"])
    p = oracle.pme_f64(s, tuple(z["grid"]), beta)
    assert rel_rms(z["pme_frc"], p["frc"]) < 1e-5
    assert float(z["pme_e_recip"]) == pytest.approx(p["e_recip"], rel=2e-6)
    assert float(z["pme_e_self"]) == pytest.approx(p["e_self"], rel=1e-6)
    assert np.allclose(z["pme_virial"], p["virial"], rtol=1e-5,
                       atol=1e-5 * np.abs(p["virial"]).max())


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_excluded_matches_reference(oracle, name):
    s, z = load_case(name)
    e = oracle.excluded_f64(s, float(z["beta"]))
    assert rel_rms(z["excl_frc"], e["frc"]) < 5e-6
    assert np.abs(z["excl_atom_energy"] - e["atom_energy"]).max() < 2e-3


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_long_range_correction(oracle, name):
    s, z = load_case(name)
    # the reference's fast-math build may reassociate the float scaling chain:
    # one ulp
    assert oracle.lrc_factor(s, float(z["cutoff"])) == pytest.approx(
        float(z["lrc_factor"]), rel=2e-7)


def test_oracle_pme_approximates_ewald(oracle, small_box):
    """The oracle's PME reciprocal sum converges to the plain Ewald sum: 1 A grid,
    order 4 gives ~1e-3 relative energy and force error (a property of the
    method, checked to make sure the oracle implements it)."""
    from sponge_b200 import systems
    s = small_box
    beta = oracle.get_beta(8.0)
    p = oracle.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)
    e, f = oracle.ewald_recip_f64(s, beta, 12)
    assert abs(p["e_recip"] - e) < 5e-3 * abs(e)
    assert rel_rms(p["frc"], f) < 1e-2


def test_reference_build_reproduces_golden_when_present(name=GOLDEN[0]):
    """Where the reference sources exist (this container), its live output
    still equals the committed fixture."""
    from oracle import oracle as om
    if not os.path.exists(om.REF_SO):
        pytest.skip("oracle/_ref not built here")
    s, z = load_case(name)
    ref = om.ReferenceCPU(exact=False)
    ref.init(s, float(z["cutoff"]), float(z["skin"]))
    counts, serial, _ = ref.nl_update()
    assert np.array_equal(counts, z["nl_counts"])
    lj = ref.lj_direct()
    assert rel_rms(lj["frc"], z["lj_frc"].astype(np.float64)) < 1e-6


def load_soft_case(name):
    from sponge_b200 import systems
    s, z = load_case(name)
    sc = systems.SoftCore(
        type_A=z["type_A"], type_B=z["type_B"], n_types_A=int(z["n_types_A"]),
        n_types_B=int(z["n_types_B"]), AA=z["AA"], AB=z["AB"], BA=z["BA"], BB=z["BB"],
        mask=z["mask"], charge_B_A=z["charge_B_A"])
    s.n_types = int(z["n_types_A"])
    return s, sc, z


@pytest.mark.parametrize("name", SOFT)
def test_oracle_soft_core_matches_reference(oracle, name):
    """FP64 soft-core restatement against LJ_SOFT_CORE's own output: forces,
    the energy split (total, LJ, inter/intra subsystem, direct Coulomb),
    virial, dH/dlambda and the tail factors, to FP32 accuracy."""
    s, sc, z = load_soft_case(name)
    cutoff, beta = float(z["cutoff"]), float(z["beta"])
    rs, cols = oracle.nl_pairs_system(s, cutoff, float(z["skin"]))
    i = np.repeat(np.arange(s.n), np.diff(rs))
    pairs = np.stack([i, cols.astype(np.int64)], 1)
    digest = hashlib.sha256(np.ascontiguousarray(pairs, np.int32).tobytes()).hexdigest()
    assert digest == str(z["nl_pair_sha256"])
    lam = float(z["lam"])
    d = oracle.soft_f64(s, sc, cutoff, beta, lam, float(z["alpha"]), float(z["p"]),
                        float(z["sigma"]), float(z["sigma_min"]), rs, cols)
    assert rel_rms(z["frc"], d["frc"]) < 5e-6
    for k in ("atom_energy", "lj_energy", "inter", "intra", "coulomb_energy"):
        scale = np.abs(d[k]).sum()
        assert abs(z[k].astype(np.float64).sum() - d[k].sum()) < 2e-6 * scale, k
        assert np.abs(z[k] - d[k]).max() < 2e-3, k
    vs = z["virial"].astype(np.float64).sum(0)
    assert np.all(np.abs(vs - d["virial"].sum(0)) < 1e-5 * np.abs(vs).max() + 1e-3)
    fac, fti = oracle.soft_lrc(s, sc, lam, cutoff)
    assert fac == pytest.approx(float(z["lrc_factor"]), rel=1e-6)
    assert fti == pytest.approx(float(z["lrc_factor_ti"]), rel=1e-6)
    V = float(np.float32(s.box) ** 3)
    # the reference sums dH/dlambda in float over the atoms
    assert d["dudl_lj"] + fti / V == pytest.approx(float(z["dhdl"]), rel=2e-5, abs=1e-3)


@pytest.mark.parametrize("name", BOXCHANGE)
def test_oracle_box_change_matches_reference(oracle, name):
    """After a barostat's box change (the reference initialised on box0,
    then the box and coordinates scaled; PME's Update_Box at the old grid
    size, the list rebuilt in its Initial grid): the exact pair set of the new
    box, and the PME forces and energies of the new box at the old grid size.
    The reciprocal virial is pinned to the reference initialised at the new
    box: Update_Box forms the virial factor with the opposite sign of the
    pi^2 m^2 / beta^2 term (PM_force.cpp:1210-1236 against :557-604), so its
    virial after a box change is not the target."""
    s, z = load_case(name)
    assert float(z["box"]) != float(z["box0"])
    rs, cols = oracle.nl_pairs_system(s, float(z["cutoff"]), float(z["skin"]))
    i = np.repeat(np.arange(s.n), np.diff(rs))
    pairs = np.stack([i, cols.astype(np.int64)], 1)
    digest = hashlib.sha256(np.ascontiguousarray(pairs, np.int32).tobytes()).hexdigest()
    assert digest == str(z["nl_pair_sha256"])
    p = oracle.pme_f64(s, tuple(z["grid"]), float(z["beta"]))
    assert rel_rms(z["pme_frc"], p["frc"]) < 1e-5
    assert float(z["pme_e_recip"]) == pytest.approx(p["e_recip"], rel=2e-6)
    assert float(z["pme_e_self"]) == pytest.approx(p["e_self"], rel=1e-6)
    assert rel_rms(z["pme_frc_fresh"], p["frc"]) < 1e-5
    assert np.allclose(z["pme_virial_fresh"], p["virial"], rtol=1e-5,
                       atol=1e-5 * np.abs(p["virial"]).max())
    assert not np.allclose(z["pme_virial"], p["virial"], rtol=1e-2)
