"""A skewed cell on the GPU: the reference's own triclinic water case
(WAT_nonortho, 4,324 sites, 60-degree angles, cutoff 8 A, skin 2 A;
tests/golden/wat_nonortho_rc8.npz) through the module entry points.

  * the neighbor list's pair set is the oracle's bit for bit: every pair the
    reference's criterion accepts on the full lower-triangular cell, which
    is the reference's own set plus the pairs its grid table misses
    (listed in the fixture);
  * LJ + direct Coulomb over that list, the PME reciprocal part on the
    reference's grid (40 x 36 x 28) and the excluded correction are within
    relative RMS 1e-5 of FP64 (forces), 1e-6 / 2e-6 (energies) and 1e-5 of
    the largest component (the reciprocal virial).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.fixture(scope="module")
def case():
    from tests import nonortho
    return nonortho.load()


def test_pair_set_bit_exact_on_skewed_cell(g, oracle, case):
    s, z = case
    box = g.Box(s)
    nl = g.make_nl(box, 8.0, 2.0)
    try:
        g.nl_update(nl, box)
        got = g.nl_pairs(nl)
    finally:
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs_system(s, 8.0, 2.0)
    want = g.csr_to_pairs(rs, cols)
    assert np.array_equal(got, want)
    assert len(got) == int(z["pair_numbers"]) + len(z["pairs_missed_by_reference"])


def test_direct_pme_excluded_on_skewed_cell(g, oracle, case):
    s, z = case
    box = g.Box(s)
    lib = g.capi.load()
    beta = oracle.get_beta(8.0)
    assert beta == float(z["beta"])
    nl = g.make_nl(box, 8.0, 2.0)
    lj = g.lj_create(box, 8.0)
    pme, pbeta, grid = g.pme_create(box, 8.0)
    try:
        g.nl_update(nl, box)
        d = g.lj_force(lj, nl, box, beta)
        p = g.pme_reciprocal(pme, box)
        e = g.pme_excluded(pme, box)
    finally:
        lib.snb_lj_destroy(lj)
        lib.snb_nl_destroy(nl)
        lib.snb_pme_destroy(pme)
    assert grid == tuple(int(k) for k in z["grid"]) and pbeta == beta
    rs, cols = oracle.nl_pairs_system(s, 8.0, 2.0)
    dw = oracle.direct_f64(s, 8.0, beta, rs, cols)
    pw = oracle.pme_f64(s, grid, beta)
    ew = oracle.excluded_f64(s, beta)
    assert g.rel_rms(d["frc"], dw["frc"]) <= FORCE_TOL
    assert g.rel_rms(p["frc"], pw["frc"]) <= FORCE_TOL
    assert g.rel_rms(e["frc"], ew["frc"]) <= FORCE_TOL
    e_dir = float(np.sum(d["atom_energy"], dtype=np.float64))
    assert abs(e_dir - dw["atom_energy"].sum()) <= 1e-6 * abs(dw["atom_energy"].sum())
    v_dir = d["virial"].astype(np.float64).sum(0)
    assert np.all(np.abs(v_dir - dw["virial"].sum(0)) <= 1e-6 * np.abs(v_dir).max() + 1e-3)
    assert p["e_recip"] == pytest.approx(pw["e_recip"], rel=2e-6)
    assert p["e_self"] == pytest.approx(pw["e_self"], rel=1e-6)
    # the skewed cell's reciprocal virial is a sum of large terms of both
    # signs: held to 1e-5 of its largest component, the bound the reference's
    # own FP32 build meets against FP64 on this case
    assert np.allclose(p["virial64"], pw["virial"], rtol=1e-5,
                       atol=1e-5 * np.abs(pw["virial"]).max())
    e_ex = float(np.sum(e["atom_energy"], dtype=np.float64))
    assert abs(e_ex - ew["atom_energy"].sum()) <= 1e-6 * abs(ew["atom_energy"].sum())


def test_engine_refuses_skewed_cell(g, case):
    s, _ = case
    with pytest.raises(g.capi.SnbError):
        g.engine_create(s, 8.0)
