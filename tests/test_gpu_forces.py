"""LJ + direct Coulomb, PME reciprocal and excluded correction on the GPU
against the FP64 oracle run of the same method.

Tolerances (written here, measured on B200):
  forces: relative RMS error <= 1e-5 against FP64;
  energies and virials: relative error <= 1e-6 of the component's magnitude
  for the pair sums; the PME reciprocal energy/virial go through a float FFT
  and are held to 2e-6.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
ENERGY_TOL = 1e-6
PME_E_TOL = 2e-6


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _direct(g, oracle, s, cutoff, accumulation):
    box = g.Box(s)
    nl = g.make_nl(box, cutoff, 2.0)
    lj = g.lj_create(box, cutoff, accumulation)
    beta = oracle.get_beta(cutoff)
    try:
        g.nl_update(nl, box)
        got = g.lj_force(lj, nl, box, beta)
    finally:
        g.capi.load().snb_lj_destroy(lj)
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs_system(s, cutoff, 2.0)
    want = oracle.direct_f64(s, cutoff, beta, rs, cols)
    return got, want


@pytest.mark.parametrize("accumulation", ["fixed64", "float"])
def test_lj_direct_matches_fp64(g, oracle, box_9k, accumulation):
    got, want = _direct(g, oracle, box_9k, 8.0, accumulation)
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL
    e_got = float(np.sum(got["atom_energy"], dtype=np.float64))
    e_want = float(np.sum(want["atom_energy"]))
    assert abs(e_got - e_want) <= ENERGY_TOL * abs(e_want) + 1e-3
    c_got = float(np.sum(got["coulomb_energy"], dtype=np.float64))
    assert abs(c_got - want["coulomb_energy"].sum()) <= ENERGY_TOL * abs(
        want["coulomb_energy"].sum()) + 1e-3
    v_got = got["virial"].astype(np.float64).sum(0)
    v_want = want["virial"].sum(0)
    assert np.all(np.abs(v_got - v_want) <= ENERGY_TOL * np.abs(v_want).max() + 1e-3)


def test_lj_per_atom_assignment_matches_reference_rule(g, oracle, small_box):
    """Pair energy and virial go to the atom with the smaller index, as in the
    reference half list; compare per atom."""
    got, want = _direct(g, oracle, small_box, 8.0, "fixed64")
    assert np.abs(got["atom_energy"] - want["atom_energy"]).max() < 2e-4
    assert np.abs(got["virial"] - want["virial"]).max() < 2e-3


def test_fixed_point_is_bitwise_deterministic(g, oracle, box_9k):
    a, _ = _direct(g, oracle, box_9k, 8.0, "fixed64")
    b, _ = _direct(g, oracle, box_9k, 8.0, "fixed64")
    for k in ("frc", "atom_energy", "virial", "coulomb_energy"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("accumulation", ["fixed64", "float"])
def test_pme_reciprocal_matches_fp64(g, oracle, box_9k, accumulation):
    s = box_9k
    box = g.Box(s)
    h, beta, grid = g.pme_create(box, 8.0, accumulation)
    try:
        got = g.pme_reciprocal(h, box)
    finally:
        g.capi.load().snb_pme_destroy(h)
    want = oracle.pme_f64(s, grid, beta)
    assert grid == (48, 48, 48)
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL
    assert abs(got["e_recip"] - want["e_recip"]) <= PME_E_TOL * abs(want["e_recip"])
    assert abs(got["e_self"] - want["e_self"]) <= 1e-9 * abs(want["e_self"])
    scale = np.abs(want["virial"]).max()
    assert np.all(np.abs(got["virial64"] - want["virial"]) <= PME_E_TOL * scale)
    assert abs(got["potential"] - (want["e_recip"] + want["e_self"])) <= 1e-6 * abs(
        want["e_self"])


def test_pme_spread_is_bitwise_deterministic(g, box_9k):
    box = g.Box(box_9k)
    outs = []
    for _ in range(2):
        h, _, _ = g.pme_create(box, 8.0)
        try:
            outs.append(g.pme_reciprocal(h, box))
        finally:
            g.capi.load().snb_pme_destroy(h)
    assert np.array_equal(outs[0]["frc"], outs[1]["frc"])


def test_pme_update_interval(g, box_9k):
    """PME_update_interval = 2: forces scaled by 2 on even steps, none on odd
    steps (PM_force.cpp:1081-1138)."""
    box = g.Box(box_9k)
    h1, _, _ = g.pme_create(box, 8.0)
    h2, _, _ = g.pme_create(box, 8.0, PME_update_interval=2)
    try:
        f1 = g.pme_reciprocal(h1, box, step=0)["frc"]
        f2 = g.pme_reciprocal(h2, box, step=0)["frc"]
        f3 = g.pme_reciprocal(h2, box, step=1)["frc"]
    finally:
        g.capi.load().snb_pme_destroy(h1)
        g.capi.load().snb_pme_destroy(h2)
    assert np.allclose(f2, 2 * f1, rtol=1e-6, atol=1e-6)
    assert not np.any(f3)


def test_excluded_correction_matches_fp64(g, oracle, box_9k):
    s = box_9k
    box = g.Box(s)
    h, beta, _ = g.pme_create(box, 8.0)
    try:
        got = g.pme_excluded(h, box)
    finally:
        g.capi.load().snb_pme_destroy(h)
    want = oracle.excluded_f64(s, beta)
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL
    e_want = want["atom_energy"].sum()
    assert abs(got["atom_energy"].astype(np.float64).sum() - e_want) <= ENERGY_TOL * abs(e_want)


def test_long_range_correction(g, oracle, box_9k):
    import torch
    s = box_9k
    box = g.Box(s)
    lj = g.lj_create(box, 8.0)
    lib = g.capi.load()
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    pot = torch.zeros(1, dtype=torch.float32, device="cuda")
    V = float(np.float32(s.box) ** 3)
    try:
        g.capi.check(lib.snb_lj_long_range_correction(lj, 1, g.ptr(vir), 1, g.ptr(pot),
                                                      g.ctypes.c_float(V), g.stream()), "lrc")
        f = lib.snb_lj_long_range_factor(lj)
    finally:
        lib.snb_lj_destroy(lj)
    want = oracle.lrc_factor(s, 8.0)
    assert f == pytest.approx(want, rel=1e-7)
    assert float(pot.cpu()[0]) == pytest.approx(want / V, rel=1e-6)
    v = vir.cpu().numpy()
    assert v[0] == pytest.approx(2 * want / V, rel=1e-6) and v[1] == 0.0
