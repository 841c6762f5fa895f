"""LJ_SOFT_CORE on the GPU (snb_lj_soft_*) against the FP64 oracle run of
the same method (oracle/snb_oracle.c, pinned to the reference's own soft-core
output by tests/test_cpu_oracle.py).

Box: 1,000 waters with a 32-site alchemical solute whose LJ and charges vanish
in state B, cutoff 8 A.  Tolerances (written here, measured on B200):
  forces: relative RMS <= 1e-5 against FP64;
  energies: |sum error| <= 1e-6 of the sum of per-atom magnitudes, per
  component (total, LJ, inter/intra subsystem LJ, direct Coulomb);
  virial: <= 1e-6 of the largest component's magnitude sum;
  dH/dlambda (LJ part plus tail term, the module's return value): 1e-5.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CUTOFF = 8.0
FORCE_TOL = 1e-5
ENERGY_TOL = 1e-6


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.fixture(scope="module")
def soft_box():
    from sponge_b200 import systems
    return systems.soft_core_box(1000, n_solute=32, seed=3)


def _params(lam, alpha=0.5, p=1.0, sigma=3.0, sigma_min=0.0):
    return {"lambda_lj": lam, "soft_core_alpha": alpha, "soft_core_powfer": p,
            "soft_core_sigma": sigma, "soft_core_sigma_min": sigma_min}


def _run(g, oracle, soft_box, params, accumulation="fixed64"):
    s, sc = soft_box
    box = g.Box(s)
    beta = oracle.get_beta(CUTOFF)
    nl = g.make_nl(box, CUTOFF, 2.0)
    h = g.soft_create(box, sc, CUTOFF, params, accumulation)
    try:
        g.nl_update(nl, box)
        got = g.soft_force(h, nl, box, sc, beta)
        dhdl = g.soft_dhdl(h, nl, box, sc, beta)
    finally:
        g.capi.load().snb_lj_soft_destroy(h)
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs_system(s, CUTOFF, 2.0)
    want = oracle.soft_f64(s, sc, CUTOFF, beta, params["lambda_lj"],
                           params["soft_core_alpha"], params["soft_core_powfer"],
                           params["soft_core_sigma"], params["soft_core_sigma_min"],
                           rs, cols)
    return s, sc, got, dhdl, want


def _close_sum(got, want, what):
    scale = np.abs(want).sum()
    err = abs(float(np.asarray(got, np.float64).sum()) - want.sum())
    assert err <= ENERGY_TOL * scale, f"{what}: {err:.3e} > {ENERGY_TOL * scale:.3e}"


@pytest.mark.parametrize("lam", [0.0, 0.3, 0.7, 1.0])
def test_soft_core_matches_fp64(g, oracle, soft_box, lam):
    s, sc, got, dhdl, want = _run(g, oracle, soft_box, _params(lam))
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL
    _close_sum(got["atom_energy"], want["atom_energy"], "atom energy")
    _close_sum(got["coulomb_energy"], want["coulomb_energy"], "direct Coulomb")
    for k, idx in (("lj_energy", 0), ("inter", 1), ("intra", 2)):
        scale = np.abs(want[k]).sum()
        assert abs(float(got["sums"][idx]) - want[k].sum()) <= ENERGY_TOL * scale + 1e-4, k
    vg = got["virial"].astype(np.float64).sum(0)
    vw = want["virial"].sum(0)
    assert np.all(np.abs(vg - vw) <= ENERGY_TOL * np.abs(want["virial"]).sum(0).max())
    fac, fti = oracle.soft_lrc(s, sc, lam, CUTOFF)
    V = float(np.float32(s.box) ** 3)
    ref_dhdl = want["dudl_lj"] + fti / V
    assert dhdl == pytest.approx(ref_dhdl, rel=1e-5, abs=1e-4)


def test_soft_core_parameter_keys(g, oracle, soft_box):
    """alpha, power and sigma_min away from their defaults (sigma_min above
    most pair sigmas, so the max(A/2B, sigma_min^6) branch is taken)."""
    s, sc, got, dhdl, want = _run(g, oracle, soft_box,
                                  _params(0.4, alpha=0.7, p=2.0, sigma=3.2, sigma_min=3.6))
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL
    _close_sum(got["atom_energy"], want["atom_energy"], "atom energy")
    fac, fti = oracle.soft_lrc(s, sc, 0.4, CUTOFF)
    V = float(np.float32(s.box) ** 3)
    assert dhdl == pytest.approx(want["dudl_lj"] + fti / V, rel=1e-5, abs=1e-4)


def test_soft_core_float_accumulation(g, oracle, soft_box):
    s, sc, got, dhdl, want = _run(g, oracle, soft_box, _params(0.5), "float")
    assert g.rel_rms(got["frc"], want["frc"]) <= FORCE_TOL


def test_soft_core_long_range_correction(g, oracle, soft_box):
    import torch
    s, sc = soft_box
    box = g.Box(s)
    h = g.soft_create(box, sc, CUTOFF, _params(0.3))
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    pot = torch.zeros(1, dtype=torch.float32, device="cuda")
    V = float(np.float32(s.box) ** 3)
    lib = g.capi.load()
    try:
        g.capi.check(lib.snb_lj_soft_long_range_correction(h, 1, g.ptr(vir), 1, g.ptr(pot),
                                                           V, g.stream()), "soft lrc")
        sums = np.zeros(4, np.float32)
        g.capi.check(lib.snb_lj_soft_energy_sums(h, sums.ctypes.data, g.stream()), "sums")
        torch.cuda.synchronize()
    finally:
        lib.snb_lj_soft_destroy(h)
    fac, _ = oracle.soft_lrc(s, sc, 0.3, CUTOFF)
    assert float(pot.cpu()[0]) == pytest.approx(fac / V, rel=1e-6)
    v = vir.cpu().numpy()
    assert v[0] == pytest.approx(2 * fac / V, rel=1e-6)
    assert v[2] == pytest.approx(2 * fac / V, rel=1e-6)
    assert v[5] == pytest.approx(2 * fac / V, rel=1e-6)
    assert v[1] == v[3] == v[4] == 0.0
    assert float(sums[3]) == pytest.approx(fac / V, rel=1e-6)
