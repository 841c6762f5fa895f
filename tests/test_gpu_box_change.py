"""A barostat's box change on the GPU: the neighbor list redrawn for the new
box, PME's Update_Box at the old grid size, and the engine's box update.

Against the reference (tests/golden/boxchange_*.npz: the reference
initialised on box0, then box and coordinates scaled; made by
tests/golden/make_golden.py) and against the FP64 oracle of the new box:
  pair set: bit-exact;
  forces: relative RMS <= 1e-5 against FP64;
  energies and virial: <= 2e-6 relative (the PME reciprocal energy goes
  through a float FFT), the virial against the reference initialised at the
  new box (its Update_Box forms the virial factor with the opposite sign of
  the m^2 term, see tests/test_cpu_oracle.py).
"""

import ctypes
import copy
import hashlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.fixture(scope="module")
def case():
    from tests.test_cpu_oracle import load_case
    s1, z = load_case("boxchange_water343_x103.npz")
    s0 = copy.deepcopy(s1)
    s0.crd = z["crd0"]
    s0.box = float(z["box0"])
    return s0, s1, z


def _fp64_total(oracle, s, cutoff, grid, skin=2.0):
    beta = oracle.get_beta(cutoff)
    rs, cols = oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    e = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, grid, beta)
    V = float(np.float32(s.box)) ** 3
    lrc = oracle.lrc_factor(s, cutoff)
    energies = dict(lj=d["lj_energy"].sum(), lrc=lrc / V, coul=d["coulomb_energy"].sum(),
                    excl=e["atom_energy"].sum(), recip=p["e_recip"], self=p["e_self"])
    vir = d["virial"].sum(0) + e["virial"].sum(0) + p["virial"]
    vir[[0, 2, 5]] += 2 * lrc / V
    return d["frc"] + e["frc"] + p["frc"], energies, vir


def test_nl_box_change_pair_set_matches_reference(g, case):
    s0, s1, z = case
    b0, b1 = g.Box(s0), g.Box(s1)
    h = g.make_nl(b0, float(z["cutoff"]), float(z["skin"]))
    lib = g.capi.load()
    try:
        g.nl_update(h, b0)
        # conditional update: the new box alone forces the rebuild
        g.nl_update(h, b1, forced=0, step=1)
        pairs = g.nl_pairs(h)
    finally:
        lib.snb_nl_destroy(h)
    digest = hashlib.sha256(np.ascontiguousarray(pairs, np.int32).tobytes()).hexdigest()
    assert len(pairs) == int(z["nl_pair_total"])
    assert digest == str(z["nl_pair_sha256"])


def test_pme_update_box_matches_reference_and_fp64(g, oracle, case):
    s0, s1, z = case
    b0, b1 = g.Box(s0), g.Box(s1)
    lib = g.capi.load()
    h, beta, grid = g.pme_create(b0, float(z["cutoff"]))
    try:
        assert grid == tuple(z["grid"])
        g.pme_reciprocal(h, b0)
        rate = np.zeros(6, np.float32)
        g.capi.check(lib.snb_pme_update_box(h, b1.b, rate.ctypes.data, ctypes.c_float(0.0)),
                     "pme_update_box")
        got = g.pme_reciprocal(h, b1)
    finally:
        lib.snb_pme_destroy(h)
    want = oracle.pme_f64(s1, grid, beta)
    assert g.rel_rms(got["frc"], want["frc"]) <= 1e-5
    assert g.rel_rms(got["frc"], z["pme_frc"]) <= 2e-5
    assert got["e_recip"] == pytest.approx(want["e_recip"], rel=2e-6)
    assert got["e_self"] == pytest.approx(want["e_self"], rel=1e-6)
    assert np.allclose(got["virial64"], want["virial"], rtol=2e-6,
                       atol=2e-6 * np.abs(want["virial"]).max())
    assert np.allclose(got["virial64"], z["pme_virial_fresh"], rtol=2e-5,
                       atol=2e-5 * np.abs(want["virial"]).max())


def test_engine_update_box_matches_fp64(g, oracle, box_9k):
    """The 9,000-atom box scaled by 1.02 after a first evaluation (the cell
    grid goes from 8 to 9 cells per axis): engine forces, energies and
    virial against FP64 of the new box at the old PME grid; then 20 graph
    steps in the new box stay finite."""
    import torch
    from sponge_b200 import systems
    s0 = box_9k
    s1 = copy.deepcopy(s0)
    s1.box = float(np.float32(s0.box * 1.02))
    s1.crd = (s0.crd.astype(np.float64) * 1.02).astype(np.float32)
    lib = g.capi.load()
    e = g.engine_create(s0, 8.0)
    g.engine_set_water_bonded(e, s0)
    crd0 = g.dev(s0.crd.reshape(-1), np.float32)
    crd1 = g.dev(s1.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s0.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    K = systems.fft_size(s0.box)
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd0), g.ptr(frc), 0, 0, 0, None,
                                          g.stream()), "engine_force")
        g.capi.check(lib.snb_engine_update_box(e, g.bnd(s1)), "engine_update_box")
        frc.zero_()
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd1), g.ptr(frc), 1, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
        vel = g.dev(s1.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s1.mass).astype(np.float32))
        st = torch.cuda.Stream()
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_md_steps_graph(
                e, g.ptr(crd1), g.ptr(vel), g.ptr(invm),
                ctypes.c_float(0.5e-3 * systems.TIME_CONVERSION), 2, 20,
                ctypes.c_void_p(st.cuda_stream)), "md_steps")
        st.synchronize()
        assert np.isfinite(crd1.cpu().numpy()).all()
    finally:
        lib.snb_engine_destroy(e)
    # FP64 of the new box with the grid of the old one (Update_Box keeps it)
    f_want, en, vir = _fp64_total(oracle, s1, 8.0, (K, K, K))
    assert g.rel_rms(frc.cpu().numpy().reshape(-1, 3), f_want) <= 1e-5
    t = tot.cpu().numpy()
    for k, idx in (("lj", 0), ("coul", 2), ("excl", 3), ("recip", 4), ("self", 5)):
        assert abs(t[idx] - en[k]) <= 2e-6 * abs(en[k]), k
    assert t[1] == pytest.approx(en["lrc"], rel=1e-6)
    assert np.all(np.abs(t[8:14] - vir) <= 2e-6 * np.abs(vir).max())
