"""Accuracy against FP64 at the benchmarked sizes.

* The 99,639-atom water + NaCl box (33,333 waters, 90 Na+ / 90 Cl-,
  L = 99.90 A, cutoff 10 A, skin 2 A, PME 100^3) after 2,000 NVE steps of the
  engine from the lattice start with the velocities rescaled to 300 K every
  100 steps (the benchmark's own equilibration):
  - the neighbor pair set (sorted i < j pairs within cutoff + skin) is
    bit-exact against the oracle's FP32 criterion (neighbor_list.cpp:347-417);
  - the engine's forces are within relative RMS 1e-5 of the FP64 run of the
    same method on the same frame; every energy component (LJ, tail, direct
    Coulomb, excluded correction, self) within 1e-6 relative, the reciprocal
    energy within 2e-6 (it goes through a float FFT), the potential sum
    within 1e-6; the virial within 1e-6 of its largest component and the
    pressure's virial part within 0.05 bar.
* The largest member of each of the six PME grid sizes of the 256-box batch
  (20^3 ... 40^3, up to 5,962 atoms), run as one batch: every box within
  1e-5 of its own FP64 run, energies per component within 2e-6.
* The ~1M-atom soft-core box (333,333 waters, 0.15 M NaCl, 64-site solute,
  cutoff 10 A, PME 216^3) at lambda 0.5 with the solute's charges off, as the
  benchmark's windows run it: forces within 1e-5 of FP64 over all atoms.
"""

import copy
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CUTOFF = 10.0
SKIN = 2.0


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _equilibrated(g, s, steps, cutoff, soft=None):
    """Frame after `steps` engine NVE steps with 300 K rescaling every 100."""
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    e = g.engine_create(s, cutoff)
    g.engine_set_water_bonded(e, s)
    hs = None
    if soft is not None:
        sc, params = soft
        hs = g.soft_create(g.Box(s), sc, cutoff, params)
        g.capi.check(lib.snb_engine_set_soft_core(e, hs), "set_soft_core")
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev((1.0 / s.mass).astype(np.float32))
    mass = torch.from_numpy(s.mass.astype(np.float64)).cuda()
    dt = 0.5e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    try:
        for c0 in range(0, steps, 100):
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_md_steps_graph(
                    e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), c0,
                    min(100, steps - c0), sp), "md_steps")
                v = vel.view(s.n, 3).double()
                t_now = float((mass[:, None] * v * v).sum()) / (3.0 * s.n * systems.KB)
                vel.mul_(float(np.sqrt(300.0 / t_now)))
        st.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        if hs is not None:
            lib.snb_lj_soft_destroy(hs)
    out = copy.copy(s)
    out.crd = crd.cpu().numpy().reshape(-1, 3).copy()
    out.vel = vel.cpu().numpy().reshape(-1, 3).copy()
    assert np.isfinite(out.crd).all()
    return out


def _engine_force(g, s, cutoff, soft=None, energy=True):
    import torch
    lib = g.capi.load()
    e = g.engine_create(s, cutoff)
    hs = None
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        if soft is not None:
            sc, params = soft
            hs = g.soft_create(g.Box(s), sc, cutoff, params)
            g.capi.check(lib.snb_engine_set_soft_core(e, hs), "set_soft_core")
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, int(energy), 1,
                                          g.ptr(tot), g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        if hs is not None:
            lib.snb_lj_soft_destroy(hs)
    return frc.cpu().numpy().reshape(s.n, 3), tot.cpu().numpy()


@pytest.fixture(scope="module")
def frame_100k(g):
    from sponge_b200 import systems
    return _equilibrated(g, systems.config_100k(seed=0), 2000, CUTOFF)


@pytest.fixture(scope="module")
def oracle_rows_100k(oracle, frame_100k):
    return oracle.nl_pairs_system(frame_100k, CUTOFF, SKIN)


def test_100k_pair_set_is_bit_exact(g, frame_100k, oracle_rows_100k):
    lib = g.capi.load()
    box = g.Box(frame_100k)
    h = g.make_nl(box, CUTOFF, SKIN)
    try:
        g.nl_update(h, box)
        got = g.nl_pairs(h)
    finally:
        lib.snb_nl_destroy(h)
    want = g.csr_to_pairs(*oracle_rows_100k)
    assert len(want) > 30_000_000
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_100k_engine_matches_fp64(g, oracle, frame_100k, oracle_rows_100k):
    from oracle import accuracy
    s = frame_100k
    frc, tot = _engine_force(g, s, CUTOFF)
    ref = accuracy.reference_totals(oracle, s, CUTOFF, SKIN, rows=oracle_rows_100k)
    V = float(np.float32(s.box)) ** 3
    acc = accuracy.compare(frc, tot, ref, V)
    print("100k accuracy", acc)
    assert acc["force_rel_rms"] <= 1e-5
    rel = acc["energy_rel"]
    for k in ("lj", "lrc", "coul", "excl", "self", "potential"):
        assert rel[k] <= 1e-6, (k, rel[k])
    assert rel["recip"] <= 2e-6
    assert acc["virial_rel"] <= 1e-6
    assert acc["pressure_err_bar"] <= 0.05


def test_batch_largest_member_of_each_grid_size_matches_fp64(g, oracle):
    from oracle import accuracy
    from sponge_b200 import systems
    lib = g.capi.load()
    best = {}
    for seed in range(256):
        n, k = systems.batch_member_size(seed)
        if k not in best or n > best[k][0]:
            best[k] = (n, seed)
    assert sorted(best) == [20, 24, 28, 32, 36, 40]
    boxes = [systems.config_batch_member(seed) for _, seed in
             (best[k] for k in sorted(best))]
    assert max(b.n for b in boxes) > 5900
    h, c = g.batch_create(boxes, 8.0)
    import torch
    n = len(c["charge"])
    crd = g.dev(c["crd"])
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(h, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(h)
    fb = frc.cpu().numpy().reshape(n, 3)
    tb = tot.cpu().numpy()
    base, en_sum = 0, {}
    for s in boxes:
        want, en, _ = accuracy.reference_totals(oracle, s, 8.0)
        err = accuracy.force_rel_rms(fb[base:base + s.n], want)
        assert err <= 1e-5, (s.n, accuracy.grid_of(s), err)
        for k, v in en.items():
            en_sum[k] = en_sum.get(k, 0.0) + v
        base += s.n
    for k, idx in accuracy.TOTAL_SLOTS.items():
        assert abs(tb[idx] - en_sum[k]) <= 2e-6 * abs(en_sum[k]), k


def test_1m_soft_core_box_matches_fp64(g, oracle):
    from oracle import accuracy
    from sponge_b200 import systems
    s, sc = systems.soft_core_box(333333, n_solute=64, seed=0)
    s = copy.copy(s)
    # the benchmark's windows: solute charges off (state B charges)
    s.charge = (s.charge.astype(np.float64) + sc.charge_B_A).astype(np.float32)
    sc = copy.copy(sc)
    sc.charge_B_A = np.zeros_like(sc.charge_B_A)
    params = {"lambda_lj": 0.5, "soft_core_alpha": 0.5, "soft_core_powfer": 1.0,
              "soft_core_sigma": 3.0, "soft_core_sigma_min": 0.0}
    s = _equilibrated(g, s, 200, CUTOFF, soft=(sc, params))
    frc, _ = _engine_force(g, s, CUTOFF, soft=(sc, params), energy=False)
    want = accuracy.soft_reference_forces(oracle, s, sc, CUTOFF, 0.5, 0.5, 1.0, 3.0, 0.0,
                                          SKIN)
    err = accuracy.force_rel_rms(frc, want)
    print("1M soft-core force rel-RMS", err)
    assert s.n > 990_000
    assert accuracy.grid_of(s) == (216, 216, 216)
    assert err <= 1e-5
