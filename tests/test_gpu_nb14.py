"""1-4 terms on the GPU (snb_nb14_* and snb_engine_set_nb14) against the
golden vectors of the reference's own NON_BOND_14 (tests/golden/
make_nb14_golden.py) and the FP64 oracle.

Cases: the 41 1-4 pairs of the Amber alanine dipeptide case and 600 seeded
pairs of a 300-water box (pairs across the periodic boundary, uncharged
atoms).  Tolerances: forces, per-atom energies and virials 1e-5 relative RMS
against FP64; the two energy sums 1e-6 relative; the engine's totals slot 6
(the 1-4 energy) 1e-6 relative; graph-replayed steps bit-equal to
stream-launched ones."""

import ctypes

import numpy as np
import pytest

from tests import test_cpu_nb14 as cn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def nb14_create(g, n, z):
    lib = g.capi.load()
    h = ctypes.c_void_p()
    a = [np.ascontiguousarray(z[k], dt) for k, dt in
         (("atom_a", np.int32), ("atom_b", np.int32), ("A", np.float32), ("B", np.float32),
          ("cf", np.float32))]
    g.capi.check(lib.snb_nb14_create(n, len(a[0]), *[x.ctypes.data for x in a],
                                     ctypes.byref(h)), "nb14_create")
    return h


@pytest.mark.parametrize("name", cn.CASES)
def test_nb14_module_matches_reference_and_fp64(g, oracle, name):
    import torch
    box, z = cn.load(name)
    lib = g.capi.load()
    n = box.n
    h = nb14_create(g, n, z)
    crd = g.dev(box.crd.reshape(-1), np.float32)
    q = g.dev(box.charge, np.float32)
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    lj, ee = ctypes.c_float(0), ctypes.c_float(0)
    try:
        g.capi.check(lib.snb_nb14_force(h, g.ptr(crd), g.ptr(q),
                                        g.capi.boundary(box.cell(), box.rcell()), g.ptr(frc),
                                        1, g.ptr(ae), 1, g.ptr(vir), g.stream()), "nb14_force")
        g.capi.check(lib.snb_nb14_energy_sums(h, ctypes.byref(lj), ctypes.byref(ee),
                                              g.stream()), "nb14_sums")
        torch.cuda.synchronize()
    finally:
        lib.snb_nb14_destroy(h)
    o = oracle.nb14_f64(box, z["atom_a"], z["atom_b"], z["A"], z["B"], z["cf"])
    f = frc.cpu().numpy().reshape(n, 3)
    assert g.rel_rms(f, o["frc"]) <= 1e-5
    assert g.rel_rms(ae.cpu().numpy(), o["atom_energy"]) <= 1e-5
    assert g.rel_rms(vir.cpu().numpy().reshape(n, 6), o["virial"]) <= 1e-5
    assert abs(ee.value - o["ee"]) <= 1e-6 * abs(o["ee"])
    assert abs(lj.value - o["lj"]) <= 1e-6 * (abs(o["lj"]) + abs(o["ee"]))
    # and against the reference's own FP32 output
    assert g.rel_rms(f, z["ref_frc"]) <= 1e-5
    assert abs(ee.value - float(z["ref_ee"])) <= 1e-6 * abs(float(z["ref_ee"]))


def test_engine_with_nb14_on_amber_case(g, oracle):
    """Engine forces with the 1-4 terms = FP64 nonbonded + FP64 1-4 terms;
    totals slot 6 = the 1-4 energy and slot 7 the sum of all."""
    import torch
    from tests import test_cpu_amber_golden as am
    s, _ = am.load_amber(0)
    box, z = cn.load("nb14_alanine_dipeptide.npz")
    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    h = nb14_create(g, s.n, z)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_set_nb14(e, h), "set_nb14")
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_nb14_destroy(h)
    f_nb, e_nb = am.nonbonded_f64(oracle, s)
    o = oracle.nb14_f64(box, z["atom_a"], z["atom_b"], z["A"], z["B"], z["cf"])
    got = frc.cpu().numpy().reshape(-1, 3)
    assert g.rel_rms(got, f_nb + o["frc"]) <= 1e-5
    t = tot.cpu().numpy()
    e14 = o["lj"] + o["ee"]
    assert abs(t[6] - e14) <= 1e-6 * (abs(o["lj"]) + abs(o["ee"]))
    assert abs(t[7] - (e_nb + e14)) <= 1e-5 * abs(e_nb)


def test_engine_nb14_graph_matches_stream(g):
    """20 NVE steps of a 300-water box with 600 1-4 pairs: graph-replayed
    steps equal stream-launched ones bit for bit."""
    import torch
    from sponge_b200 import systems
    s = systems.water_box(300, seed=3)
    _, z = cn.load("nb14_water_box.npz")
    lib = g.capi.load()
    dt = 0.5e-3 * systems.TIME_CONVERSION
    out = []
    for graph in (False, True):
        e = g.engine_create(s, 8.0)
        g.engine_set_water_bonded(e, s)
        h = nb14_create(g, s.n, z)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        st = torch.cuda.Stream()
        try:
            g.capi.check(lib.snb_engine_set_nb14(e, h), "set_nb14")
            fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
            with torch.cuda.stream(st):
                g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                                20, ctypes.c_void_p(st.cuda_stream)), "md")
            st.synchronize()
        finally:
            lib.snb_engine_destroy(e)
            lib.snb_nb14_destroy(h)
        out.append(crd.cpu().numpy())
    assert np.isfinite(out[1]).all()
    assert np.array_equal(out[0], out[1])
