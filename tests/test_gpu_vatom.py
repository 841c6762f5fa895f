"""Virtual atoms on the GPU (snb_vatom_*, snb_engine_set_virtual_atoms).

  * Coordinate refresh and force redistribution against the reference's own
    formulas (tests/golden/vatom_*.npz): positions within 2e-5 A, forces
    within relative RMS 1e-6; records given in shuffled order are placed in
    dependency levels (two for the mixed case);
  * a type-3 site whose direction has zero length is reported, not faulted;
  * a four-site water box in the engine: the force evaluation moves the M
    sites' forces onto the waters' atoms, within relative RMS 1e-5 of the
    FP64 oracle of the 4-site system with the same move; graph-replayed MD
    equals stream-launched MD bit for bit and keeps every M site where its
    formula puts it;
  * the reference's Amber TIP4P-Ew case: type-2 sites fitted to the first
    frame's extra points reproduce the extra points of all three frames
    (sander's positions) within 1e-3 A, and the engine's forces with the
    extra points' forces moved onto the waters keep each water's net force
    and torque against sander's within the reference test's tolerances.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _create(g, n, records):
    # the arrays stay referenced until the call returns
    ty, vi, fr, pa = (np.ascontiguousarray(records[0], np.int32),
                      np.ascontiguousarray(records[1], np.int32),
                      np.ascontiguousarray(records[2], np.int32),
                      np.ascontiguousarray(records[3], np.float32))
    h = ctypes.c_void_p()
    g.capi.check(g.capi.load().snb_vatom_create(
        n, len(ty), ty.ctypes.data, vi.ctypes.data, fr.ctypes.data, pa.ctypes.data,
        ctypes.byref(h)), "vatom_create")
    return h


@pytest.mark.parametrize("name", ["vatom_wat_nonortho.npz", "vatom_mixed.npz"])
def test_module_matches_reference_formulas(g, name):
    import torch
    from tests.test_cpu_vatom import load
    z, rcell, records = load(name)
    lib = g.capi.load()
    perm = np.random.default_rng(5).permutation(len(records[0]))
    h = _create(g, len(z["crd_in"]), tuple(np.asarray(r)[perm] for r in records))
    crd = g.dev(z["crd_in"].reshape(-1), np.float32)
    frc = g.dev(z["frc_in"].reshape(-1), np.float32)
    bnd = g.capi.boundary(z["cell"], rcell)
    lv = ctypes.c_int(0)
    try:
        g.capi.check(lib.snb_vatom_levels(h, ctypes.byref(lv)), "levels")
        g.capi.check(lib.snb_vatom_coordinate_refresh(h, g.ptr(crd), bnd, g.stream()),
                     "refresh")
        g.capi.check(lib.snb_vatom_force_redistribute(h, g.ptr(crd), bnd, g.ptr(frc),
                                                      g.stream()), "redistribute")
        bad = ctypes.c_int(0)
        g.capi.check(lib.snb_vatom_status(h, ctypes.byref(bad), g.stream()), "status")
        torch.cuda.synchronize()
    finally:
        lib.snb_vatom_destroy(h)
    assert bad.value == -1
    assert lv.value == (2 if "mixed" in name else 1)
    x = crd.cpu().numpy().reshape(-1, 3)
    f = frc.cpu().numpy().reshape(-1, 3).astype(np.float64)
    assert np.abs(x - z["crd_out"]).max() <= 2e-5
    want = z["frc_out"].astype(np.float64)
    assert np.linalg.norm(f - want) / np.linalg.norm(want) <= 1e-6
    assert not np.any(f[z["virtual_atom"]])


def test_zero_direction_is_reported(g):
    import torch
    lib = g.capi.load()
    crd = np.array([[1, 1, 1], [1, 1, 1], [2, 2, 2], [0, 0, 0]], np.float32)
    records = (np.array([3]), np.array([3]), np.array([[0, 1, 2]]),
               np.array([[0.5, 0.0]], np.float32))
    h = _create(g, 4, records)
    d = g.dev(crd.reshape(-1), np.float32)
    L = [10.0, 0, 10.0, 0, 0, 10.0]
    R = [0.1, 0, 0.1, 0, 0, 0.1]
    bad = ctypes.c_int(0)
    try:
        g.capi.check(lib.snb_vatom_coordinate_refresh(h, g.ptr(d), g.capi.boundary(L, R),
                                                      g.stream()), "refresh")
        g.capi.check(lib.snb_vatom_status(h, ctypes.byref(bad), g.stream()), "status")
        torch.cuda.synchronize()
    finally:
        lib.snb_vatom_destroy(h)
    assert bad.value == 0
    assert np.array_equal(d.cpu().numpy().reshape(-1, 3)[3], crd[0])


def test_cycles_and_unknown_types_are_refused(g):
    lib = g.capi.load()
    h = ctypes.c_void_p()
    cyc = (np.array([1, 1], np.int32), np.array([2, 3], np.int32),
           np.array([[3, 0, -1], [2, 0, -1]], np.int32), np.zeros((2, 2), np.float32))
    for recs in (cyc, (np.array([4], np.int32), np.array([2], np.int32),
                       np.array([[0, 1, -1]], np.int32), np.zeros((1, 2), np.float32))):
        ty, vi, fr, pa = recs
        rc = lib.snb_vatom_create(5, len(ty), ty.ctypes.data, vi.ctypes.data, fr.ctypes.data,
                                  pa.ctypes.data, ctypes.byref(h))
        assert rc != 0


def _engine_with_sites(g, s, records, cutoff=8.0):
    e = g.engine_create(s, cutoff)
    g.engine_set_water_bonded(e, s)
    v = _create(g, s.n, records)
    g.capi.check(g.capi.load().snb_engine_set_virtual_atoms(e, v), "set_virtual_atoms")
    return e, v


def test_engine_moves_site_forces(g, oracle):
    import torch
    from sponge_b200 import systems
    from tests import tip4p
    s, records = tip4p.tip4p_box(1000, seed=3)
    lib = g.capi.load()
    e, v = _engine_with_sites(g, s, records)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_vatom_destroy(v)
    beta = oracle.get_beta(8.0)
    rs, cols = oracle.nl_pairs_system(s, 8.0, 2.0)
    want = (oracle.direct_f64(s, 8.0, beta, rs, cols)["frc"] +
            oracle.excluded_f64(s, beta)["frc"] +
            oracle.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)["frc"])
    _, want, _ = oracle.vatom_f64(records, s.cell(), s.rcell(), s.crd, want)
    got = frc.cpu().numpy().reshape(-1, 3)
    assert g.rel_rms(got, want) <= 1e-5
    assert not np.any(got[records[1]])


def _md(g, s, records, steps, graph):
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    e, v = _engine_with_sites(g, s, records)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    m = s.mass.astype(np.float64)
    invm = g.dev(np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0).astype(np.float32))
    dt = 0.5e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
    try:
        with torch.cuda.stream(st):
            g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                            steps, ctypes.c_void_p(st.cuda_stream)), "md_steps")
        st.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_vatom_destroy(v)
    return crd.cpu().numpy().reshape(-1, 3), vel.cpu().numpy().reshape(-1, 3)


def test_engine_md_with_sites(g):
    from tests import tip4p
    s, records = tip4p.tip4p_box(1000, seed=3)
    a = _md(g, s, records, 120, graph=False)
    b = _md(g, s, records, 120, graph=True)
    assert np.isfinite(a[0]).all()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    x = a[0].astype(np.float64)
    o, h1, h2 = (records[2][:, k] for k in range(3))
    ab = float(records[3][0, 0])
    L = s.box
    d1 = x[h1] - x[o]
    d1 -= L * np.round(d1 / L)
    d2 = x[h2] - x[o]
    d2 -= L * np.round(d2 / L)
    want = x[o] + ab * d1 + ab * d2
    dm = x[records[1]] - want
    dm -= L * np.round(dm / L)
    assert np.abs(dm).max() <= 1e-4
    assert not np.any(a[1][records[1]])  # the sites carry no velocity


def _amber_sites(z, s):
    """Type-2 records for the waters' extra points (O, H1, H2, EP in residue
    order), a and b fitted to frame 0 by least squares."""
    lab, ptr = z["residue_label"], z["residue_pointer"]
    rows = []
    for k in range(len(lab)):
        if lab[k] != "WAT":
            continue
        o = int(ptr[k])
        rows.append((o, o + 1, o + 2, o + 3))
    rows = np.array(rows, np.int32)
    x = z["crd64"]
    A = np.stack([(x[rows[:, 1]] - x[rows[:, 0]]).reshape(-1),
                  (x[rows[:, 2]] - x[rows[:, 0]]).reshape(-1)], 1)
    rhs = (x[rows[:, 3]] - x[rows[:, 0]]).reshape(-1)
    (a, b), *_ = np.linalg.lstsq(A, rhs, rcond=None)
    m = len(rows)
    return (np.full(m, 2, np.int32), rows[:, 3].copy(), rows[:, :3].copy(),
            np.tile(np.array([a, b], np.float32), (m, 1))), rows


@pytest.mark.parametrize("iteration", [0, 1, 2])
def test_amber_extra_points(g, oracle, iteration):
    import torch
    from tests import test_cpu_amber_golden as am
    s0, z0 = am.load_amber(0)
    records, rows = _amber_sites(z0, s0)
    s, z = am.load_amber(iteration)
    lib = g.capi.load()
    # the sites placed from the frame's O and H atoms land on sander's extra points
    v = _create(g, s.n, records)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    try:
        g.capi.check(lib.snb_vatom_coordinate_refresh(v, g.ptr(crd), g.bnd(s), g.stream()),
                     "refresh")
        torch.cuda.synchronize()
    finally:
        lib.snb_vatom_destroy(v)
    x = crd.cpu().numpy().reshape(-1, 3)
    assert np.abs(x[rows[:, 3]] - z["crd"][rows[:, 3]]).max() <= 1e-3
    # engine forces with the extra points' forces moved onto the waters
    e = g.engine_create(s, 8.0)
    v = _create(g, s.n, records)
    g.capi.check(lib.snb_engine_set_virtual_atoms(e, v), "set_virtual_atoms")
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 0, 0, None,
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_vatom_destroy(v)
    got = frc.cpu().numpy().reshape(-1, 3).astype(np.float64)
    ref = np.asarray(z["amber_forces"], np.float64)
    assert not np.any(got[rows[:, 3]])
    xs = np.asarray(z["crd64"], np.float64)
    dF, dT = [], []
    for w in rows:
        r = xs[w] - xs[w[0]]
        dF.append(got[w].sum(0) - ref[w].sum(0))
        dT.append(np.cross(r, got[w]).sum(0) - np.cross(r, ref[w]).sum(0))
    dF, dT = np.array(dF), np.array(dT)
    print(f"\nframe {iteration}: water net force max |dF| {np.abs(dF).max():.4f}, "
          f"RMS {np.sqrt((dF ** 2).mean()):.4f}; torque max |dT| {np.abs(dT).max():.4f}")
    assert np.abs(dF).max() <= 0.10 and np.sqrt((dF ** 2).mean()) <= 0.03
    assert np.abs(dT).max() <= 0.10 and np.sqrt((dT ** 2).mean()) <= 0.03
