"""The fused engine (one stream, one fixed-point accumulator, CUDA graph) on
the GPU: total nonbonded force and energies against the FP64 oracle, graph
replay against stream launches, and NVE energy conservation."""

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


def oracle_total(oracle, s, cutoff, skin=2.0):
    from sponge_b200 import systems
    beta = oracle.get_beta(cutoff)
    rs, cols = oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    e = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)
    V = float(np.float32(s.box)) ** 3
    lrc = oracle.lrc_factor(s, cutoff)
    frc = d["frc"] + e["frc"] + p["frc"]
    energies = dict(lj=d["lj_energy"].sum(), lrc=lrc / V, coul=d["coulomb_energy"].sum(),
                    excl=e["atom_energy"].sum(), recip=p["e_recip"], self=p["e_self"])
    vir = d["virial"].sum(0) + e["virial"].sum(0) + p["virial"]
    vir[[0, 2, 5]] += 2 * lrc / V
    return frc, energies, vir


@pytest.mark.parametrize("own_fft", [0, 1])
def test_engine_force_and_energy(g, oracle, box_9k, own_fft):
    """Forces, energies and the virial against FP64, with the PME
    convolution through cuFFT and through the library's own FFT passes."""
    import torch
    s = box_9k
    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    c = np.array([4, 0, 8, 256, 16, 0, 0, 0, own_fft], np.int32)
    g.capi.check(lib.snb_engine_set_launch_shapes(e, c.ctypes.data), "shapes")
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
    f_want, en, vir = oracle_total(oracle, s, 8.0)
    f_got = frc.cpu().numpy().reshape(s.n, 3)
    assert g.rel_rms(f_got, f_want) <= 1e-5
    t = tot.cpu().numpy()
    for k, idx in (("lj", 0), ("coul", 2), ("excl", 3), ("recip", 4), ("self", 5)):
        assert abs(t[idx] - en[k]) <= 2e-6 * abs(en[k]), k
    assert t[1] == pytest.approx(en["lrc"], rel=1e-6)
    total = sum(en.values())
    assert abs(t[7] - total) <= 1e-6 * sum(abs(v) for v in en.values())
    assert np.all(np.abs(t[8:14] - vir) <= 2e-6 * np.abs(vir).max())


def _run_md(g, s, steps, graph, cutoff=8.0):
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    e = g.engine_create(s, cutoff)
    g.engine_set_water_bonded(e, s)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev((1.0 / s.mass).astype(np.float32))
    dt = 0.5e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
        try:
            g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                            steps, ctypes.c_void_p(st.cuda_stream)), "md_steps")
            st.synchronize()
        finally:
            lib.snb_engine_destroy(e)
    return crd.cpu().numpy().reshape(-1, 3), vel.cpu().numpy().reshape(-1, 3)


def test_graph_replay_is_bitwise_identical(g, box_9k):
    c1, v1 = _run_md(g, box_9k, 40, graph=False)
    c2, v2 = _run_md(g, box_9k, 40, graph=True)
    assert np.array_equal(c1, c2)
    assert np.array_equal(v1, v2)


def test_nve_energy_is_conserved(g, oracle, small_box):
    """100 leap-frog steps at 0.5 fs from the unrelaxed lattice start: the
    total energy (kinetic from the mid-step velocity average) moves by less
    than 2% of the kinetic energy."""
    import copy
    import torch
    from sponge_b200 import systems
    s = copy.deepcopy(small_box)
    lib = g.capi.load()

    def energy(crd, vel):
        t = copy.deepcopy(s)
        t.crd = crd
        _, en, _ = oracle_total(oracle, t, 8.0)
        pot = sum(en.values())
        # bonded energy
        b = t.bonds
        d = crd[b[:, 0]] - crd[b[:, 1]]
        d -= np.round(d / t.box) * t.box
        r = np.linalg.norm(d.astype(np.float64), axis=1)
        eb = systems.BOND_K * ((r - systems.BOND_R0) ** 2).sum()
        a = t.angles
        u = crd[a[:, 0]] - crd[a[:, 1]]
        w = crd[a[:, 2]] - crd[a[:, 1]]
        u -= np.round(u / t.box) * t.box
        w -= np.round(w / t.box) * t.box
        c = (u * w).sum(1) / np.linalg.norm(u, axis=1) / np.linalg.norm(w, axis=1)
        ea = systems.ANGLE_K * ((np.arccos(np.clip(c, -1, 1)) - systems.ANGLE_T0) ** 2).sum()
        ke = 0.5 * (t.mass[:, None] * vel.astype(np.float64) ** 2).sum()
        return pot + eb + ea, ke

    e0p, _ = energy(s.crd, s.vel)
    c, v = _run_md(g, s, 100, graph=True)
    s2 = copy.deepcopy(s)
    s2.crd, s2.vel = c, v
    c2, v2 = _run_md(g, s2, 1, graph=False)
    p1, k1 = energy(c, (v + v2) / 2)
    _, k0 = energy(s.crd, s.vel)
    e_start = e0p + k0
    e_end = p1 + k1
    assert np.isfinite(e_end)
    assert abs(e_end - e_start) <= 2e-2 * k0


def test_autotune_keeps_results_bitwise(g, box_9k):
    """Launch shapes change only the schedule: the fixed-point forces after
    tuning equal those before, bit for bit, and crd / vel come back intact."""
    import torch
    from sponge_b200 import systems
    s = box_9k
    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    g.engine_set_water_bonded(e, s)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev((1.0 / s.mass).astype(np.float32))
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    dt = 0.5e-3 * systems.TIME_CONVERSION

    def force():
        f = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(f), 0, 0, 0, None, sp),
                         "engine_force")
        st.synchronize()
        return f.cpu().numpy()

    try:
        f0 = force()
        c0, v0 = crd.cpu().numpy(), vel.cpu().numpy()
        choice = np.zeros(9, np.int32)
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_autotune(e, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                 ctypes.c_float(dt), 3, choice.ctypes.data,
                                                 sp), "autotune")
        st.synchronize()
        assert np.array_equal(crd.cpu().numpy(), c0)
        assert np.array_equal(vel.cpu().numpy(), v0)
        assert choice[0] in (2, 4, 8) and choice[1] in (0, 2, 3)
        assert choice[2] in (4, 8, 16) and choice[3] in (128, 256, 512)
        assert choice[4] in (4, 8, 16)
        assert (choice[5], choice[6]) in ((8, 1), (8, 2), (8, 4), (0, 0))
        assert choice[7] in (0, 1) and choice[8] in (0, 1)
        f1 = force()
        assert np.array_equal(f0, f1)
        with torch.cuda.stream(st):  # graph steps with the tuned shapes
            g.capi.check(lib.snb_engine_md_steps_graph(e, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                       ctypes.c_float(dt), 0, 20, sp), "md")
        st.synchronize()
        assert np.isfinite(crd.cpu().numpy()).all()
    finally:
        lib.snb_engine_destroy(e)


@pytest.mark.parametrize("shape", [(8, 1), (8, 4), (16, 4), (16, 8), (0, 0)])
def test_launch_shapes_keep_forces_bitwise(g, box_9k, shape):
    """Every spread shape (tiles, or int64 global atomics), every
    rows-in-flight choice of the pair kernel and its hit stash give the same
    fixed-point forces, bit for bit, as the tile spread of edge 8 with 2
    warps, 8 rows per block and no stash, through graph steps too."""
    import torch
    from sponge_b200 import systems
    s = box_9k
    lib = g.capi.load()
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    dt = ctypes.c_float(0.5e-3 * systems.TIME_CONVERSION)
    out = []
    for choice in ([4, 0, 8, 256, 8, 8, 2, 0, 0], [8, 0, 16, 128, 16, *shape, 0, 0],
                   [2, 2, 4, 512, 4, *shape, 1, 0], [4, 0, 8, 256, 8, *shape, 1, 0],
                   [8, 3, 8, 256, 16, *shape, 1, 0]):
        e = g.engine_create(s, 8.0)
        g.engine_set_water_bonded(e, s)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        f = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
        c = np.array(choice, np.int32)
        try:
            g.capi.check(lib.snb_engine_set_launch_shapes(e, c.ctypes.data), "shapes")
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(f), 0, 0, 0, None, sp),
                             "engine_force")
                g.capi.check(lib.snb_engine_md_steps_graph(e, g.ptr(crd), g.ptr(vel),
                                                           g.ptr(invm), dt, 1, 10, sp), "md")
            st.synchronize()
            out.append((f.cpu().numpy(), crd.cpu().numpy(), vel.cpu().numpy()))
        finally:
            lib.snb_engine_destroy(e)
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a, b)


def test_launch_shapes_refuse_values_outside_the_tuned_set(g, box_9k):
    lib = g.capi.load()
    e = g.engine_create(box_9k, 8.0)
    try:
        for bad in ([3, 0, 8, 256, 8, 8, 2, 0, 0], [4, 0, 8, 256, 6, 8, 2, 0, 0],
                    [4, 0, 8, 256, 8, 16, 2, 0, 0], [4, 0, 8, 256, 8, 12, 4, 0, 0],
                    [4, 0, 8, 256, 8, 8, 2, 2, 0], [4, 0, 8, 256, 8, 8, 2, 0, 2]):
            c = np.array(bad, np.int32)
            assert lib.snb_engine_set_launch_shapes(e, c.ctypes.data) != 0
    finally:
        lib.snb_engine_destroy(e)


@pytest.mark.parametrize("waters", [216, 520, 1400])
def test_own_fft_matches_cufft(g, waters):
    """The library's own FFT passes (grids 20^3 = 4 5, 28^3 = 4 7, 36^3 =
    4 3 3) against cuFFT through the whole engine force: forces, reciprocal
    energy and virial agree to float rounding."""
    import torch
    from sponge_b200 import systems
    s = systems.water_box(waters, seed=3)
    lib = g.capi.load()
    out = []
    for own in (0, 1):
        e = g.engine_create(s, 8.0)
        c = np.array([4, 0, 8, 256, 16, 0, 0, 0, own], np.int32)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
        tot = torch.zeros(16, dtype=torch.float64, device="cuda")
        try:
            g.capi.check(lib.snb_engine_set_launch_shapes(e, c.ctypes.data), "shapes")
            g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                              g.stream()), "engine_force")
            torch.cuda.synchronize()
        finally:
            lib.snb_engine_destroy(e)
        out.append((frc.cpu().numpy(), tot.cpu().numpy()))
    (f0, t0), (f1, t1) = out
    assert g.rel_rms(f1, f0) <= 1e-6
    assert abs(t1[4] - t0[4]) <= 1e-6 * abs(t0[4])
    assert np.all(np.abs(t1[8:14] - t0[8:14]) <= 1e-6 * np.abs(t0[8:14]).max())
