"""A batch of independent boxes in one engine (snb_batch_create): every box's
forces against the FP64 oracle run of that box alone, and against the same
box run through the single-box engine; energies summed over the boxes; NVE
steps of the whole batch against single-box runs.

Tolerances: forces relative RMS <= 1e-5 against FP64 per box; batch vs
single-box engine <= 1e-6 relative RMS (same kernels and fixed-point sums;
only the batched FFT plans differ); energies per component within 2e-6 of
the component's magnitude, as for one box.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CUTOFF = 8.0


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.fixture(scope="module")
def boxes():
    """Five boxes of 200-700 waters (grids 20^3-28^3; the two smallest have
    3 cells per axis, the index ownership rule, the rest 5 and more)."""
    from sponge_b200 import systems
    return [systems.water_box(nw, seed=s, ion_pairs=None)
            for s, nw in enumerate([200, 450, 700, 260, 520])]


def _force(g, h, crd, n, energy=True):
    import torch
    lib = g.capi.load()
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    g.capi.check(lib.snb_engine_force(h, g.ptr(crd), g.ptr(frc), 0, int(energy), 1,
                                      g.ptr(tot), g.stream()), "engine_force")
    torch.cuda.synchronize()
    return frc.cpu().numpy().reshape(n, 3), tot.cpu().numpy()


def test_batch_forces_match_fp64_and_single_box(g, oracle, boxes):
    from sponge_b200 import systems
    lib = g.capi.load()
    h, c = g.batch_create(boxes, CUTOFF)
    try:
        crd = g.dev(c["crd"])
        fb, tb = _force(g, h, crd, len(c["charge"]))
    finally:
        lib.snb_engine_destroy(h)
    from tests.test_gpu_engine import oracle_total
    base = 0
    en_sum = {}
    for s in boxes:
        got = fb[base:base + s.n]
        want, en, _ = oracle_total(oracle, s, CUTOFF)
        assert g.rel_rms(got, want) <= 1e-5
        for k, v in en.items():
            en_sum[k] = en_sum.get(k, 0.0) + v
        # the same box alone through the single-box engine
        hs = g.engine_create(s, CUTOFF)
        try:
            fs, _ = _force(g, hs, g.dev(s.crd.reshape(-1), np.float32), s.n)
        finally:
            lib.snb_engine_destroy(hs)
        assert g.rel_rms(got, fs) <= 1e-6
        base += s.n
    for k, idx in (("lj", 0), ("coul", 2), ("excl", 3), ("recip", 4), ("self", 5)):
        assert abs(tb[idx] - en_sum[k]) <= 2e-6 * abs(en_sum[k]), k
    assert tb[1] == pytest.approx(en_sum["lrc"], rel=1e-6)
    assert abs(tb[7] - sum(en_sum.values())) <= 1e-6 * sum(abs(v) for v in en_sum.values())


def _export_pairs(g, h):
    """The engine's pair set as sorted (lo, hi) rows, and its kept total."""
    import torch
    lib = g.capi.load()
    cnt = ctypes.c_longlong(0)
    g.capi.check(lib.snb_engine_stats(h, None, ctypes.byref(cnt), g.stream()), "stats")
    n = cnt.value
    pi = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    pj = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    got = ctypes.c_longlong(0)
    g.capi.check(lib.snb_engine_export_pairs(h, g.ptr(pi), g.ptr(pj), n, ctypes.byref(got),
                                             g.stream()), "engine_export_pairs")
    p = np.stack([pi[:got.value].cpu().numpy(), pj[:got.value].cpu().numpy()], 1)
    return p.astype(np.int64), n, got.value


def _pairs_within(crd, box, cutoff, base, excluded):
    """(lo, hi) global ids of one box's pairs closer than cutoff (minimum
    image), excluded pairs left out."""
    d = crd[:, None, :] - crd[None, :, :]
    d -= box * np.round(d / box)
    r2 = (d * d).sum(-1)
    i, j = np.nonzero(np.triu(r2 < cutoff * cutoff, 1))
    keep = [(a, b) not in excluded for a, b in zip(i + base, j + base)]
    return np.stack([i + base, j + base], 1)[np.array(keep, bool)]


def test_batch_md_matches_single_boxes(g, boxes):
    """100 graph-replayed NVE steps of the batch stay with single-box runs of
    the same boxes (both fixed-point; coordinates agree to 1e-3 A).  Each box
    rebuilds its own list when its own atoms moved past the skin allowance;
    after the steps every box's list still holds every pair within the
    cutoff, and the kept pair total equals the exported list's size."""
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    dt = 0.5e-3 * systems.TIME_CONVERSION
    steps = 100
    h, c = g.batch_create(boxes, CUTOFF)
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    try:
        nb = np.concatenate([s.bonds + off for s, off in
                             zip(boxes, np.cumsum([0] + [s.n for s in boxes])[:-1])])
        na = np.concatenate([s.angles + off for s, off in
                             zip(boxes, np.cumsum([0] + [s.n for s in boxes])[:-1])])
        bonded = type("B", (), {})()
        bonded.bonds, bonded.angles = nb.astype(np.int32), na.astype(np.int32)
        g.engine_set_water_bonded(h, bonded)
        crd, vel = g.dev(c["crd"]), g.dev(c["vel"])
        invm = g.dev((1.0 / c["mass"]).astype(np.float32))
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_md_steps_graph(h, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                       ctypes.c_float(dt), 0, steps, sp),
                         "batch md")
        st.synchronize()
        cb = crd.cpu().numpy().reshape(-1, 3)
        listed, total, exported = _export_pairs(g, h)
    finally:
        lib.snb_engine_destroy(h)
    assert total == exported
    excluded = set()
    for a in range(len(c["excl_numbers"])):
        for k in range(c["excl_numbers"][a]):
            b = int(c["excl_list"][c["excl_start"][a] + k])
            excluded.add((min(a, b), max(a, b)))
    listed = set(map(tuple, listed.tolist()))
    base = 0
    for s in boxes:
        need = _pairs_within(cb[base:base + s.n].astype(np.float64), float(s.box), CUTOFF,
                             base, excluded)
        missing = [p for p in map(tuple, need.tolist()) if p not in listed]
        assert not missing, f"box at atom {base}: {len(missing)} pairs within the cutoff unlisted"
        base += s.n
    base = 0
    for s in boxes:
        hs = g.engine_create(s, CUTOFF)
        try:
            g.engine_set_water_bonded(hs, s)
            crd = g.dev(s.crd.reshape(-1), np.float32)
            vel = g.dev(s.vel.reshape(-1), np.float32)
            invm = g.dev((1.0 / s.mass).astype(np.float32))
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_md_steps_graph(hs, g.ptr(crd), g.ptr(vel),
                                                           g.ptr(invm), ctypes.c_float(dt),
                                                           0, steps, sp), "single md")
            st.synchronize()
            cs = crd.cpu().numpy().reshape(-1, 3)
        finally:
            lib.snb_engine_destroy(hs)
        assert np.abs(cb[base:base + s.n] - cs).max() < 1e-3
        base += s.n


def test_batch_rejects_cross_system_exclusion(g, boxes):
    lib = g.capi.load()
    c = g.batch_concat(boxes[:2])
    el = c["excl_list"].copy()
    el[0] = boxes[0].n + 1  # points into the second box
    import ctypes as ct
    s0 = boxes[0]
    A = np.ascontiguousarray(s0.lj_A, np.float32)
    B = np.ascontiguousarray(s0.lj_B, np.float32)
    h = ct.c_void_p()
    o = g.capi.options(cutoff=CUTOFF)
    rc = lib.snb_batch_create(ct.byref(o), 2, c["counts"].ctypes.data, c["boxes"].ctypes.data,
                              s0.n_types, c["lj_type"].ctypes.data, A.ctypes.data,
                              B.ctypes.data, c["charge"].ctypes.data,
                              c["excl_start"].ctypes.data, c["excl_numbers"].ctypes.data,
                              el.ctypes.data, c["n_excl"], ct.byref(h))
    assert rc == 1
    assert b"between two systems" in lib.snb_last_error()


def test_batch_own_fft_matches_cufft(g, boxes):
    """The batch's own FFT passes (one launch per pass over the five boxes'
    grids 20^3-28^3, lines in registers) against the batched cuFFT plans
    through the whole batch force: forces, reciprocal energy and virial agree
    to float rounding, and no cuFFT kernel is left in the step graph."""
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    out = []
    for own in (0, 1):
        h, c = g.batch_create(boxes, CUTOFF)
        n = len(c["charge"])
        try:
            shapes = np.zeros(9, np.int32)
            crd = g.dev(c["crd"])
            vel = g.dev(np.zeros_like(c["crd"]))
            invm = g.dev((1.0 / c["mass"]).astype(np.float32))
            st = torch.cuda.Stream()
            sp = ctypes.c_void_p(st.cuda_stream)
            # the engine's own shapes first, then the FFT switched
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_autotune(h, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                     ctypes.c_float(0.0), 1,
                                                     shapes.ctypes.data, sp), "autotune")
            st.synchronize()
            shapes[8] = own
            g.capi.check(lib.snb_engine_set_launch_shapes(h, shapes.ctypes.data), "shapes")
            frc, tot = _force(g, h, crd, n)
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_md_steps_graph(
                    h, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                    ctypes.c_float(0.5e-3 * systems.TIME_CONVERSION), 0, 2, sp), "md")
            st.synchronize()
            kn, libk, bodyk = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
            g.capi.check(lib.snb_engine_graph_info(h, ctypes.byref(kn), ctypes.byref(libk),
                                                   ctypes.byref(bodyk), sp), "graph_info")
        finally:
            lib.snb_engine_destroy(h)
        out.append((frc, tot, libk.value))
    (f0, t0, l0), (f1, t1, l1) = out
    assert l0 > 0 and l1 == 0
    assert g.rel_rms(f1, f0) <= 1e-6
    assert abs(t1[4] - t0[4]) <= 1e-6 * abs(t0[4])
    assert np.all(np.abs(t1[8:14] - t0[8:14]) <= 1e-6 * np.abs(t0[8:14]).max())


def test_batch_own_fft_every_class_of_length(g):
    """Grids of 24, 32, 36, 48, 56 and 64 points per axis in one batch (the
    register passes compiled for the longest axis, 64): the whole batch
    force with the own passes against the batched cuFFT plans."""
    import torch
    from sponge_b200 import systems
    boxes = [systems.water_box(nw, seed=k, ion_pairs=None)
             for k, nw in enumerate([381, 948, 1373, 3361, 5411, 8161])]
    assert sorted({systems.fft_size(b.box) for b in boxes}) == [24, 32, 36, 48, 56, 64]
    lib = g.capi.load()
    out = []
    for own in (0, 1):
        h, c = g.batch_create(boxes, CUTOFF)
        try:
            shapes = np.array([2, 0, 16, 128, 16, 8, 2, 0, own], np.int32)
            g.capi.check(lib.snb_engine_set_launch_shapes(h, shapes.ctypes.data), "shapes")
            out.append(_force(g, h, g.dev(c["crd"]), len(c["charge"])))
        finally:
            lib.snb_engine_destroy(h)
    (f0, t0), (f1, t1) = out
    assert g.rel_rms(f1, f0) <= 1e-6
    assert abs(t1[4] - t0[4]) <= 1e-6 * abs(t0[4])
    assert np.all(np.abs(t1[8:14] - t0[8:14]) <= 1e-6 * np.abs(t0[8:14]).max())


def test_batch_force_only_own_fft_matches_cufft(g, boxes):
    """Force-only calls of a batch (the own passes multiply by the table of
    the influence function and form no sums) against the batched cuFFT
    plans."""
    import torch
    lib = g.capi.load()
    out = []
    for own in (0, 1):
        h, c = g.batch_create(boxes, CUTOFF)
        n = len(c["charge"])
        try:
            shapes = np.array([2, 0, 16, 128, 16, 8, 2, 0, own], np.int32)
            g.capi.check(lib.snb_engine_set_launch_shapes(h, shapes.ctypes.data), "shapes")
            crd = g.dev(c["crd"])
            frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
            tot = torch.zeros(16, dtype=torch.float64, device="cuda")
            g.capi.check(lib.snb_engine_force(h, g.ptr(crd), g.ptr(frc), 0, 0, 0,
                                              g.ptr(tot), g.stream()), "engine_force")
            torch.cuda.synchronize()
            out.append(frc.cpu().numpy())
        finally:
            lib.snb_engine_destroy(h)
    assert g.rel_rms(out[1], out[0]) <= 1e-6
