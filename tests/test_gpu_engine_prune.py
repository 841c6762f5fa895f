"""Pruned rows in the engine (snb_engine_set_prune_margin): MD with pruning
equals MD without it bit for bit, through graph replay and stream launches,
with flexible and with rigid (SETTLE) water, and a force call on coordinates
from outside the MD loop scans the full rows.

Why bit for bit: a pair outside cutoff + margin at a prune pass stays outside
the cutoff until an atom has moved half the margin, which forces the next
pass; the pairs within the cutoff are thus the same on every step, in the
same order within each row, and the fixed-point sums do not depend on order.
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


def _md(g, s, steps, graph, margin, cutoff=8.0, dt_fs=0.5, settle=None):
    """crd, vel after `steps` NVE steps, and the prune passes taken."""
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    e = g.engine_create(s, cutoff)
    if settle is None:
        g.engine_set_water_bonded(e, s)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev((1.0 / s.mass).astype(np.float32))
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    passes = ctypes.c_int(0)
    h = None
    try:
        g.capi.check(lib.snb_engine_set_prune_margin(e, ctypes.c_float(margin)), "prune margin")
        if settle is not None:
            h = settle()
            g.capi.check(lib.snb_engine_set_settle(e, h), "set_settle")
        fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
        dt = dt_fs * 1e-3 * systems.TIME_CONVERSION
        with torch.cuda.stream(st):
            g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                            steps, sp), "md_steps")
        st.synchronize()
        g.capi.check(lib.snb_engine_prune_passes(e, ctypes.byref(passes), None, sp), "passes")
    finally:
        lib.snb_engine_destroy(e)
        if h is not None:
            lib.snb_settle_destroy(h)
    return crd.cpu().numpy().reshape(-1, 3), vel.cpu().numpy().reshape(-1, 3), passes.value


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("margin", [0.3, 1.0])
def test_pruned_md_is_bitwise_unchanged(g, box_9k, graph, margin):
    steps = 120
    c0, v0, p0 = _md(g, box_9k, steps, graph, 0.0)
    c1, v1, p1 = _md(g, box_9k, steps, graph, margin)
    assert p0 == 0
    # the first step and every list rebuild prune; a small margin also
    # prunes between rebuilds
    assert p1 >= 2
    if margin == 0.3:
        assert p1 >= 8
    assert p1 < steps
    assert np.array_equal(c0, c1)
    assert np.array_equal(v0, v1)


def test_pruned_md_with_settle_is_bitwise_unchanged(g):
    """Rigid water at 2 fs: the check runs on the constrained positions."""
    from sponge_b200 import systems
    from tests.golden import make_settle_golden as mg
    from tests.test_gpu_settle import settle_create
    s = systems.water_box(300, seed=21)
    o = np.arange(0, s.n, 3)
    ai = np.concatenate([o, o, o + 1]).astype(np.int32)
    aj = np.concatenate([o + 1, o + 2, o + 2]).astype(np.int32)
    r0 = np.concatenate([np.full(len(o), mg.R_OH), np.full(len(o), mg.R_OH),
                         np.full(len(o), mg.R_HH)]).astype(np.float32)
    mk = lambda: settle_create(g, s.n, ai, aj, r0, s.mass)  # noqa: E731
    c0, v0, _ = _md(g, s, 100, True, 0.0, dt_fs=2.0, settle=mk)
    c1, v1, p1 = _md(g, s, 100, True, 0.4, dt_fs=2.0, settle=mk)
    assert p1 >= 8
    assert np.array_equal(c0, c1)
    assert np.array_equal(v0, v1)


def test_force_call_scans_full_rows(g, box_9k):
    """After pruned MD steps, forces on coordinates moved by up to 0.45 A
    (beyond half the 0.3 A margin) equal those of an engine without
    pruning."""
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    s = box_9k
    rng = np.random.default_rng(5)
    moved = (s.crd + rng.uniform(-0.26, 0.26, s.crd.shape)).astype(np.float32)
    out = []
    for margin in (0.0, 0.3):
        e = g.engine_create(s, 8.0)
        g.engine_set_water_bonded(e, s)
        try:
            g.capi.check(lib.snb_engine_set_prune_margin(e, ctypes.c_float(margin)), "margin")
            crd = g.dev(s.crd.reshape(-1), np.float32)
            vel = g.dev(s.vel.reshape(-1), np.float32)
            invm = g.dev((1.0 / s.mass).astype(np.float32))
            dt = 0.5e-3 * systems.TIME_CONVERSION
            g.capi.check(lib.snb_engine_md_steps(e, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                 ctypes.c_float(dt), 0, 10, g.stream()),
                         "md_steps")
            c2 = g.dev(moved.reshape(-1), np.float32)
            frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
            tot = torch.zeros(16, dtype=torch.float64, device="cuda")
            g.capi.check(lib.snb_engine_force(e, g.ptr(c2), g.ptr(frc), 10, 1, 1, g.ptr(tot),
                                              g.stream()), "engine_force")
            torch.cuda.synchronize()
            out.append((frc.cpu().numpy(), tot.cpu().numpy()))
        finally:
            lib.snb_engine_destroy(e)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_prune_margin_refuses_bad_values(g, box_9k):
    lib = g.capi.load()
    e = g.engine_create(box_9k, 8.0)
    try:
        for bad in (-0.5, float("nan"), 1e6):
            assert lib.snb_engine_set_prune_margin(e, ctypes.c_float(bad)) == \
                g.capi.SNB_ERR_BAD_INPUT
        assert lib.snb_engine_set_prune_margin(e, ctypes.c_float(0.0)) == g.capi.SNB_OK
    finally:
        lib.snb_engine_destroy(e)


def test_pruned_batch_md_is_bitwise_unchanged(g):
    """A batch of five boxes, 120 graph-replayed steps: pruned rows (per-box
    minimum images in the check) against full rows."""
    import torch
    from sponge_b200 import systems
    boxes = [systems.water_box(nw, seed=s, ion_pairs=None)
             for s, nw in enumerate([200, 450, 700, 260, 520])]
    offs = np.cumsum([0] + [b.n for b in boxes])[:-1]
    lib = g.capi.load()
    dt = 0.5e-3 * systems.TIME_CONVERSION
    out = []
    for margin in (0.0, 0.8):
        h, c = g.batch_create(boxes, 8.0)
        try:
            bonded = type("B", (), {})()
            bonded.bonds = np.concatenate([b.bonds + o for b, o in zip(boxes, offs)]).astype(np.int32)
            bonded.angles = np.concatenate([b.angles + o for b, o in zip(boxes, offs)]).astype(np.int32)
            g.engine_set_water_bonded(h, bonded)
            g.capi.check(lib.snb_engine_set_prune_margin(h, ctypes.c_float(margin)), "margin")
            crd, vel = g.dev(c["crd"]), g.dev(c["vel"])
            invm = g.dev((1.0 / c["mass"]).astype(np.float32))
            st = torch.cuda.Stream()
            sp = ctypes.c_void_p(st.cuda_stream)
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_md_steps_graph(h, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                           ctypes.c_float(dt), 0, 120, sp), "md")
            st.synchronize()
            passes = ctypes.c_int(0)
            g.capi.check(lib.snb_engine_prune_passes(h, ctypes.byref(passes), None, sp), "passes")
        finally:
            lib.snb_engine_destroy(h)
        out.append((crd.cpu().numpy(), vel.cpu().numpy(), passes.value))
    assert out[0][2] == 0 and out[1][2] >= 2
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_pruned_soft_core_md_is_bitwise_unchanged(g):
    """The engine's soft-core rows at lambda 0.5: 80 graph-replayed steps
    with pruned rows against full rows."""
    import torch
    from sponge_b200 import systems
    s, sc = systems.soft_core_box(1000, n_solute=32, seed=3)
    lib = g.capi.load()
    box = g.Box(s)
    dt = 0.5e-3 * systems.TIME_CONVERSION
    params = {"lambda_lj": 0.5, "soft_core_alpha": 0.5, "soft_core_powfer": 1.0,
              "soft_core_sigma": 3.0, "soft_core_sigma_min": 0.0}
    out = []
    for margin in (0.0, 0.3):
        e = g.engine_create(s, 10.0)
        g.engine_set_water_bonded(e, s)
        h = g.soft_create(box, sc, 10.0, params)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        st = torch.cuda.Stream()
        sp = ctypes.c_void_p(st.cuda_stream)
        passes = ctypes.c_int(0)
        try:
            g.capi.check(lib.snb_engine_set_soft_core(e, h), "set_soft_core")
            g.capi.check(lib.snb_engine_set_prune_margin(e, ctypes.c_float(margin)), "margin")
            with torch.cuda.stream(st):
                g.capi.check(lib.snb_engine_md_steps_graph(e, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                           ctypes.c_float(dt), 0, 80, sp), "md")
            st.synchronize()
            g.capi.check(lib.snb_engine_prune_passes(e, ctypes.byref(passes), None, sp), "passes")
        finally:
            lib.snb_engine_destroy(e)
            lib.snb_lj_soft_destroy(h)
        out.append((crd.cpu().numpy(), vel.cpu().numpy(), passes.value))
    assert out[1][2] >= 2
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
