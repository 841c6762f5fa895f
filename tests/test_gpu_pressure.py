"""Stress and pressure of the engine (snb_engine_pressure, after
MD_INFORMATION::Get_pressure, MD_core.cpp:1080-1107): the potential virial
of snb_engine_force plus the kinetic tensor over the volume, against numpy
on the same arrays (1e-9 relative); and, with SETTLE, the constraint virial
of one MD step against the constraint forces worked out from the step
itself (m (x_final - x_unconstrained) / dt^2 against the start positions;
1e-2 relative, the FP32 position differences set it)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PRES = 6.946827162543585e4


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def kinetic(vel, mass):
    v = np.asarray(vel, np.float64)
    m = np.asarray(mass, np.float64)[:, None]
    return np.array([(m[:, 0] * v[:, 0] * v[:, 0]).sum(), (m[:, 0] * 2 * v[:, 0] * v[:, 1]).sum(),
                     (m[:, 0] * v[:, 1] * v[:, 1]).sum(), (m[:, 0] * 2 * v[:, 0] * v[:, 2]).sum(),
                     (m[:, 0] * 2 * v[:, 1] * v[:, 2]).sum(), (m[:, 0] * v[:, 2] * v[:, 2]).sum()])


def test_pressure_from_virial_and_kinetic(g):
    import torch
    from sponge_b200 import systems
    s = systems.water_box(500, seed=4)
    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    mass = g.dev(s.mass, np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(7, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "force")
        g.capi.check(lib.snb_engine_pressure(e, g.ptr(vel), g.ptr(mass), g.ptr(tot), g.ptr(out),
                                             g.stream()), "pressure")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
    V = float(np.float32(s.box)) ** 3
    t = tot.cpu().numpy()
    want = (t[8:14] + kinetic(s.vel, s.mass)) / V
    got = out.cpu().numpy()
    assert np.abs(got[:6] - want).max() <= 1e-9 * np.abs(want).max()
    assert got[6] == pytest.approx((want[0] + want[2] + want[5]) / 3 * PRES, rel=1e-9)


def test_pressure_takes_the_settle_constraint_virial(g):
    import torch
    from sponge_b200 import systems
    from tests.golden import make_settle_golden as mg
    from tests.test_gpu_settle import settle_create
    s = systems.water_box(216, seed=5)
    o = np.arange(0, s.n, 3)
    ai = np.concatenate([o, o, o + 1]).astype(np.int32)
    aj = np.concatenate([o + 1, o + 2, o + 2]).astype(np.int32)
    r0 = np.concatenate([np.full(len(o), mg.R_OH), np.full(len(o), mg.R_OH),
                         np.full(len(o), mg.R_HH)]).astype(np.float32)
    lib = g.capi.load()
    dt = np.float32(2e-3 * systems.TIME_CONVERSION)
    invm_h = (1.0 / s.mass).astype(np.float32)
    # forces at the start (a fresh engine builds the same list)
    e0 = g.engine_create(s, 8.0)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e0, g.ptr(crd), g.ptr(frc), 0, 0, 0, None,
                                          g.stream()), "force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e0)
    f0 = frc.cpu().numpy().reshape(-1, 3)
    e = g.engine_create(s, 8.0)
    h = settle_create(g, s.n, ai, aj, r0, s.mass)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev(invm_h)
    mass = g.dev(s.mass, np.float32)
    out = torch.zeros(7, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    try:
        g.capi.check(lib.snb_engine_set_settle(e, h), "set_settle")
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_md_steps(e, g.ptr(crd), g.ptr(vel), g.ptr(invm),
                                                 ctypes.c_float(dt), 0, 1,
                                                 ctypes.c_void_p(st.cuda_stream)), "md")
            g.capi.check(lib.snb_engine_pressure(e, g.ptr(vel), g.ptr(mass), None, g.ptr(out),
                                                 ctypes.c_void_p(st.cuda_stream)), "pressure")
        st.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_settle_destroy(h)
    x1 = crd.cpu().numpy().reshape(-1, 3).astype(np.float64)
    v1 = vel.cpu().numpy().reshape(-1, 3)
    v_unc = s.vel + dt * (invm_h[:, None] * f0)
    x_unc = s.crd.astype(np.float64) + np.float64(dt) * v_unc.astype(np.float64)
    F = s.mass[:, None].astype(np.float64) * (x1 - x_unc) / np.float64(dt) ** 2
    L = np.float64(np.float32(s.box))
    rel = s.crd.astype(np.float64).copy()
    for k in (1, 2):  # hydrogens next to their oxygen
        d = rel[o + k] - rel[o]
        rel[o + k] = rel[o] + d - np.round(d / L) * L
    W = np.array([(F[:, 0] * rel[:, 0]).sum(),
                  (F[:, 0] * rel[:, 1] + F[:, 1] * rel[:, 0]).sum(),
                  (F[:, 1] * rel[:, 1]).sum(),
                  (F[:, 0] * rel[:, 2] + F[:, 2] * rel[:, 0]).sum(),
                  (F[:, 1] * rel[:, 2] + F[:, 2] * rel[:, 1]).sum(),
                  (F[:, 2] * rel[:, 2]).sum()])
    V = L ** 3
    got = out.cpu().numpy()[:6] * V - kinetic(v1, s.mass)
    assert np.abs(got - W).max() <= 1e-2 * np.abs(W).max()
