"""SETTLE on the GPU (snb_settle_* and snb_engine_set_settle) against the
golden vectors of the reference's own SETTLE and the FP64 oracle (iterated
SHAKE on the same constraints), with the tolerances of
tests/test_cpu_settle.py; a rigid pair without a real update reported to the
host; and rigid-water MD in the engine at 2 fs: graph-replayed steps equal
stream-launched ones bit for bit and every constraint holds to 1e-4 A."""

import ctypes

import numpy as np
import pytest

from tests import test_cpu_settle as cs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def settle_create(g, n, ai, aj, r0, mass):
    lib = g.capi.load()
    h = ctypes.c_void_p()
    a = [np.ascontiguousarray(ai, np.int32), np.ascontiguousarray(aj, np.int32),
         np.ascontiguousarray(r0, np.float32), np.ascontiguousarray(mass, np.float32)]
    g.capi.check(lib.snb_settle_create(n, len(a[0]), *[x.ctypes.data for x in a],
                                       ctypes.byref(h)), "settle_create")
    return h


def test_settle_module_matches_reference_and_fp64(g, oracle):
    import torch
    z = cs.load()
    lib = g.capi.load()
    n = len(z["mass"])
    h = settle_create(g, n, z["atom_i"], z["atom_j"], z["constant_r"], z["mass"])
    nt, np_, nl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    left = np.zeros(len(z["atom_i"]), np.int32)
    crd_old = g.dev(z["crd_old"].reshape(-1), np.float32)
    crd = g.dev(z["crd_new"].reshape(-1), np.float32)
    vel = g.dev(z["vel"].reshape(-1), np.float32)
    stress = torch.zeros(6, dtype=torch.float32, device="cuda")
    bnd = g.capi.boundary(z["cell"], z["rcell"])
    bad = ctypes.c_int(0)
    try:
        g.capi.check(lib.snb_settle_counts(h, ctypes.byref(nt), ctypes.byref(np_),
                                           ctypes.byref(nl), left.ctypes.data), "counts")
        g.capi.check(lib.snb_settle_remember_last_coordinates(h, g.ptr(crd_old), bnd,
                                                              g.stream()), "remember")
        g.capi.check(lib.snb_settle_do(h, g.ptr(crd), bnd, g.ptr(vel), ctypes.c_float(z["dt"]),
                                       ctypes.c_float(1.0), ctypes.c_float(1.0), 1,
                                       g.ptr(stress), g.stream()), "settle_do")
        g.capi.check(lib.snb_settle_status(h, ctypes.byref(bad), g.stream()), "status")
        torch.cuda.synchronize()
    finally:
        lib.snb_settle_destroy(h)
    assert [nt.value, np_.value, nl.value] == list(z["ref_counts"])
    got_left = np.stack([z["atom_i"][left[:nl.value]], z["atom_j"][left[:nl.value]]], 1)
    assert np.array_equal(got_left, z["ref_left"])
    assert bad.value == -1
    o = cs.oracle_step(oracle, z)
    x = crd.cpu().numpy().reshape(n, 3)
    v = vel.cpu().numpy().reshape(n, 3)
    s = stress.cpu().numpy()
    cs.check_against_oracle(z, o, x, v, s)
    # and against the reference's own FP32 step
    assert np.abs(x - z["ref_crd"]).max() <= 2 * cs.TOL_CRD


def test_settle_reports_a_pair_without_solution(g):
    """A rigid pair whose new bond is perpendicular to the old one and five
    times too long has no real update: the pair is left as it is and the
    status call returns SNB_ERR_BAD_INPUT with its index."""
    import torch
    lib = g.capi.load()
    mass = np.array([12.0, 16.0, 1.0], np.float32)
    h = settle_create(g, 3, [0], [1], [1.0], mass)
    old = np.array([[10, 10, 10], [11, 10, 10], [15, 15, 15]], np.float32)
    new = np.array([[10, 10, 10], [10, 15, 10], [15, 15, 15]], np.float32)
    crd_old = g.dev(old.reshape(-1))
    crd = g.dev(new.reshape(-1))
    vel = torch.zeros(9, dtype=torch.float32, device="cuda")
    bnd = g.capi.boundary([40, 0, 40, 0, 0, 40], [1 / 40, 0, 1 / 40, 0, 0, 1 / 40])
    bad = ctypes.c_int(0)
    try:
        g.capi.check(lib.snb_settle_remember_last_coordinates(h, g.ptr(crd_old), bnd,
                                                              g.stream()), "remember")
        g.capi.check(lib.snb_settle_do(h, g.ptr(crd), bnd, g.ptr(vel), ctypes.c_float(0.04),
                                       ctypes.c_float(1.0), ctypes.c_float(1.0), 0, None,
                                       g.stream()), "settle_do")
        rc = lib.snb_settle_status(h, ctypes.byref(bad), g.stream())
        rc2 = lib.snb_settle_status(h, ctypes.byref(bad), g.stream())
    finally:
        lib.snb_settle_destroy(h)
    assert rc == g.capi.SNB_ERR_BAD_INPUT
    assert b"no real position update" in lib.snb_last_error()
    assert rc2 == g.capi.SNB_OK and bad.value == -1
    assert np.array_equal(crd.cpu().numpy().reshape(3, 3), new)


def test_engine_rigid_water_md(g):
    """100 NVE steps of 300 rigid waters at 2 fs (SETTLE, no water bonds or
    angles): graph replay equals stream launches bit for bit; every O-H and
    H-H length holds to 1e-4 A."""
    import torch
    from sponge_b200 import systems
    from tests.golden import make_settle_golden as mg
    s = systems.water_box(300, seed=21)
    o = np.arange(0, s.n, 3)
    ai = np.concatenate([o, o, o + 1]).astype(np.int32)
    aj = np.concatenate([o + 1, o + 2, o + 2]).astype(np.int32)
    r0 = np.concatenate([np.full(len(o), mg.R_OH), np.full(len(o), mg.R_OH),
                         np.full(len(o), mg.R_HH)]).astype(np.float32)
    lib = g.capi.load()
    dt = 2e-3 * systems.TIME_CONVERSION
    out = []
    for graph in (False, True):
        e = g.engine_create(s, 8.0)
        h = settle_create(g, s.n, ai, aj, r0, s.mass)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        st = torch.cuda.Stream()
        try:
            g.capi.check(lib.snb_engine_set_settle(e, h), "set_settle")
            fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
            with torch.cuda.stream(st):
                g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                                100, ctypes.c_void_p(st.cuda_stream)), "md")
            st.synchronize()
        finally:
            lib.snb_engine_destroy(e)
            lib.snb_settle_destroy(h)
        out.append(crd.cpu().numpy().reshape(-1, 3).astype(np.float64))
    assert np.isfinite(out[1]).all()
    assert np.array_equal(out[0], out[1])
    x = out[1]
    d = x[aj] - x[ai]
    L = np.float64(s.box)
    d -= np.round(d / L) * L
    assert np.abs(np.linalg.norm(d, axis=1) - r0).max() <= 1e-4
