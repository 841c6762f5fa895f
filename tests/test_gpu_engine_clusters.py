"""The engine's cluster form of the neighbor list.

On request a single rectangular box with at least five cells per axis runs
on clusters (up to four atoms of a cell, each neighbour cluster stored once
per cluster with its 4x4 pair mask) instead of the default rows.  Held
here:
  * the pair set is the oracle's FP32 pair set bit for bit (the reference's
    criterion, exclusions, each pair once), at two cutoffs, with atoms
    far outside the box (unwrapped images) and with random positions;
  * forces, energies and virials of both list forms are within 1e-5 / 1e-6
    of FP64, and within 1e-6 of each other;
  * graph-replayed MD steps equal stream-launched ones bit for bit, and a
    list that outgrows its rows is regrown and the steps repeated;
  * boxes below five cells per axis keep the rows.
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


def _clusters(g, e):
    g.capi.check(g.capi.load().snb_engine_set_list_form(e, 1), "set_list_form")
    return _form(g, e)


def _form(g, e):
    c = ctypes.c_int(-1)
    g.capi.check(g.capi.load().snb_engine_list_form(e, ctypes.byref(c)), "list_form")
    return c.value


def _force(g, e, s, step=0):
    import torch
    lib = g.capi.load()
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), step, 1, 1, g.ptr(tot),
                                      g.stream()), "engine_force")
    torch.cuda.synchronize()
    return frc.cpu().numpy().reshape(s.n, 3), tot.cpu().numpy()


def _pairs(g, e):
    import torch
    lib = g.capi.load()
    cnt = ctypes.c_longlong(0)
    g.capi.check(lib.snb_engine_stats(e, None, ctypes.byref(cnt), g.stream()), "stats")
    n = cnt.value
    pi = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    pj = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    got = ctypes.c_longlong(0)
    g.capi.check(lib.snb_engine_export_pairs(e, g.ptr(pi), g.ptr(pj), n, ctypes.byref(got),
                                             g.stream()), "engine_export_pairs")
    assert got.value == n
    p = np.stack([pi[:n].cpu().numpy(), pj[:n].cpu().numpy()], 1).astype(np.int64)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


@pytest.mark.parametrize("cutoff", [8.0, 10.0])
def test_cluster_pair_set_bit_exact(g, oracle, box_9k, cutoff):
    s = box_9k
    e = g.engine_create(s, cutoff)
    try:
        assert _clusters(g, e) == 1
        _force(g, e, s)
        got = _pairs(g, e)
    finally:
        g.capi.load().snb_engine_destroy(e)
    rs, cols = oracle.nl_pairs_system(s, cutoff, 2.0)
    want = g.csr_to_pairs(rs, cols)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_cluster_pair_set_unwrapped_and_random(g, oracle):
    from sponge_b200 import systems
    rng = np.random.default_rng(11)
    s = systems.water_box(2000, seed=5)
    s.crd[:50] += np.float32(2 * s.box)          # images far outside the box
    s.crd[50:100] -= np.float32(3 * s.box)
    s.crd[100:400] = (rng.random((300, 3)) * s.box).astype(np.float32)  # overlaps
    e = g.engine_create(s, 7.0, skin=1.5)
    try:
        assert _clusters(g, e) == 1
        _force(g, e, s)
        got = _pairs(g, e)
    finally:
        g.capi.load().snb_engine_destroy(e)
    rs, cols = oracle.nl_pairs_system(s, 7.0, 1.5)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))


def test_forms_agree_with_fp64_and_each_other(g, oracle, box_9k):
    from tests.test_gpu_engine import oracle_total
    s = box_9k
    lib = g.capi.load()
    out = {}
    for form in (1, 0):
        e = g.engine_create(s, 8.0)
        try:
            g.capi.check(lib.snb_engine_set_list_form(e, form), "set_list_form")
            assert _form(g, e) == form
            out[form] = _force(g, e, s)
        finally:
            lib.snb_engine_destroy(e)
    f_want, en, vir = oracle_total(oracle, s, 8.0)
    for form, (f, t) in out.items():
        assert g.rel_rms(f, f_want) <= 1e-5, form
        for k, idx in (("lj", 0), ("coul", 2), ("excl", 3), ("recip", 4), ("self", 5)):
            assert abs(t[idx] - en[k]) <= 2e-6 * abs(en[k]), (form, k)
        scale = np.abs(vir).max()
        assert np.abs(t[8:14] - vir).max() <= 2e-6 * scale, form
    assert g.rel_rms(out[1][0], out[0][0]) <= 1e-6


def _md(g, e, s, steps, graph, first=0):
    import torch
    from sponge_b200 import systems
    lib = g.capi.load()
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev((1.0 / s.mass).astype(np.float32))
    dt = 0.5e-3 * systems.TIME_CONVERSION
    fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
    st = torch.cuda.Stream()  # graph replay needs a stream of its own
    with torch.cuda.stream(st):
        g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), first,
                        steps, ctypes.c_void_p(st.cuda_stream)), "md_steps")
    st.synchronize()
    return crd.cpu().numpy(), vel.cpu().numpy()


def test_graph_equals_stream_on_clusters(g, box_9k):
    s = box_9k
    res = []
    for graph in (False, True):
        e = g.engine_create(s, 8.0)
        g.engine_set_water_bonded(e, s)
        try:
            assert _clusters(g, e) == 1
            res.append(_md(g, e, s, 120, graph))
        finally:
            g.capi.load().snb_engine_destroy(e)
    assert np.isfinite(res[0][0]).all()
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])


def test_dense_region_regrows_cluster_rows(g, oracle):
    """Half the box packed at twice the density: the first build outgrows the
    rows sized from the mean density, regrows them and builds again."""
    from sponge_b200 import systems
    s = systems.water_box(3000, seed=2)
    L = np.float32(s.box)
    x = s.crd[:, 0] - np.floor(s.crd[:, 0] / L) * L
    s.crd[:, 0] = np.where(x < L / 2, x * np.float32(0.5), x)  # left half squeezed
    e = g.engine_create(s, 8.0)
    try:
        assert _clusters(g, e) == 1
        _force(g, e, s)
        got = _pairs(g, e)
    finally:
        g.capi.load().snb_engine_destroy(e)
    rs, cols = oracle.nl_pairs_system(s, 8.0, 2.0)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))


def test_small_box_uses_rows(g, small_box):
    lib = g.capi.load()
    e = g.engine_create(small_box, 8.0)
    try:
        assert _form(g, e) == 0
        assert lib.snb_engine_set_list_form(e, 1) != 0
    finally:
        lib.snb_engine_destroy(e)
