"""Neighbor list on the GPU against the oracle's FP32 pair set (bit-exact)."""

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


@pytest.mark.parametrize("name,cutoff", [("small_box", 8.0), ("box_9k", 8.0),
                                         ("box_9k", 10.0)])
def test_pair_set_bit_exact(g, oracle, request, name, cutoff):
    s = request.getfixturevalue(name)
    box = g.Box(s)
    nl = g.make_nl(box, cutoff, 2.0)
    try:
        g.nl_update(nl, box)
        got = g.nl_pairs(nl)
    finally:
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs_system(s, cutoff, 2.0)
    want = g.csr_to_pairs(rs, cols)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_pair_set_random_positions_and_no_exclusions(g, oracle):
    from sponge_b200 import systems
    rng = np.random.default_rng(7)
    s = systems.water_box(300, seed=3)
    s.crd = (rng.random((s.n, 3)) * s.box).astype(np.float32)  # overlaps allowed
    s.crd[:10] += np.float32(3 * s.box)  # unwrapped images far outside the box
    s.excl_numbers[:] = 0
    box = g.Box(s)
    nl = g.make_nl(box, 7.0, 1.5)
    try:
        g.nl_update(nl, box)
        got = g.nl_pairs(nl)
    finally:
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs(s.crd, s.cell(), s.rcell(), 7.0, 1.5)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))


def test_reference_layout_export(g, oracle, small_box):
    """d_nl in ATOM_GROUP layout: row i holds j > i (global), same sets."""
    import torch
    s = small_box
    box = g.Box(s)
    nl = g.make_nl(box, 8.0, 2.0)
    lib = g.capi.load()
    maxn = 1200
    groups = torch.zeros(s.n * 2, dtype=torch.int64, device="cuda")  # 16 B per row
    slab = torch.zeros(s.n * maxn, dtype=torch.int32, device="cuda")
    try:
        g.nl_update(nl, box)
        g.capi.check(lib.snb_nl_export_atom_groups(nl, g.ptr(groups), g.ptr(slab), maxn,
                                                   g.stream()), "export_groups")
        torch.cuda.synchronize()
    finally:
        lib.snb_nl_destroy(nl)
    raw = groups.cpu().numpy().view(np.int32).reshape(s.n, 4)
    counts = raw[:, 0]
    ptrs = groups.cpu().numpy().reshape(s.n, 2)[:, 1]
    base = slab.data_ptr()
    assert np.all(ptrs == base + 4 * maxn * np.arange(s.n))
    sl = slab.cpu().numpy().reshape(s.n, maxn)
    rs, cols = oracle.nl_pairs_system(s, 8.0, 2.0)
    for i in range(s.n):
        row = np.sort(sl[i, :counts[i]])
        assert np.array_equal(row, cols[rs[i]:rs[i + 1]])


def test_conditional_update_follows_skin_permit(g, oracle, small_box):
    """No rebuild below skin*skin_permit displacement, rebuild above it
    (NEIGHBOR_LIST::Update with CONDITIONAL_UPDATE)."""
    import torch
    s = small_box
    box = g.Box(s)
    nl = g.make_nl(box, 8.0, 2.0)
    try:
        g.nl_update(nl, box, forced=1)
        p0 = g.nl_pairs(nl)
        moved = s.crd.copy()
        moved[5] += np.float32([0.9, 0.0, 0.0])  # 0.9 A < 1.0 A trigger
        crd = torch.from_numpy(moved.reshape(-1)).cuda()
        g.nl_update(nl, box, crd=crd, forced=0)
        assert np.array_equal(g.nl_pairs(nl), p0)
        moved[5] += np.float32([0.2, 0.0, 0.0])  # now 1.1 A
        crd = torch.from_numpy(moved.reshape(-1)).cuda()
        g.nl_update(nl, box, crd=crd, forced=0)
        got = g.nl_pairs(nl)
    finally:
        g.capi.load().snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs(moved, s.cell(), s.rcell(), 8.0, 2.0, s.excl_start,
                               s.excl_numbers, s.excl_list)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))


def test_list_overflow_regrows(g, oracle, small_box):
    """A too-small pair store raises the overflow flag; Check_Overflow
    regrows it and the forced rebuild is then exact."""
    s = small_box
    box = g.Box(s)
    nl = g.make_nl(box, 8.0, 2.0)
    lib = g.capi.load()
    try:
        # shrink: move the box's atoms onto a tight cluster so the list outgrows
        # the capacity estimated at creation
        import torch
        dense = (s.crd - s.crd.mean(0)) * np.float32(0.5) + np.float32(s.box / 2)
        crd = torch.from_numpy(dense.astype(np.float32).reshape(-1)).cuda()
        g.nl_update(nl, box, forced=1)  # the first build, at the lattice density
        g.nl_update(nl, box, crd=crd, forced=1)
        regrown = ctypes.c_int(0)
        g.capi.check(lib.snb_nl_check_overflow(nl, ctypes.byref(regrown), g.stream()),
                     "check_overflow")
        assert regrown.value == 1
        g.nl_update(nl, box, crd=crd, forced=1)
        g.capi.check(lib.snb_nl_check_overflow(nl, ctypes.byref(regrown), g.stream()),
                     "check_overflow")
        assert regrown.value == 0
        got = g.nl_pairs(nl)
    finally:
        lib.snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs(dense.astype(np.float32), s.cell(), s.rcell(), 8.0, 2.0,
                               s.excl_start, s.excl_numbers, s.excl_list)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))


def test_list_is_deterministic(g, box_9k):
    """Two builds from the same coordinates give the same rows in the same
    order (stable cell sort, ballot-ordered fill)."""
    import torch
    box = g.Box(box_9k)
    lib = g.capi.load()
    outs = []
    for _ in range(2):
        nl = g.make_nl(box, 8.0, 2.0)
        try:
            g.nl_update(nl, box)
            cnt = ctypes.c_longlong(0)
            g.capi.check(lib.snb_nl_pair_count(nl, ctypes.byref(cnt), g.stream()), "")
            pi = torch.empty(cnt.value, dtype=torch.int32, device="cuda")
            pj = torch.empty(cnt.value, dtype=torch.int32, device="cuda")
            g.capi.check(lib.snb_nl_export_pairs(nl, g.ptr(pi), g.ptr(pj), cnt.value,
                                                 ctypes.byref(cnt), g.stream()), "")
            outs.append((pi.cpu().numpy(), pj.cpu().numpy()))
        finally:
            lib.snb_nl_destroy(nl)
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_first_build_regrows_by_itself(g, oracle, small_box):
    """A first build that outgrows the rows sized from the box's mean density
    (here the atoms packed into an eighth of the box) regrows and builds
    again before it returns: the list is exact without a Check_Overflow."""
    import torch
    s = small_box
    box = g.Box(s)
    nl = g.make_nl(box, 8.0, 2.0)
    lib = g.capi.load()
    dense = (s.crd - s.crd.mean(0)) * np.float32(0.5) + np.float32(s.box / 2)
    try:
        crd = torch.from_numpy(dense.astype(np.float32).reshape(-1)).cuda()
        g.nl_update(nl, box, crd=crd, forced=1)
        got = g.nl_pairs(nl)
    finally:
        lib.snb_nl_destroy(nl)
    rs, cols = oracle.nl_pairs(dense.astype(np.float32), s.cell(), s.rcell(), 8.0, 2.0,
                               s.excl_start, s.excl_numbers, s.excl_list)
    assert np.array_equal(got, g.csr_to_pairs(rs, cols))
