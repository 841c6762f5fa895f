"""snb_pme_excluded_force_noalloc (static device scratch, no allocation)
against snb_pme_excluded_force on the same inputs.

Both run the same excluded-pair kernel with fixed-point accumulation, so the
results are expected to agree to the last bit; the test holds them to
relative 1e-6 (forces, per-atom energies, per-atom virials).  Two calls in a
row check that each call leaves the shared scratch at zero for the next one,
and a call at a different atom count in between checks that a smaller call
does not leave stale sums in the stride of a larger one.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-6


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _noalloc(g, box, beta, energy=True, virial=True):
    import torch
    lib = g.capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    g.capi.check(lib.snb_pme_excluded_force_noalloc(
        n, g.ptr(box.crd), box.b, g.ptr(box.charge), ctypes.c_float(beta), g.ptr(box.es),
        g.ptr(box.el), g.ptr(box.en), g.ptr(frc), int(energy), g.ptr(ae), int(virial),
        g.ptr(vir), g.stream()), "pme_excluded_force_noalloc")
    torch.cuda.synchronize()
    return dict(frc=frc.cpu().numpy().reshape(n, 3), atom_energy=ae.cpu().numpy(),
                virial=vir.cpu().numpy().reshape(n, 6))


def _with_handle(g, box):
    h, beta, _ = g.pme_create(box, 8.0)
    try:
        return beta, g.pme_excluded(h, box)
    finally:
        g.capi.load().snb_pme_destroy(h)


def _same(got, want):
    for k in ("frc", "atom_energy", "virial"):
        a = np.asarray(got[k], np.float64)
        b = np.asarray(want[k], np.float64)
        assert np.allclose(a, b, rtol=TOL, atol=TOL * np.abs(b).max()), k


def test_noalloc_matches_handle_path_on_consecutive_calls(g, box_9k, small_box):
    big, small = g.Box(box_9k), g.Box(small_box)
    beta, want_big = _with_handle(g, big)
    beta_s, want_small = _with_handle(g, small)
    _same(_noalloc(g, big, beta), want_big)
    _same(_noalloc(g, big, beta), want_big)
    _same(_noalloc(g, small, beta_s), want_small)
    _same(_noalloc(g, big, beta), want_big)


def test_noalloc_forces_only_then_full(g, box_9k):
    box = g.Box(box_9k)
    beta, want = _with_handle(g, box)
    got = _noalloc(g, box, beta, energy=False, virial=False)
    assert np.allclose(got["frc"], want["frc"], rtol=TOL,
                       atol=TOL * np.abs(want["frc"]).max())
    assert not np.any(got["atom_energy"]) and not np.any(got["virial"])
    _same(_noalloc(g, box, beta), want)


def test_noalloc_rejects_more_atoms_than_its_scratch(g):
    lib = g.capi.load()
    limit = 65536
    unit = [1.0, 0.0, 1.0, 0.0, 0.0, 1.0]
    rc = lib.snb_pme_excluded_force_noalloc(
        limit + 1, None, g.capi.boundary(unit, unit), None, ctypes.c_float(0.3),
        None, None, None, None, 0, None, 0, None, None)
    assert rc == 1
    assert b"65536" in lib.snb_last_error()


def test_noalloc_later_calls_leave_free_device_memory_unchanged(g, box_9k):
    """After the first call (which may load the module and with it the static
    array), further calls take no device memory: the free bytes the driver
    reports stay the same and torch's allocator sees no new reservation."""
    import torch
    box = g.Box(box_9k)
    beta, want = _with_handle(g, box)
    _same(_noalloc(g, box, beta), want)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    lib = g.capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    reserved1 = torch.cuda.memory_reserved()
    for _ in range(3):
        g.capi.check(lib.snb_pme_excluded_force_noalloc(
            n, g.ptr(box.crd), box.b, g.ptr(box.charge), ctypes.c_float(beta), g.ptr(box.es),
            g.ptr(box.el), g.ptr(box.en), g.ptr(frc), 1, g.ptr(ae), 1, g.ptr(vir),
            g.stream()), "pme_excluded_force_noalloc")
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_reserved() == reserved1
    assert free2 == free1, (free0, free1, free2, reserved0, reserved1)


def test_noalloc_call_captured_in_a_graph(g, box_9k):
    """After a first call outside any capture, a call captured in a CUDA
    graph and replayed gives the handle path's results, replay after
    replay (the scratch is cleared by each call)."""
    import torch
    lib = g.capi.load()
    box = g.Box(box_9k)
    beta, want = _with_handle(g, box)
    _noalloc(g, box, beta)  # the first call resolves the scratch
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side, capture_error_mode="thread_local"):
            g.capi.check(lib.snb_pme_excluded_force_noalloc(
                n, g.ptr(box.crd), box.b, g.ptr(box.charge), ctypes.c_float(beta),
                g.ptr(box.es), g.ptr(box.el), g.ptr(box.en), g.ptr(frc), 1, g.ptr(ae), 1,
                g.ptr(vir), ctypes.c_void_p(side.cuda_stream)), "captured call")
    torch.cuda.synchronize()
    for _ in range(2):
        for t in (frc, ae, vir):
            t.zero_()
        graph.replay()
        torch.cuda.synchronize()
        _same(dict(frc=frc.cpu().numpy().reshape(n, 3), atom_energy=ae.cpu().numpy(),
                   virial=vir.cpu().numpy().reshape(n, 6)), want)
    del graph
