"""The solvent split of the direct-space pairs (SOLVENT_LENNARD_JONES,
solvent_LJ.cpp:256-432, beside LENNARD_JONES_INFORMATION with
solvent_numbers, main.cpp:1453-1467): snb_lj_pme_direct_force with the last
S atoms declared solvent leaves out the pairs of two solvent atoms, and
snb_solvent_lj_pme_direct_force adds exactly those.

Box: 400 waters, cutoff 8 A; the last 300 waters are the solvent block.
The two calls together give the unsplit forces (relative RMS <= 1e-6; only
the order of the FP32 row sums differs), per-atom energies, Coulomb energies
and virials (summed: within 1e-6 relative) and match the FP64 oracle
(<= 1e-5); the solvent call alone moves no atom outside the block; a
solvent count beyond the atom count is rejected."""

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


def split_force(g, h, nl, box, beta, solvent_n, which):
    import torch
    lib = g.capi.load()
    n = box.n
    out = dict(frc=torch.zeros(3 * n, dtype=torch.float32, device="cuda"),
               ae=torch.zeros(n, dtype=torch.float32, device="cuda"),
               vir=torch.zeros(6 * n, dtype=torch.float32, device="cuda"),
               ce=torch.zeros(n, dtype=torch.float32, device="cuda"))
    P = {k: g.ptr(v) for k, v in out.items()}
    if which in ("lj", "both"):
        g.capi.check(lib.snb_lj_pme_direct_force(
            h, n, n, solvent_n, 0, g.ptr(box.crd), g.ptr(box.charge), P["frc"], box.b, nl,
            ctypes.c_float(beta), 1, P["ae"], 1, P["vir"], P["ce"], g.stream()), "lj")
    if which in ("solvent", "both"):
        g.capi.check(lib.snb_solvent_lj_pme_direct_force(
            h, nl, n, solvent_n, g.ptr(box.crd), g.ptr(box.charge), P["frc"], box.b,
            ctypes.c_float(beta), 1, P["ae"], 1, P["vir"], P["ce"], g.stream()), "solvent")
    torch.cuda.synchronize()
    return {k: v.cpu().numpy().astype(np.float64) for k, v in out.items()}


def test_solvent_split_adds_up(g, oracle):
    from sponge_b200 import systems
    s = systems.water_box(400, seed=2)
    box = g.Box(s)
    lib = g.capi.load()
    nl = g.make_nl(box, CUTOFF, 2.0)
    h = g.lj_create(box, CUTOFF)
    beta = oracle.get_beta(CUTOFF)
    S = 900
    try:
        g.nl_update(nl, box)
        full = split_force(g, h, nl, box, beta, 0, "lj")
        both = split_force(g, h, nl, box, beta, S, "both")
        solv = split_force(g, h, nl, box, beta, S, "solvent")
        bad = lib.snb_solvent_lj_pme_direct_force(
            h, nl, s.n, s.n + 1, g.ptr(box.crd), g.ptr(box.charge), None, box.b,
            ctypes.c_float(beta), 0, None, 0, None, None, g.stream())
    finally:
        lib.snb_lj_destroy(h)
        lib.snb_nl_destroy(nl)
    assert g.rel_rms(both["frc"], full["frc"]) <= 1e-6
    for k in ("ae", "ce"):
        assert abs(both[k].sum() - full[k].sum()) <= 1e-6 * np.abs(full[k]).sum()
    assert np.abs(both["vir"].sum(0) - full["vir"].sum(0)).max() <= \
        1e-6 * np.abs(full["vir"]).sum()
    # the solvent call touches only the block, and does real work there
    f = solv["frc"].reshape(-1, 3)
    assert not np.any(f[: s.n - S]) and np.abs(f[s.n - S:]).sum() > 0
    assert not np.any(solv["ae"][: s.n - S])
    # against the FP64 direct-space pairs
    rs, cols = oracle.nl_pairs_system(s, CUTOFF, 2.0)
    d = oracle.direct_f64(s, CUTOFF, beta, rs, cols)
    assert g.rel_rms(both["frc"].reshape(-1, 3), d["frc"]) <= 1e-5
    assert bad == g.capi.SNB_ERR_BAD_INPUT
