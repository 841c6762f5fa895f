"""The BOND and ANGLE modules on the GPU (snb_bond_*, snb_angle_*) against
the FP64 oracle on the reference's golden inputs (tests/golden/bonded_*.npz:
the Amber alanine dipeptide case's terms, the triclinic water case's bond
file in its skewed cell, 300 displaced waters): forces within relative RMS
1e-5, per-atom energies and the energy sums within 1e-5 of FP64, the virial
sums within 1e-5 of their largest component (5e-5 for forces and virials of
the Amber bonds, whose r - r0 is formed in FP32 as the reference forms it;
the reference itself is at 2.2e-5 there); the results added to the caller's arrays (+=).
"""

import ctypes

import numpy as np
import pytest

from tests.test_cpu_bonded import CASES, load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _run(g, kind, z, rcell, terms):
    import torch
    lib = g.capi.load()
    n = len(z["crd"])
    h = ctypes.c_void_p()
    arr = [np.ascontiguousarray(t) for t in terms]
    ptrs = [a.ctypes.data for a in arr]
    create = lib.snb_bond_create if kind == "bond" else lib.snb_angle_create
    g.capi.check(create(n, len(arr[0]), *ptrs, ctypes.byref(h)), f"{kind}_create")
    crd = g.dev(z["crd"].reshape(-1), np.float32)
    base = np.random.default_rng(3).normal(size=3 * n).astype(np.float32)
    frc = torch.from_numpy(base.copy()).cuda()  # the module adds to what is there
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    bnd = g.capi.boundary(z["cell"], rcell)
    force = lib.snb_bond_force if kind == "bond" else lib.snb_angle_force
    energy = lib.snb_bond_energy if kind == "bond" else lib.snb_angle_energy
    destroy = lib.snb_bond_destroy if kind == "bond" else lib.snb_angle_destroy
    e = ctypes.c_float(0)
    try:
        g.capi.check(force(h, g.ptr(crd), bnd, g.ptr(frc), 1, g.ptr(ae), 1, g.ptr(vir),
                           g.stream()), f"{kind}_force")
        g.capi.check(energy(h, ctypes.byref(e), g.stream()), f"{kind}_energy")
        torch.cuda.synchronize()
    finally:
        destroy(h)
    return (frc.cpu().numpy().reshape(n, 3) - base.reshape(n, 3), ae.cpu().numpy(),
            vir.cpu().numpy().reshape(n, 6), e.value)


@pytest.mark.parametrize("name", CASES)
def test_bond_angle_modules_match_fp64(g, oracle, name):
    z, rcell, bonds, angles = load(name)
    want_b, want_a = oracle.bonded_f64(z["crd"], z["cell"], rcell, bonds, angles)
    for kind, terms, want in (("bond", bonds, want_b), ("angle", angles, want_a)):
        if len(terms[0]) == 0:
            continue
        f, ae, vir, e = _run(g, kind, z, rcell, terms)
        tol = 5e-5 if (kind == "bond" and "amber" in name) else 1e-5
        assert g.rel_rms(f, want["frc"]) <= tol, kind
        assert e == pytest.approx(want["energy"], rel=1e-5), kind
        assert np.abs(ae - want["atom_energy"]).max() <= 1e-5 * np.abs(
            want["atom_energy"]).max() + 1e-6, kind
        vs = vir.astype(np.float64).sum(0)
        ws = want["virial"].sum(0)
        assert np.all(np.abs(vs - ws) <= tol * np.abs(ws).max() + 1e-4), kind
