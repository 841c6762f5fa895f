"""The reference's own GPU path (FP32 arithmetic, float atomics; its module
sources compiled as CUDA into oracle/_ref/libsponge_ref_gpu.so) next to the
fixed-point engine on the same 9,000-atom box: both against the FP64 oracle,
and a short NVE run of each from the same start."""

import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.fixture(scope="module")
def refgpu(g, box_9k):
    from oracle.oracle import ReferenceGPU
    r = ReferenceGPU()
    r.init(box_9k, 8.0, 2.0)
    return r


def _fp64_total(oracle, s, cutoff, skin=2.0):
    from sponge_b200 import systems
    beta = oracle.get_beta(cutoff)
    rs, cols = oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    e = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)
    V = float(np.float32(s.box)) ** 3
    lrc = oracle.lrc_factor(s, cutoff) / V
    frc = d["frc"] + e["frc"] + p["frc"]
    parts = [d["lj_energy"].sum(), d["coulomb_energy"].sum(), e["atom_energy"].sum(),
             p["e_recip"], p["e_self"], lrc]
    # the total is a small difference of large terms: errors are stated
    # relative to the sum of the terms' magnitudes
    return frc, sum(parts), sum(abs(x) for x in parts)


def test_reference_gpu_against_fp64(g, refgpu, oracle, box_9k):
    """The float-atomic path is within 1e-3 relative RMS of FP64 (it is the
    comparison point, not held to the 1e-5 bar); the fixed-point engine on
    the same frame is within 1e-5."""
    import torch
    s = box_9k
    assert refgpu.grid == (48, 48, 48)
    assert refgpu.beta == pytest.approx(oracle.get_beta(8.0), rel=1e-7)
    out = refgpu.force(forced=True)
    f64, e64, scale = _fp64_total(oracle, s, 8.0)
    err_ref = g.rel_rms(out["frc"], f64)
    e_ref = float(out["atom_energy"].astype(np.float64).sum()) + out["potential"]

    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
    err_ours = g.rel_rms(frc.cpu().numpy().reshape(-1, 3), f64)
    e_ours = float(tot.cpu().numpy()[7])
    print(f"\nforce rel-RMS vs FP64: reference GPU {err_ref:.3e}, fixed point {err_ours:.3e}; "
          f"energy error / sum of |terms|: reference GPU {abs(e_ref - e64) / scale:.3e}, "
          f"fixed point {abs(e_ours - e64) / scale:.3e}")
    assert err_ref < 1e-3
    assert abs(e_ref - e64) <= 1e-4 * scale
    assert err_ours <= 1e-5
    assert abs(e_ours - e64) <= 1e-6 * scale


def test_reference_gpu_nve_follows_engine(g, refgpu, box_9k):
    """40 NVE steps at 0.5 fs from the same start: the reference's GPU
    modules (with its bond and angle modules) and the fixed-point engine
    stay within 1e-3 A of each other."""
    import ctypes
    import torch
    from sponge_b200 import systems
    s = copy.deepcopy(box_9k)
    dt = 0.5e-3 * systems.TIME_CONVERSION
    inv_m = (1.0 / s.mass).astype(np.float32)
    refgpu.set_bonded(s.bonds, systems.BOND_K, systems.BOND_R0, s.angles,
                      systems.ANGLE_K, systems.ANGLE_T0)
    refgpu.set_state(s.crd, s.vel, inv_m)
    ms = refgpu.md_steps(40, dt)
    c_ref, v_ref = refgpu.get_state()
    assert ms > 0 and np.isfinite(c_ref).all()

    lib = g.capi.load()
    e = g.engine_create(s, 8.0)
    g.engine_set_water_bonded(e, s)
    crd = g.dev(s.crd.reshape(-1), np.float32)
    vel = g.dev(s.vel.reshape(-1), np.float32)
    invm = g.dev(inv_m)
    st = torch.cuda.Stream()
    try:
        with torch.cuda.stream(st):
            g.capi.check(lib.snb_engine_md_steps_graph(
                e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0, 40,
                ctypes.c_void_p(st.cuda_stream)), "md_steps")
        st.synchronize()
    finally:
        lib.snb_engine_destroy(e)
    c_ours = crd.cpu().numpy().reshape(-1, 3)
    dmax = float(np.abs(c_ours - c_ref).max())
    print(f"\nmax |crd difference| after 40 steps: {dmax:.2e} A")
    assert dmax <= 1e-3
    count, overflow = refgpu.pair_count()
    assert overflow == 0 and count > 0
