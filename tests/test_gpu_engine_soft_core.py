"""The fused engine with soft-core LJ (snb_engine_set_soft_core) against the
FP64 oracle: soft-core direct terms (oracle/snb_oracle.c, pinned to the
reference's own LJ_SOFT_CORE output by tests/test_cpu_oracle.py) plus the
excluded correction and PME of the same frame.

Box: 1,000 waters with a 32-site alchemical solute whose LJ and charges vanish
in state B, cutoff 8 A.  Tolerances: forces relative RMS <= 1e-5; LJ and
direct Coulomb energies within 2e-6 of their magnitude; the tail term within
1e-6 relative."""

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
def soft_box():
    from sponge_b200 import systems
    return systems.soft_core_box(1000, n_solute=32, seed=3)


def _params(lam):
    return {"lambda_lj": lam, "soft_core_alpha": 0.5, "soft_core_powfer": 1.0,
            "soft_core_sigma": 3.0, "soft_core_sigma_min": 0.0}


@pytest.mark.parametrize("lam", [0.0, 0.5, 1.0])
def test_engine_soft_core_matches_fp64(g, oracle, soft_box, lam):
    import torch
    from sponge_b200 import systems
    s, sc = soft_box
    lib = g.capi.load()
    box = g.Box(s)
    e = g.engine_create(s, CUTOFF)
    h = g.soft_create(box, sc, CUTOFF, _params(lam))
    crd = g.dev(s.crd.reshape(-1), np.float32)
    frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    try:
        g.capi.check(lib.snb_engine_set_soft_core(e, h), "set_soft_core")
        g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 1, 1, g.ptr(tot),
                                          g.stream()), "engine_force")
        torch.cuda.synchronize()
    finally:
        lib.snb_engine_destroy(e)
        lib.snb_lj_soft_destroy(h)
    beta = oracle.get_beta(CUTOFF)
    rs, cols = oracle.nl_pairs_system(s, CUTOFF, 2.0)
    d = oracle.soft_f64(s, sc, CUTOFF, beta, lam, 0.5, 1.0, 3.0, 0.0, rs, cols)
    ex = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)
    want = d["frc"] + ex["frc"] + p["frc"]
    got = frc.cpu().numpy().reshape(-1, 3)
    assert g.rel_rms(got, want) <= 1e-5
    t = tot.cpu().numpy()
    for idx, key in ((0, "lj_energy"), (2, "coulomb_energy")):
        scale = np.abs(d[key]).sum()
        assert abs(t[idx] - d[key].sum()) <= 2e-6 * scale, key
    f, _ = oracle.soft_lrc(s, sc, lam, CUTOFF)
    V = float(np.float32(s.box)) ** 3
    assert t[1] == pytest.approx(f / V, rel=1e-6)


def test_engine_soft_core_md_runs(g, soft_box):
    """20 graph-replayed NVE steps with soft-core pair terms at lambda 0.5 stay
    finite and match the same steps launched on the stream bit for bit."""
    import torch
    from sponge_b200 import systems
    s, sc = soft_box
    lib = g.capi.load()
    box = g.Box(s)
    dt = 0.5e-3 * systems.TIME_CONVERSION
    out = []
    for graph in (False, True):
        e = g.engine_create(s, CUTOFF)
        g.engine_set_water_bonded(e, s)
        h = g.soft_create(box, sc, CUTOFF, _params(0.5))
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        st = torch.cuda.Stream()
        try:
            g.capi.check(lib.snb_engine_set_soft_core(e, h), "set_soft_core")
            fn = lib.snb_engine_md_steps_graph if graph else lib.snb_engine_md_steps
            with torch.cuda.stream(st):
                g.capi.check(fn(e, g.ptr(crd), g.ptr(vel), g.ptr(invm), ctypes.c_float(dt), 0,
                                20, ctypes.c_void_p(st.cuda_stream)), "md")
            st.synchronize()
        finally:
            lib.snb_engine_destroy(e)
            lib.snb_lj_soft_destroy(h)
        out.append(crd.cpu().numpy())
    assert np.isfinite(out[1]).all()
    assert np.array_equal(out[0], out[1])
