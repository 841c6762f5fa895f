"""The engine on the reference's Amber comparison case (alanine dipeptide in
TIP4P-Ew water, a rectangular 30.10 x 30.51 x 42.00 A box, extra points as
charged sites): nonbonded forces against the FP64 oracle (relative RMS
<= 1e-5) and, with the FP64 bonded terms of tests/test_cpu_amber_golden.py,
the total against sander's forces and energy at the reference's own
tolerances."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.mark.parametrize("iteration", [0, 1, 2])
def test_engine_matches_fp64_and_amber(g, oracle, iteration):
    import torch
    from tests import test_cpu_amber_golden as am
    s, z = am.load_amber(iteration)
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
    f_nb, e_nb = am.nonbonded_f64(oracle, s)
    got = frc.cpu().numpy().reshape(-1, 3).astype(np.float64)
    assert g.rel_rms(got, f_nb) <= 1e-5
    e_gpu = float(tot.cpu().numpy()[7])
    assert abs(e_gpu - e_nb) <= 1e-5 * abs(e_nb)
    x = np.asarray(z["crd64"], np.float64)
    f_b = am.bonded_forces(z, x, am.solute_atoms(z))
    st = am.compare(z, got + f_b, e_gpu + am.bonded_energy(z, x))
    print(f"\nAmber TIP4P-Ew alanine dipeptide frame {iteration}, engine: "
          f"|dE| {st['de']:.4f}, "
          f"max |dF| {st['max_abs']:.4f}, RMS dF {st['rms']:.4f}, cos {st['cos']:.6f}")
    assert st["de"] <= 0.5
    assert st["max_abs"] <= 0.10
    assert st["rms"] <= 0.03
    assert st["cos"] >= 0.999
