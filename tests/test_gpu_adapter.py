"""One force evaluation driven through the reference-side adapter
(oracle/_ref/libsponge_nb_adapter.so: SPONGE's module structs with the
reference's member signatures over the C ABI), against the same calls made
on the C ABI directly.

The adapter's driver runs main.cpp's one-rank order (forced list update,
excluded correction, LJ + direct Coulomb, LJ tail, PME reciprocal, then
Step_Print) with the LJ tables in Xponge::system.  The same calls on the C
ABI in the same order, on the legacy default stream, must give the same
bits: forces, per-atom energies and virials, the box virial, the potential
and the printed sums.  The forces are also held to the FP64 oracle.

The adapter ends the process through CONTROLLER::Throw_SPONGE_Error on an
error, as the reference does, so it runs in a child process.
"""

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ADAPTER_SO = os.path.join(ROOT, "oracle", "_ref", "libsponge_nb_adapter.so")
CUTOFF, SKIN = 8.0, 2.0
PRINTS = ["LJ_short", "LJ_long", "LJ", "PM", "PM_direct", "PM_reciprocal", "PM_self",
          "PM_correction", "beta"]


def _system():
    sys.path.insert(0, ROOT)
    from sponge_b200 import systems
    return systems.water_box(216, seed=1)


def _c(a, dt):
    return np.ascontiguousarray(a, dt)


def run_adapter(out_path):
    """Child process: adapter_force on the 648-atom box, results to out_path."""
    s = _system()
    lib = ctypes.CDLL(ADAPTER_SO)
    n = s.n
    keep = dict(crd=_c(s.crd.reshape(-1), np.float32), q=_c(s.charge, np.float32),
                t=_c(s.lj_type, np.int32), A=_c(s.lj_A, np.float32),
                B=_c(s.lj_B, np.float32), es=_c(s.excl_start, np.int32),
                en=_c(s.excl_numbers, np.int32), el=_c(s.excl_list, np.int32),
                cell=_c(s.cell(), np.float32), rcell=_c(s.rcell(), np.float32))
    out = dict(frc=np.zeros(3 * n, np.float32), atom_energy=np.zeros(n, np.float32),
               atom_virial=np.zeros(6 * n, np.float32), virial=np.zeros(6, np.float32),
               potential=np.zeros(1, np.float32), prints=np.zeros(9, np.float32))
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    rc = lib.adapter_force(
        ctypes.c_int(n), P(keep["crd"]), P(keep["q"]), ctypes.c_int(s.n_types),
        P(keep["t"]), P(keep["A"]), P(keep["B"]), P(keep["es"]), P(keep["en"]),
        ctypes.c_int(len(keep["el"])), P(keep["el"]), P(keep["cell"]), P(keep["rcell"]),
        ctypes.c_float(CUTOFF), ctypes.c_float(SKIN), P(out["frc"]),
        P(out["atom_energy"]), P(out["atom_virial"]), P(out["virial"]),
        P(out["potential"]), P(out["prints"]))
    np.savez(out_path, rc=np.int32(rc), **out)


def run_c_abi(s):
    """The adapter's sequence of calls made on the C ABI directly."""
    import torch

    from sponge_b200 import capi
    from tests.gpu_helpers import dev, ptr
    lib = capi.load()
    n = s.n
    b = capi.boundary(s.cell(), s.rcell())
    crd, q = dev(s.crd.reshape(-1), np.float32), dev(s.charge, np.float32)
    local = dev(np.arange(n, dtype=np.int32))
    es, en, el = (dev(s.excl_start, np.int32), dev(s.excl_numbers, np.int32),
                  dev(s.excl_list, np.int32))
    z = lambda k: torch.zeros(k, dtype=torch.float32, device="cuda")  # noqa: E731
    frc, energy, atom_vir, vir, pot = z(3 * n), z(n), z(6 * n), z(6), z(1)
    corr, direct = z(n), z(n)
    cell = s.cell()
    volume = np.float32(cell[0]) * np.float32(cell[2]) * np.float32(cell[5])
    L = np.array([cell[0], cell[2], cell[5]], np.float32)
    nl, lj, pme = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    t, A, B = _c(s.lj_type, np.int32), _c(s.lj_A, np.float32), _c(s.lj_B, np.float32)
    capi.check(lib.snb_pme_create(ctypes.byref(capi.options(cutoff=CUTOFF)), n, b,
                                  L.ctypes.data, CUTOFF, ctypes.byref(pme)), "pme")
    capi.check(lib.snb_lj_create(ctypes.byref(capi.options(cutoff=CUTOFF)), n, s.n_types,
                                 t.ctypes.data, A.ctypes.data, B.ctypes.data, CUTOFF,
                                 ctypes.byref(lj)), "lj")
    capi.check(lib.snb_nl_create(ctypes.byref(capi.options(cutoff=CUTOFF, skin=SKIN)), n,
                                 CUTOFF, SKIN, b, ctypes.byref(nl)), "nl")
    beta = float(lib.snb_pme_beta(pme))
    try:
        capi.check(lib.snb_lj_get_local(lj, ptr(local), n, 0, None), "get_local")
        capi.check(lib.snb_nl_update(nl, ptr(local), n, 0, ptr(crd), b, 0, 1, ptr(es),
                                     ptr(el), ptr(en), None), "nl_update")
        capi.check(lib.snb_pme_excluded_force(pme, n, ptr(local), ptr(local), ptr(crd), b,
                                              ptr(q), ptr(es), ptr(el), ptr(en), ptr(frc),
                                              1, ptr(corr), 1, ptr(atom_vir), None),
                   "excluded")
        energy += corr
        capi.check(lib.snb_lj_pme_direct_force(lj, n, n, 0, 0, ptr(crd), ptr(q), ptr(frc),
                                               b, nl, ctypes.c_float(beta), 1, ptr(energy),
                                               1, ptr(atom_vir), ptr(direct), None),
                   "lj_direct")
        capi.check(lib.snb_lj_long_range_correction(lj, 1, ptr(vir), 1, ptr(pot),
                                                    ctypes.c_float(volume), None), "tail")
        capi.check(lib.snb_pme_reciprocal_force(pme, ptr(crd), b, ptr(q), ptr(frc), 1, 1,
                                                ptr(vir), ptr(pot), 0, None), "recip")
        torch.cuda.synchronize()
        lj_sum = ctypes.c_float(0)
        capi.check(lib.snb_lj_energy_sum(lj, ctypes.byref(lj_sum), None), "lj_sum")
        rec, slf = ctypes.c_double(0), ctypes.c_double(0)
        v6 = np.zeros(6)
        capi.check(lib.snb_pme_energies(pme, ctypes.byref(rec), ctypes.byref(slf),
                                        v6.ctypes.data, None), "pme_energies")
        factor = np.float32(lib.snb_lj_long_range_factor(lj))
    finally:
        lib.snb_nl_destroy(nl)
        lib.snb_lj_destroy(lj)
        lib.snb_pme_destroy(pme)
    host = lambda x: x.cpu().numpy()  # noqa: E731
    # the adapter sums in double, one atom after another
    direct_e = np.float32(np.cumsum(host(direct).astype(np.float64))[-1])
    corr_e = np.float32(np.cumsum(host(corr).astype(np.float64))[-1])
    lj_long = np.float32(factor / volume)
    prints = [lj_sum.value, lj_long, np.float32(lj_sum.value) + lj_long, None, direct_e,
              np.float32(rec.value), np.float32(slf.value), corr_e, np.float32(beta)]
    prints[3] = (np.float32(direct_e) + np.float32(rec.value) + np.float32(slf.value)
                 + np.float32(corr_e))
    return dict(frc=host(frc), atom_energy=host(energy), atom_virial=host(atom_vir),
                virial=host(vir), potential=host(pot),
                prints=np.array(prints, np.float32), beta=beta)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(ADAPTER_SO), reason="adapter library not built")
def test_adapter_matches_c_abi(tmp_path):
    out = tmp_path / "adapter.npz"
    r = subprocess.run([sys.executable, os.path.abspath(__file__), str(out)], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
    got = np.load(out)
    assert int(got["rc"]) == 0
    s = _system()
    want = run_c_abi(s)
    for k in ("frc", "atom_energy", "atom_virial", "virial", "potential"):
        assert np.array_equal(got[k], want[k]), k
    for i, name in enumerate(PRINTS):
        assert got["prints"][i] == want["prints"][i], (name, got["prints"][i],
                                                        want["prints"][i])

    # and the forces are the path's: held to the FP64 oracle
    from oracle.oracle import Oracle
    from sponge_b200 import systems
    o = Oracle()
    beta = want["beta"]
    rs, cols = o.nl_pairs_system(s, CUTOFF, SKIN)
    ref = (o.direct_f64(s, CUTOFF, beta, rs, cols)["frc"] + o.excluded_f64(s, beta)["frc"]
           + o.pme_f64(s, (systems.fft_size(s.box),) * 3, beta)["frc"])
    f = got["frc"].reshape(-1, 3).astype(np.float64)
    assert np.linalg.norm(f - ref) / np.linalg.norm(ref) < 1e-5


if __name__ == "__main__":
    run_adapter(sys.argv[1])
