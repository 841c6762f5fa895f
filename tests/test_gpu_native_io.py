"""The engine fed from SPONGE's native input files (read through snb_read_*)
against the same box from in-memory arrays, and the binary force
trajectory (snb_append_frc_traj) read back."""

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


def test_engine_from_native_files(g, box_9k, tmp_path):
    import copy
    import torch
    from tests import test_cpu_native_io as nio
    s = box_9k
    paths = {"LJ_in_file": str(tmp_path / "lj.txt"), "charge_in_file": str(tmp_path / "q.txt"),
             "exclude_in_file": str(tmp_path / "excl.txt")}
    nio.write_lj(paths["LJ_in_file"], s)
    nio.write_per_atom(paths["charge_in_file"], s.charge, "{:.9g}")
    nio.write_excl(paths["exclude_in_file"], s)
    t, A, B, typ = nio.read_lj(paths["LJ_in_file"])
    st, num, lst = nio.read_excl(paths["exclude_in_file"])
    q = nio.read_floats("snb_read_charge_in_file", paths["charge_in_file"])
    f = copy.deepcopy(s)
    f.n_types, f.lj_A, f.lj_B, f.lj_type = t, A, B, typ
    f.excl_start, f.excl_numbers, f.excl_list = st, num, lst
    f.charge = q
    lib = g.capi.load()
    crd = g.dev(s.crd.reshape(-1), np.float32)
    out = []
    for box in (s, f):
        e = g.engine_create(box, 8.0)
        frc = torch.zeros(3 * s.n, dtype=torch.float32, device="cuda")
        try:
            g.capi.check(lib.snb_engine_force(e, g.ptr(crd), g.ptr(frc), 0, 0, 0, None,
                                              g.stream()), "engine_force")
            torch.cuda.synchronize()
        finally:
            lib.snb_engine_destroy(e)
        out.append(frc)
    # the files carry the tables to 9 significant digits
    assert g.rel_rms(out[1].cpu().numpy(), out[0].cpu().numpy()) <= 1e-6
    # two frames of the force trajectory
    path = str(tmp_path / "frc.dat").encode()
    for frc in out:
        g.capi.check(lib.snb_append_frc_traj(path, g.ptr(frc), s.n, g.stream()), "frc_traj")
    traj = np.fromfile(path.decode(), np.float32).reshape(2, s.n, 3)
    assert np.array_equal(traj[0], out[0].cpu().numpy().reshape(-1, 3))
    assert np.array_equal(traj[1], out[1].cpu().numpy().reshape(-1, 3))
