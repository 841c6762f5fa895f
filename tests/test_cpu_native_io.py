"""SPONGE's native text inputs read through the C ABI (snb_read_*; host code,
no GPU) against the reference's own loaders (xponge/load/native/*.hpp in
oracle/_ref) on files written here from seeded boxes: the same arrays bit
for bit, and the reference's errors on malformed files."""

import ctypes
import os

import numpy as np
import pytest


def _write(path, header, *blocks):
    with open(path, "w") as f:
        f.write(header + "\n")
        for b in blocks:
            for row in b:
                f.write(row + "\n")


def write_lj(path, s):
    """LJ_in_file: "N T", A = A'/12 and B = B'/6 per type pair, N types."""
    A = np.asarray(s.lj_A, np.float64) / 12.0
    B = np.asarray(s.lj_B, np.float64) / 6.0
    _write(path, f"{s.n} {s.n_types}", [f"{a:.9g}" for a in A], [f"{b:.9g}" for b in B],
           [str(int(t)) for t in s.lj_type])


def write_soft(path, n, sc):
    AA, AB = np.asarray(sc.AA, np.float64) / 12.0, np.asarray(sc.AB, np.float64) / 6.0
    BA, BB = np.asarray(sc.BA, np.float64) / 12.0, np.asarray(sc.BB, np.float64) / 6.0
    _write(path, f"{n} {sc.n_types_A} {sc.n_types_B}",
           [f"{x:.9g}" for x in AA], [f"{x:.9g}" for x in AB],
           [f"{x:.9g}" for x in BA], [f"{x:.9g}" for x in BB],
           [f"{int(a)} {int(b)}" for a, b in zip(sc.type_A, sc.type_B)])


def write_per_atom(path, values, fmt):
    _write(path, str(len(values)), [fmt.format(v) for v in values])


def write_excl(path, s):
    rows = []
    for i in range(s.n):
        a, c = int(s.excl_start[i]), int(s.excl_numbers[i])
        rows.append(" ".join([str(c)] + [str(int(j)) for j in s.excl_list[a:a + c]]))
    _write(path, f"{s.n} {len(s.excl_list)}", rows)


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    from sponge_b200 import systems
    d = tmp_path_factory.mktemp("native")
    s, sc = systems.soft_core_box(300, n_solute=16, seed=1)
    paths = {"LJ_in_file": d / "lj.txt", "LJ_soft_core_in_file": d / "lj_soft.txt",
             "charge_in_file": d / "charge.txt", "mass_in_file": d / "mass.txt",
             "exclude_in_file": d / "excl.txt", "subsys_division_in_file": d / "subsys.txt"}
    write_lj(paths["LJ_in_file"], s)
    write_soft(paths["LJ_soft_core_in_file"], s.n, sc)
    write_per_atom(paths["charge_in_file"], s.charge, "{:.9g}")
    write_per_atom(paths["mass_in_file"], s.mass, "{:.9g}")
    write_excl(paths["exclude_in_file"], s)
    write_per_atom(paths["subsys_division_in_file"], sc.mask, "{:d}")
    return s, sc, {k: str(v) for k, v in paths.items()}


def _lib():
    from sponge_b200 import capi
    return capi, capi.load()


def _ref():
    from oracle import oracle as om
    if not os.path.exists(om.REF_SO):
        pytest.skip("oracle/_ref not built here")
    return om.ReferenceCPU(exact=False)


def read_lj(path):
    capi, lib = _lib()
    n, t = ctypes.c_int(0), ctypes.c_int(0)
    capi.check(lib.snb_read_lj_in_file(path.encode(), ctypes.byref(n), ctypes.byref(t),
                                       None, None, None), "read_lj")
    p = t.value * (t.value + 1) // 2
    A, B = np.zeros(p, np.float32), np.zeros(p, np.float32)
    typ = np.zeros(n.value, np.int32)
    capi.check(lib.snb_read_lj_in_file(path.encode(), ctypes.byref(n), ctypes.byref(t),
                                       A.ctypes.data, B.ctypes.data, typ.ctypes.data),
               "read_lj")
    return t.value, A, B, typ


def read_excl(path):
    capi, lib = _lib()
    n, m = ctypes.c_int(0), ctypes.c_int(0)
    capi.check(lib.snb_read_exclude_in_file(path.encode(), ctypes.byref(n), ctypes.byref(m),
                                            None, None, None), "read_excl")
    st, num = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)
    lst = np.zeros(max(m.value, 1), np.int32)
    capi.check(lib.snb_read_exclude_in_file(path.encode(), ctypes.byref(n), ctypes.byref(m),
                                            st.ctypes.data, num.ctypes.data, lst.ctypes.data),
               "read_excl")
    return st, num, lst[:m.value]


def read_floats(fn, path):
    capi, lib = _lib()
    n = ctypes.c_int(0)
    capi.check(getattr(lib, fn)(path.encode(), ctypes.byref(n), None), fn)
    out = np.zeros(n.value, np.float32)
    capi.check(getattr(lib, fn)(path.encode(), ctypes.byref(n), out.ctypes.data), fn)
    return out


def test_native_inputs_match_reference_loaders(files):
    s, sc, paths = files
    capi, lib = _lib()
    ref = _ref()
    ref.native_load(paths)
    t, A, B, typ = read_lj(paths["LJ_in_file"])
    assert t == s.n_types
    assert np.array_equal(A, ref.native_get("lj_A"))
    assert np.array_equal(B, ref.native_get("lj_B"))
    assert np.array_equal(typ, ref.native_get("lj_type", np.int32))
    # the file round trip is within float rounding of the stored tables
    assert np.allclose(A, s.lj_A, rtol=1e-6) and np.array_equal(typ, s.lj_type)
    st, num, lst = read_excl(paths["exclude_in_file"])
    assert np.array_equal(num, ref.native_get("excl_numbers", np.int32))
    assert np.array_equal(lst, ref.native_get("excl_list", np.int32))
    assert np.array_equal(st, s.excl_start) and np.array_equal(lst, s.excl_list)
    q = read_floats("snb_read_charge_in_file", paths["charge_in_file"])
    m = read_floats("snb_read_mass_in_file", paths["mass_in_file"])
    assert np.array_equal(q, ref.native_get("charge"))
    assert np.array_equal(m, ref.native_get("mass"))
    # soft core and subsystem division
    n, ta, tb = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    path = paths["LJ_soft_core_in_file"].encode()
    capi.check(lib.snb_read_lj_soft_core_in_file(path, ctypes.byref(n), ctypes.byref(ta),
                                                 ctypes.byref(tb), None, None, None, None,
                                                 None, None), "read_soft")
    pa, pb = ta.value * (ta.value + 1) // 2, tb.value * (tb.value + 1) // 2
    arr = [np.zeros(pa, np.float32), np.zeros(pa, np.float32), np.zeros(pb, np.float32),
           np.zeros(pb, np.float32), np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)]
    capi.check(lib.snb_read_lj_soft_core_in_file(path, ctypes.byref(n), ctypes.byref(ta),
                                                 ctypes.byref(tb),
                                                 *[a.ctypes.data for a in arr]), "read_soft")
    for a, key in zip(arr, ("AA", "AB", "BA", "BB", "type_A", "type_B")):
        assert np.array_equal(a, ref.native_get(key, a.dtype)), key
    mask = np.zeros(n.value, np.int32)
    nn = ctypes.c_int(0)
    capi.check(lib.snb_read_subsys_division_in_file(
        paths["subsys_division_in_file"].encode(), ctypes.byref(nn), mask.ctypes.data),
        "read_subsys")
    assert np.array_equal(mask, ref.native_get("subsys", np.int32))
    assert np.array_equal(mask, sc.mask)


def test_native_inputs_reject_malformed_files(files, tmp_path):
    capi, lib = _lib()
    _, _, paths = files
    n, t = ctypes.c_int(0), ctypes.c_int(0)
    # a truncated LJ table
    lines = open(paths["LJ_in_file"]).read().split("\n")
    bad = tmp_path / "lj_bad.txt"
    bad.write_text("\n".join(lines[:5]))
    A, B = np.zeros(1000, np.float32), np.zeros(1000, np.float32)
    typ = np.zeros(10000, np.int32)
    rc = lib.snb_read_lj_in_file(str(bad).encode(), ctypes.byref(n), ctypes.byref(t),
                                 A.ctypes.data, B.ctypes.data, typ.ctypes.data)
    assert rc == capi.SNB_ERR_BAD_INPUT
    assert b"LJ_in_file is not right" in lib.snb_last_error()
    # an exclusion file whose total does not match its rows
    rows = open(paths["exclude_in_file"]).read().split("\n")
    hdr = rows[0].split()
    bad2 = tmp_path / "excl_bad.txt"
    bad2.write_text("\n".join([f"{hdr[0]} {int(hdr[1]) + 1}"] + rows[1:]))
    m = ctypes.c_int(0)
    st = np.zeros(int(hdr[0]), np.int32)
    num = np.zeros(int(hdr[0]), np.int32)  # held by name: the reader writes into it
    lst = np.zeros(int(hdr[1]) + 1, np.int32)
    rc = lib.snb_read_exclude_in_file(str(bad2).encode(), ctypes.byref(n), ctypes.byref(m),
                                      st.ctypes.data, num.ctypes.data, lst.ctypes.data)
    assert rc == capi.SNB_ERR_BAD_INPUT
    assert b"excluded_atom_numbers is not right" in lib.snb_last_error()
    rc = lib.snb_read_charge_in_file(str(tmp_path / "missing.txt").encode(),
                                     ctypes.byref(n), None)
    assert rc == capi.SNB_ERR_BAD_INPUT
