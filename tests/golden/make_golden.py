"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own CPU build of the hot-path modules (oracle/_ref,
compiled from its sources by `make -C oracle ref`) on small seeded boxes and
stores inputs and outputs.  Needs the reference sources (this container);
the committed .npz files are what the tests read everywhere else.

    python tests/golden/make_golden.py
"""

import dataclasses
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceCPU, build_oracle  # noqa: E402
from sponge_b200 import systems  # noqa: E402


def pair_digest(pairs: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(pairs, np.int32).tobytes()).hexdigest()


def reference_pairs(counts, serial):
    i = np.repeat(np.arange(len(counts)), counts)
    p = np.stack([i, serial.astype(np.int64)], 1)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def make_case(name, s, cutoff, skin):
    ref = ReferenceCPU(exact=False)
    beta = ref.init(s, cutoff, skin)
    counts, serial, ov = ref.nl_update()
    assert not ov.any()
    pairs = reference_pairs(counts, serial)
    lj = ref.lj_direct()
    pme = ref.pme_reciprocal()
    ex = ref.pme_excluded()
    V = float(np.float32(s.box) ** 3)
    lrc = ref.lj_long_range(V)
    # pair set again from the build without fast-math / FMA contraction
    ref_exact = ReferenceCPU(exact=True)
    ref_exact.init(s, cutoff, skin)
    c2, s2, _ = ref_exact.nl_update()
    pairs_exact = reference_pairs(c2, s2)
    assert np.array_equal(pairs, pairs_exact)
    out = dict(
        crd=s.crd, charge=s.charge, lj_type=s.lj_type, lj_A=s.lj_A, lj_B=s.lj_B,
        excl_start=s.excl_start, excl_numbers=s.excl_numbers, excl_list=s.excl_list,
        box=np.float64(s.box), cutoff=np.float32(cutoff), skin=np.float32(skin),
        beta=np.float32(beta), grid=np.array(ref.grid, np.int32),
        nl_counts=counts, nl_pair_total=np.int64(len(pairs)),
        nl_pair_sha256=np.array(pair_digest(pairs)),
        lj_frc=lj["frc"], lj_atom_energy=lj["atom_energy"], lj_virial=lj["virial"],
        lj_lj_energy=lj["lj_energy"], lj_coulomb_energy=lj["coulomb_energy"],
        pme_frc=pme["frc"], pme_virial=pme["virial"], pme_potential=np.float32(pme["potential"]),
        pme_e_recip=np.float32(pme["e_recip"]), pme_e_self=np.float32(pme["e_self"]),
        excl_frc=ex["frc"], excl_atom_energy=ex["atom_energy"], excl_virial=ex["virial"],
        lrc_factor=np.float32(lrc["factor"]), lrc_potential=np.float32(lrc["potential"]),
        lrc_virial=lrc["virial"],
    )
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(pairs), "pairs")


def make_soft_case(name, s, sc, cutoff, skin, params):
    """LJ_SOFT_CORE on a box with an alchemical solute: forces, the energy
    split, virial, dH/dlambda and the tail factors from the reference."""
    ref = ReferenceCPU(exact=False)
    beta = ref.init(s, cutoff, skin)
    ref.soft_init(sc, params)
    counts, serial, ov = ref.nl_update()
    assert not ov.any()
    pairs = reference_pairs(counts, serial)
    r = ref.soft_direct()
    dhdl = ref.soft_dhdl(sc.charge_B_A)
    V = float(np.float32(s.box) ** 3)
    lr = ref.soft_long_range(V)
    out = dict(
        crd=s.crd, charge=s.charge, lj_type=s.lj_type, lj_A=s.lj_A, lj_B=s.lj_B,
        excl_start=s.excl_start, excl_numbers=s.excl_numbers, excl_list=s.excl_list,
        box=np.float64(s.box), cutoff=np.float32(cutoff), skin=np.float32(skin),
        beta=np.float32(beta), nl_pair_total=np.int64(len(pairs)),
        nl_pair_sha256=np.array(pair_digest(pairs)),
        type_A=sc.type_A, type_B=sc.type_B, n_types_A=np.int32(sc.n_types_A),
        n_types_B=np.int32(sc.n_types_B), AA=sc.AA, AB=sc.AB, BA=sc.BA, BB=sc.BB,
        mask=sc.mask, charge_B_A=sc.charge_B_A,
        lam=np.float32(params["lambda_lj"]), alpha=np.float32(params["soft_core_alpha"]),
        p=np.float32(params["soft_core_powfer"]),
        sigma=np.float32(params["soft_core_sigma"]),
        sigma_min=np.float32(params["soft_core_sigma_min"]),
        frc=r["frc"], atom_energy=r["atom_energy"], virial=r["virial"],
        lj_energy=r["lj_energy"], inter=r["inter"], intra=r["intra"],
        coulomb_energy=r["coulomb_energy"], dhdl=np.float32(dhdl),
        lrc_factor=np.float32(lr["factor"]), lrc_factor_ti=np.float32(lr["factor_ti"]),
        lrc_potential=np.float32(lr["potential"]), lrc_virial=lr["virial"],
    )
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(pairs), "pairs")


def make_box_change_case(name, s, cutoff, skin, scale):
    """A barostat's box change: the reference initialised on box s.box, then
    the box and coordinates scaled by `scale` (Main_Box_Change for a small
    change: PME Update_Box at the old grid size, the list rebuilt in its old
    grid); the pair set and PME terms at the new box."""
    ref = ReferenceCPU(exact=False)
    beta = ref.init(s, cutoff, skin)
    counts, serial, ov = ref.nl_update()
    assert not ov.any()
    box1 = float(np.float32(s.box * scale))
    crd1 = (s.crd.astype(np.float64) * scale).astype(np.float32)
    ref.box_change(box1)
    counts, serial, ov = ref.nl_update(crd=crd1, forced=True)
    assert not ov.any()
    pairs = reference_pairs(counts, serial)
    pme = ref.pme_reciprocal(crd=crd1)
    # the same box and coordinates in a reference initialised there: its
    # Initial forms the virial factor (1 + pi^2 m^2 / beta^2) that Update_Box
    # (PM_force.cpp:1210-1236) forms with the opposite sign of the m^2 term
    s1 = dataclasses.replace(s, crd=crd1, box=box1)
    fresh = ReferenceCPU(exact=False)
    fresh.init(s1, cutoff, skin)
    assert fresh.grid == ref.grid
    fresh.nl_update()
    pme_fresh = fresh.pme_reciprocal()
    out = dict(
        crd=crd1, crd0=s.crd, charge=s.charge, lj_type=s.lj_type, lj_A=s.lj_A,
        lj_B=s.lj_B, excl_start=s.excl_start, excl_numbers=s.excl_numbers,
        excl_list=s.excl_list, box=np.float64(box1), box0=np.float64(s.box),
        cutoff=np.float32(cutoff), skin=np.float32(skin), beta=np.float32(beta),
        grid=np.array(ref.grid, np.int32), nl_pair_total=np.int64(len(pairs)),
        nl_pair_sha256=np.array(pair_digest(pairs)),
        pme_frc=pme["frc"], pme_virial=pme["virial"],
        pme_e_recip=np.float32(pme["e_recip"]), pme_e_self=np.float32(pme["e_self"]),
        pme_frc_fresh=pme_fresh["frc"], pme_virial_fresh=pme_fresh["virial"],
    )
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(pairs), "pairs")


def main(names=None):
    """Writes every fixture, or only those named (the fixtures differ from run
    to run at the last bit where the reference sums with OpenMP, so committed
    ones are left alone unless asked for)."""
    build_oracle()
    want = lambda n: not names or n in names  # noqa: E731
    # 216 waters, L = 18.63 A, grid 20^3, cutoff 8
    if want("water216_rc8"):
        make_case("water216_rc8", systems.water_box(216, seed=1), 8.0, 2.0)
    # 343 waters + 1 NaCl pair, cutoff 9, skin 1.5 (non-default keys)
    if want("water343_nacl_rc9"):
        make_case("water343_nacl_rc9", systems.water_box(343, seed=5, ion_pairs=1), 9.0, 1.5)
    # 300 waters + a 16-site alchemical solute; two soft-core parameter sets
    s, sc = systems.soft_core_box(300, n_solute=16, seed=1)
    if want("soft_water300_s16_lam050"):
        make_soft_case("soft_water300_s16_lam050", s, sc, 8.0, 2.0,
                       {"lambda_lj": 0.5, "soft_core_alpha": 0.5, "soft_core_powfer": 1.0,
                        "soft_core_sigma": 3.0, "soft_core_sigma_min": 0.0})
    if want("soft_water300_s16_lam025_p2"):
        make_soft_case("soft_water300_s16_lam025_p2", s, sc, 8.0, 2.0,
                       {"lambda_lj": 0.25, "soft_core_alpha": 0.7, "soft_core_powfer": 2.0,
                        "soft_core_sigma": 3.2, "soft_core_sigma_min": 3.6})
    # 343 waters + 1 NaCl pair, the box and coordinates scaled by 1.03 after
    # Initial (grid 24^3 kept)
    if want("boxchange_water343_x103"):
        make_box_change_case("boxchange_water343_x103",
                             systems.water_box(343, seed=5, ion_pairs=1), 9.0, 1.5, 1.03)


if __name__ == "__main__":
    main(sys.argv[1:])
