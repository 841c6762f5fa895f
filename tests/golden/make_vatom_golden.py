"""Golden vectors for virtual atoms from the reference's own formulas.

The reference's virtual-atom position and force functions
(virtual_atoms/virtual_atom_math.h, header-only, called record by record by
oracle/ref_build/ref_harness.cpp's ref_vatom) on two cases:

  * vatom_wat_nonortho.npz: the reference's triclinic TIP4P water case, its
    virtual_atom_in_file (WAT_virtual_atom.txt: one type-2 site per water)
    read by the reference's own loader, in its skewed cell; a seeded force
    on every site is moved onto the waters' atoms;
  * vatom_mixed.npz: 200 atoms in a 30 A box with sites of all four types
    (0 mirror, 1 on a line, 2 in a plane, 3 at a distance along a
    direction), a second layer of sites built from first-layer sites, and a
    type-3 site with d = 0; seeded forces on every atom.

Records are stored in an order where every site follows its sources.  Needs
the reference checkout, named by SPONGE_REFERENCE:

    SPONGE_REFERENCE=<reference checkout> python tests/golden/make_vatom_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def save(name, ref, records, cell, crd, frc):
    x, f, bad = ref.vatom(records, cell, crd, frc)
    assert bad == 0
    ty, vi, fr, pa = records
    np.savez_compressed(os.path.join(HERE, name), type=np.asarray(ty, np.int32),
                        virtual_atom=np.asarray(vi, np.int32), source=np.asarray(fr, np.int32),
                        parameter=np.asarray(pa, np.float32), cell=np.asarray(cell, np.float32),
                        crd_in=np.asarray(crd, np.float32), frc_in=np.asarray(frc, np.float32),
                        crd_out=x, frc_out=f)
    print(name, len(ty), "records")


def mixed_case(rng):
    n_real = 200
    L = np.float32(30.0)
    crd = (rng.random((n_real, 3)) * L).astype(np.float32)
    ty, vi, fr, pa = [], [], [], []
    nxt = n_real

    def add(t, src, p, q=0.0):
        nonlocal nxt
        ty.append(t)
        vi.append(nxt)
        fr.append(list(src) + [-1] * (3 - len(src)))
        pa.append([p, q])
        nxt += 1
        return nxt - 1

    first = []
    for k in range(20):  # layer 1: sites on real atoms
        a, b, c = rng.choice(n_real, 3, replace=False)
        first.append(add(0, [a], float(rng.uniform(5, 25))))
        first.append(add(1, [a, b], float(rng.uniform(-0.5, 1.5))))
        first.append(add(2, [a, b, c], float(rng.uniform(0, 0.5)), float(rng.uniform(0, 0.5))))
        first.append(add(3, [a, b, c], float(rng.uniform(-1.5, 1.5)),
                         float(rng.uniform(0, 1))))
    add(3, [0, 1, 2], 0.0, 0.5)  # d = 0: the site sits on atom 1
    for k in range(10):  # layer 2: sites built from first-layer sites
        a, b = rng.choice(first, 2, replace=False)
        c = int(rng.integers(0, n_real))
        add(1, [a, c], float(rng.uniform(0, 1)))
        add(2, [c, a, b], float(rng.uniform(0, 0.4)), float(rng.uniform(0, 0.4)))
    n = nxt
    x = np.zeros((n, 3), np.float32)
    x[:n_real] = crd
    x[n_real:] = crd[0]  # placeholders, overwritten by the positions pass
    frc = rng.normal(0, 10, (n, 3)).astype(np.float32)
    cell = np.array([L, 0, L, 0, 0, L], np.float32)
    return (np.array(ty), np.array(vi), np.array(fr), np.array(pa, np.float32)), cell, x, frc


def main():
    root = os.environ.get("SPONGE_REFERENCE", "")
    if not root:
        raise SystemExit("set SPONGE_REFERENCE to the reference checkout's root")
    from oracle.oracle import ReferenceCPU, build_oracle
    build_oracle(with_reference=True)
    ref = ReferenceCPU(exact=False)
    rng = np.random.default_rng(21)

    case = os.path.join(root, "benchmarks", "performance", "nonortho", "statics",
                        "WAT_nonortho")
    ref.native_load({"virtual_atom_in_file": os.path.join(case, "WAT_virtual_atom.txt")})
    m = len(ref.native_get("vatom_type", np.int32))
    records = (ref.native_get("vatom_type", np.int32), ref.native_get("vatom_virtual", np.int32),
               ref.native_get("vatom_from", np.int32).reshape(m, 3),
               ref.native_get("vatom_param").reshape(m, 2))
    w = np.load(os.path.join(HERE, "wat_nonortho_rc8.npz"))
    frc = rng.normal(0, 10, w["crd"].shape).astype(np.float32)
    save("vatom_wat_nonortho.npz", ref, records, w["cell"], w["crd"], frc)

    records, cell, x, frc = mixed_case(rng)
    save("vatom_mixed.npz", ref, records, cell, x, frc)


if __name__ == "__main__":
    main()
