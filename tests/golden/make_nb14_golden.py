"""Golden vectors of the 1-4 terms (NON_BOND_14, nb14/nb14.cpp:8-103), made by
the reference's own NON_BOND_14 compiled from its sources into oracle/_ref
(the exact-arithmetic build):

  nb14_alanine_dipeptide.npz   the 1-4 pairs of the Amber comparison case
      (amber_alanine_dipeptide_tip4pew_iter0.npz): each dihedral whose third
      index is not negative gives the pair (first, fourth atom) with
      A' = B' scale 1 / SCNB times the pair's LJ table entry and Coulomb scale
      1 / SCEE, as the reference's Amber loader stores them;
  nb14_water_box.npz           seeded pairs of a 300-water box at 2.5-6 A,
      many across the periodic boundary, with scale factors from a small set
      and a few atoms uncharged (the reference's 1e-10 charge floor).

Each file holds the inputs (coordinates, charges, cell, pairs and their
parameters) and the reference's forces, per-atom energies and virials and the
two energy sums.  Needs oracle/_ref (this container):

    python tests/golden/make_nb14_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


class Box:
    """What the reference run needs of a system: atoms and a cell."""

    def __init__(self, crd, charge, cell, rcell):
        self.crd, self.charge = np.asarray(crd, np.float32), np.asarray(charge, np.float32)
        self.n = len(self.crd)
        self._cell, self._rcell = np.asarray(cell, np.float32), np.asarray(rcell, np.float32)

    def cell(self):
        return self._cell

    def rcell(self):
        return self._rcell


def amber_pairs(z):
    """SPONGE's 1-4 list of the Amber case: (a, b, A', B', c)."""
    d = z["dihedrals"]
    d = d[d[:, 2] >= 0]
    a = (np.abs(d[:, 0]) // 3).astype(np.int32)
    b = (np.abs(d[:, 3]) // 3).astype(np.int32)
    t = d[:, 4] - 1
    lj_scale = (1.0 / z["scnb"][t]).astype(np.float32)
    cf = (1.0 / z["scee"][t]).astype(np.float32)
    ta, tb = z["lj_type"][a], z["lj_type"][b]
    lo, hi = np.minimum(ta, tb), np.maximum(ta, tb)
    k = hi * (hi + 1) // 2 + lo
    A = (lj_scale * z["lj_A"][k]).astype(np.float32)
    B = (lj_scale * z["lj_B"][k]).astype(np.float32)
    return a, b, A, B, cf


def water_pairs(s, m, seed):
    """m pairs of atoms 2.5-6 A apart (minimum image) in box s."""
    rng = np.random.default_rng(seed)
    L = np.float64(s.box)
    x = s.crd.astype(np.float64)
    a_out, b_out = [], []
    while len(a_out) < m:
        i = int(rng.integers(s.n))
        d = x - x[i]
        d -= np.round(d / L) * L
        r = np.sqrt((d * d).sum(1))
        cand = np.nonzero((r > 2.5) & (r < 6.0))[0]
        if len(cand) == 0:
            continue
        a_out.append(i)
        b_out.append(int(rng.choice(cand)))
    a = np.array(a_out, np.int32)
    b = np.array(b_out, np.int32)
    lj_scale = rng.choice(np.float32([0.5, 1.0 / 1.2, 1.0]), m).astype(np.float32)
    cf = rng.choice(np.float32([0.5, 1.0 / 1.2, 1.0]), m).astype(np.float32)
    ta, tb = s.lj_type[a], s.lj_type[b]
    lo, hi = np.minimum(ta, tb), np.maximum(ta, tb)
    k = hi * (hi + 1) // 2 + lo
    A = (lj_scale * s.lj_A[k]).astype(np.float32)
    B = (lj_scale * s.lj_B[k]).astype(np.float32)
    return a, b, A, B, cf


def run_reference(box, a, b, A, B, cf):
    from oracle import oracle as om
    ref = om.ReferenceCPU(exact=True)
    return ref.nb14(box, a, b, A, B, cf)


def save(name, box, a, b, A, B, cf):
    r = run_reference(box, a, b, A, B, cf)
    path = os.path.join(HERE, name)
    np.savez_compressed(path, crd=box.crd, charge=box.charge, cell=box.cell(),
                        rcell=box.rcell(), atom_a=a, atom_b=b, A=A, B=B, cf=cf,
                        ref_frc=r["frc"], ref_atom_energy=r["atom_energy"],
                        ref_virial=r["virial"], ref_lj=np.float64(r["lj"]),
                        ref_ee=np.float64(r["ee"]))
    print(path, os.path.getsize(path), "bytes;", len(a), "pairs; LJ", r["lj"], "EE", r["ee"])


def main():
    from sponge_b200 import systems
    z = np.load(os.path.join(HERE, "amber_alanine_dipeptide_tip4pew_iter0.npz"))
    L = np.asarray(z["box"], np.float32)
    box = Box(z["crd"], z["charge"], [L[0], 0, L[1], 0, 0, L[2]],
              [np.float32(1) / L[0], 0, np.float32(1) / L[1], 0, 0, np.float32(1) / L[2]])
    save("nb14_alanine_dipeptide.npz", box, *amber_pairs(z))

    s = systems.water_box(300, seed=3)
    q = s.charge.copy()
    rng = np.random.default_rng(4)
    q[rng.choice(s.n, 12, replace=False)] = 0.0
    box = Box(s.crd, q, s.cell(), s.rcell())
    save("nb14_water_box.npz", box, *water_pairs(s, 600, seed=5))


if __name__ == "__main__":
    main()
