"""Known answer from outside this project: the reference's Amber comparison
case (alanine dipeptide in TIP4P-Ew water, 2,398 sites; sander's forces and
potential energy of the minimised frame and of two frames the reference's
test perturbs from it, cutoff 8 A, PME; the fixtures
tests/golden/amber_alanine_dipeptide_tip4pew_iter*.npz are made by
tests/golden/make_amber_golden.py).

The nonbonded part comes from the FP64 oracle of this path (LJ + direct
Coulomb over the neighbor-list pairs within the cutoff, PME reciprocal,
excluded correction, LJ tail term), with the TIP4P-Ew extra points as charged
sites.  The bonded part (bonds, angles, dihedrals with their 1-4 terms scaled
by SCNB / SCEE) is evaluated here in FP64; its forces by central differences.
Comparison as the reference's own test does it
(benchmarks/comparison/tests/amber/tests/comp_alanine_dipeptide.py:86-92):
each water's net force and each other atom's force; |dE| <= 0.5 kcal/mol,
max |dF| <= 0.10, RMS dF <= 0.03 kcal/mol/A, cosine >= 0.999.  Amber moves
the extra points' forces onto their waters' atoms, which leaves the net
force of each water unchanged.
"""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FRAMES = [0, 1, 2]  # the minimised frame and its 0.02 / 0.05 A perturbations


def load_amber(iteration=0):
    from sponge_b200 import systems

    z = np.load(os.path.join(HERE, "golden",
                             f"amber_alanine_dipeptide_tip4pew_iter{iteration}.npz"))

    class RectSystem(systems.System):
        """A rectangular box of lengths `lengths`."""

        def cell(self):
            Lx, Ly, Lz = (np.float32(v) for v in self.lengths)
            return np.array([Lx, 0, Ly, 0, 0, Lz], np.float32)

        def rcell(self):
            Lx, Ly, Lz = (np.float32(1.0) / np.float32(v) for v in self.lengths)
            return np.array([Lx, 0, Ly, 0, 0, Lz], np.float32)

    s = RectSystem(
        crd=z["crd"], vel=np.zeros_like(z["crd"]), charge=z["charge"], lj_type=z["lj_type"],
        lj_A=z["lj_A"], lj_B=z["lj_B"], mass=z["mass"], excl_start=z["excl_start"],
        excl_numbers=z["excl_numbers"], excl_list=z["excl_list"],
        bonds=np.zeros((0, 2), np.int32), angles=np.zeros((0, 3), np.int32),
        box=float(z["box"][0]), n_types=int(z["n_types"]))
    s.lengths = [float(v) for v in z["box"]]
    return s, z


def grid_of(s):
    from sponge_b200 import systems
    return tuple(systems.fft_size(L) for L in s.lengths)


def nonbonded_f64(oracle, s, cutoff=8.0, skin=2.0):
    beta = oracle.get_beta(cutoff)
    rs, cols = oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    e = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, grid_of(s), beta)
    V = float(np.prod(np.float32(s.lengths)))
    lrc = oracle.lrc_factor(s, cutoff) / V
    energy = (d["lj_energy"].sum() + d["coulomb_energy"].sum() + e["atom_energy"].sum()
              + p["e_recip"] + p["e_self"] + lrc)
    return d["frc"] + e["frc"] + p["frc"], energy


def _dihedral(p0, p1, p2, p3):
    b0, b1, b2 = p0 - p1, p2 - p1, p3 - p2
    b1n = b1 / np.linalg.norm(b1, axis=-1, keepdims=True)
    v = b0 - (b0 * b1n).sum(-1, keepdims=True) * b1n
    w = b2 - (b2 * b1n).sum(-1, keepdims=True) * b1n
    x = (v * w).sum(-1)
    y = (np.cross(b1n, v) * w).sum(-1)
    return np.arctan2(y, x)


def bonded_energy(z, x, atoms=None):
    """Amber's bonded energy (k (r - r0)^2, k (theta - theta0)^2,
    k (1 + cos(n phi - phase)), and the 1-4 LJ / SCNB + Coulomb / SCEE of the
    dihedrals whose third index is not negative) at coordinates x (FP64).
    `atoms`: only the terms that touch these atoms."""
    L = np.asarray(z["box"], np.float64)

    def disp(a, b):
        d = x[a] - x[b]
        return d - np.round(d / L) * L

    def keep(idx):
        return np.ones(len(idx), bool) if atoms is None else np.isin(idx, atoms).any(1)

    e = 0.0
    b = np.abs(z["bonds"])
    m = keep(b[:, :2] // 3)
    i, j, t = b[m, 0] // 3, b[m, 1] // 3, b[m, 2] - 1
    r = np.linalg.norm(disp(i, j), axis=1)
    e += (z["bond_k"][t] * (r - z["bond_r0"][t]) ** 2).sum()
    a = np.abs(z["angles"])
    m = keep(a[:, :3] // 3)
    i, j, k, t = a[m, 0] // 3, a[m, 1] // 3, a[m, 2] // 3, a[m, 3] - 1
    u, w = disp(i, j), disp(k, j)
    c = (u * w).sum(1) / np.linalg.norm(u, axis=1) / np.linalg.norm(w, axis=1)
    th = np.arccos(np.clip(c, -1.0, 1.0))
    e += (z["angle_k"][t] * (th - z["angle_t0"][t]) ** 2).sum()
    d = z["dihedrals"]
    m = keep(np.abs(d[:, :4]) // 3)
    d = d[m]
    i, j, k, l4 = (np.abs(d[:, c]) // 3 for c in range(4))
    t = d[:, 4] - 1
    p1 = x[j]
    p0 = p1 + disp(i, j)
    p2 = p1 + disp(k, j)
    p3 = p2 + disp(l4, k)
    phi = _dihedral(p0, p1, p2, p3)
    e += (z["dih_k"][t] * (1.0 + np.cos(z["dih_n"][t] * phi - z["dih_phase"][t]))).sum()
    one4 = d[:, 2] >= 0
    i, l4, t = i[one4], l4[one4], t[one4]
    r = np.linalg.norm(disp(i, l4), axis=1)
    ti, tl = z["lj_type"][i], z["lj_type"][l4]
    ab = z["nb_index"][ti, tl]
    lj = z["acoef"][ab] / r ** 12 - z["bcoef"][ab] / r ** 6
    q = z["charge"].astype(np.float64)
    e += (lj / z["scnb"][t]).sum() + (q[i] * q[l4] / r / z["scee"][t]).sum()
    return float(e)


def bonded_forces(z, x, atoms, h=1e-5):
    """-dE/dx of the bonded energy for `atoms` by central differences."""
    f = np.zeros((len(x), 3))
    for a in atoms:
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, c] += h
            xm[a, c] -= h
            f[a, c] = -(bonded_energy(z, xp, atoms) - bonded_energy(z, xm, atoms)) / (2 * h)
    return f


def entity_forces(z, f):
    """Each water residue's net force, then each other atom's force."""
    ptr = list(z["residue_pointer"]) + [len(f)]
    out = []
    for r, name in enumerate(z["residue_label"]):
        a, b = ptr[r], ptr[r + 1]
        if name in ("WAT", "HOH"):
            out.append(f[a:b].sum(0))
        else:
            out.extend(f[a:b])
    return np.asarray(out)


def compare(z, f_total, e_total):
    ref = entity_forces(z, np.asarray(z["amber_forces"], np.float64))
    got = entity_forces(z, f_total)
    diff = got - ref
    stats = dict(max_abs=float(np.abs(diff).max()),
                 rms=float(np.sqrt((diff ** 2).sum(1).mean())),
                 cos=float((got * ref).sum() / np.linalg.norm(got) / np.linalg.norm(ref)),
                 de=abs(e_total - float(z["amber_epot"])))
    return stats


def solute_atoms(z):
    ptr = list(z["residue_pointer"]) + [len(z["crd"])]
    return [a for r, name in enumerate(z["residue_label"]) if name not in ("WAT", "HOH")
            for a in range(ptr[r], ptr[r + 1])]


@pytest.mark.parametrize("iteration", FRAMES)
def test_oracle_matches_amber_known_answer(oracle, iteration):
    s, z = load_amber(iteration)
    f_nb, e_nb = nonbonded_f64(oracle, s)
    x = np.asarray(z["crd64"], np.float64)
    f_b, e_b = bonded_forces(z, x, solute_atoms(z)), bonded_energy(z, x)
    st = compare(z, f_nb + f_b, e_nb + e_b)
    print(f"\nAmber TIP4P-Ew alanine dipeptide frame {iteration}, FP64 oracle: "
          f"|dE| {st['de']:.4f}, "
          f"max |dF| {st['max_abs']:.4f}, RMS dF {st['rms']:.4f}, cos {st['cos']:.6f}")
    assert st["de"] <= 0.5
    assert st["max_abs"] <= 0.10
    assert st["rms"] <= 0.03
    assert st["cos"] >= 0.999
