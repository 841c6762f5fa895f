"""Seeded synthetic water / NaCl boxes in SPONGE's internal units.

The boxes stand in for the reference's benchmark inputs (no external dataset is
used).  Units follow SPONGE (``SPONGE/common.h``): length in Angstrom, energy in
kcal/mol, charges pre-multiplied by 18.2223 so that q_i*q_j/r is kcal/mol, time
step in internal units (1 ps = 20.455 units).  LJ pair tables are stored the way
``Xponge::Native_Load_LJ`` leaves them (``xponge/load/native/lj.hpp:47,57``):
A' = 12 * 4*eps*sigma^12 and B' = 6 * 4*eps*sigma^6, indexed by the triangular
pair index of ``Get_LJ_Type`` (``Lennard_Jones_force.h:19-28``).

Geometry rule: stated molecule counts at 1.0 g/cm^3, box length from the
density, PME grid from ``Get_Fft_Patameter(L / 1.0)`` (``common.cpp:639-659``).
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

CHARGE_SCALE = np.float32(18.2223)          # common.h CONSTANT_SPONGE_CHARGE_SCALE
TIME_CONVERSION = 20.455                    # common.h CONSTANT_TIME_CONVERTION
KB = 0.00198716                             # common.h CONSTANT_kB (kcal/mol/K)
AVOGADRO = 6.02214076e23
WATER_VOLUME_A3 = 18.01528 / AVOGADRO * 1e24  # volume of one molecule at 1 g/cm^3

# LJ atom types: 0 O, 1 H (no LJ), 2 Na+, 3 Cl-
LJ_SIGMA = np.array([3.1507, 0.0, 2.439, 4.478])
LJ_EPS = np.array([0.1521, 0.0, 0.0874, 0.0355])
MASS = np.array([15.9994, 1.008, 22.98977, 35.453])
CHARGE_E = {"O": -0.834, "H": 0.417, "Na": 1.0, "Cl": -1.0}

BOND_K, BOND_R0 = 553.0, 0.9572
ANGLE_K, ANGLE_T0 = 100.0, math.radians(104.52)


def lj_pair_index(a: int, b: int) -> int:
    """Triangular pair index max*(max+1)/2 + min (Get_LJ_Type)."""
    hi, lo = max(a, b), min(a, b)
    return hi * (hi + 1) // 2 + lo


def lj_tables(n_types: int = 4):
    """Lorentz-Berthelot mixed A'/B' tables as float32 in SPONGE's stored form."""
    npair = n_types * (n_types + 1) // 2
    A = np.zeros(npair, np.float32)
    B = np.zeros(npair, np.float32)
    for a in range(n_types):
        for b in range(a + 1):
            eps = math.sqrt(LJ_EPS[a] * LJ_EPS[b])
            if eps == 0.0:
                continue
            sig = 0.5 * (LJ_SIGMA[a] + LJ_SIGMA[b])
            k = lj_pair_index(a, b)
            A[k] = np.float32(4.0 * eps * sig ** 12) * np.float32(12.0)
            B[k] = np.float32(4.0 * eps * sig ** 6) * np.float32(6.0)
    return A, B


def check_2357(n: int) -> bool:
    for p in (2, 3, 5, 7):
        while n > 1 and n % p == 0:
            n //= p
    return n == 1


def fft_size(length: float) -> int:
    """Grid size rule of Get_Fft_Patameter (common.cpp:639-659)."""
    t = (int(math.ceil(length + 3)) >> 2) << 2
    for lo, hi, v in ((60, 68, 64), (120, 136, 128), (240, 272, 256),
                      (480, 544, 512), (960, 1088, 1024)):
        if lo <= t <= hi:
            t = v
            break
    while not check_2357(t):
        t += 4
    return t


@dataclasses.dataclass
class System:
    """One periodic box, atoms in residue order (the caller's order)."""
    crd: np.ndarray          # (N, 3) float32, Angstrom
    vel: np.ndarray          # (N, 3) float32, Angstrom per internal time unit
    charge: np.ndarray       # (N,) float32, scaled by 18.2223
    lj_type: np.ndarray      # (N,) int32
    lj_A: np.ndarray         # (npair,) float32
    lj_B: np.ndarray         # (npair,) float32
    mass: np.ndarray         # (N,) float32
    excl_start: np.ndarray   # (N,) int32  one-directional (j > i) CSR, as Xponge
    excl_numbers: np.ndarray  # (N,) int32
    excl_list: np.ndarray    # (E,) int32
    bonds: np.ndarray        # (nb, 2) int32
    angles: np.ndarray       # (na, 3) int32  (H, O, H)
    box: float               # cubic box length
    n_types: int = 4

    @property
    def n(self) -> int:
        return int(self.crd.shape[0])

    def cell(self) -> np.ndarray:
        """LTMatrix3 {a11, a21, a22, a31, a32, a33} of the box."""
        L = np.float32(self.box)
        return np.array([L, 0, L, 0, 0, L], np.float32)

    def rcell(self) -> np.ndarray:
        r = np.float32(1.0) / np.float32(self.box)
        return np.array([r, 0, r, 0, 0, r], np.float32)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _orient_waters(rng, o_pos, kind, box, h_clash=1.6, max_rounds=200):
    """Uniformly random orientations, redrawn for the molecules whose H atoms
    come closer than `h_clash` A to an atom of another molecule (rejection
    sampling: orientations stay uniform, conditioned on no such clash)."""
    from scipy.spatial import cKDTree
    n = len(o_pos)
    half = ANGLE_T0 / 2
    h_local = np.array([[math.sin(half), 0.0, math.cos(half)],
                        [-math.sin(half), 0.0, math.cos(half)]]) * BOND_R0
    h_pos = o_pos[:, None, :] + np.einsum("nij,kj->nki",
                                          _random_rotations(rng, n), h_local)
    water = kind == 0
    mol = np.repeat(np.arange(n), 3)
    is_h = np.tile([False, True, True], n)
    live = np.repeat(water, 3) | (np.tile([True, False, False], n))
    idx = np.nonzero(live)[0]
    redo = None
    for _ in range(max_rounds):
        pts = np.concatenate([o_pos[:, None, :], h_pos], 1).reshape(-1, 3)
        tree = cKDTree(np.mod(pts[idx], box), boxsize=box)
        if redo is None:
            pairs = tree.query_pairs(h_clash, output_type="ndarray")
        else:
            # only molecules redrawn last round can clash now: every clashing
            # pair has a redrawn member (the water owning the H), and pairs
            # between unchanged molecules were clash-free before
            moved = np.nonzero(np.isin(mol[idx], redo))[0]
            near = tree.query_ball_point(tree.data[moved], h_clash)
            pairs = np.array(sorted({(min(p, q), max(p, q))
                                     for p, row in zip(moved, near) for q in row if q != p}),
                             dtype=np.int64).reshape(-1, 2)
        if len(pairs) == 0:
            break
        a, b = idx[pairs[:, 0]], idx[pairs[:, 1]]
        bad = (mol[a] != mol[b]) & (is_h[a] | is_h[b])
        redo = np.unique(np.concatenate([mol[a[bad & is_h[a]]], mol[b[bad & is_h[b]]]]))
        redo = redo[water[redo]]
        if len(redo) == 0:
            break
        h_pos[redo] = o_pos[redo, None, :] + np.einsum(
            "nij,kj->nki", _random_rotations(rng, len(redo)), h_local)
    return h_pos


def ion_pairs_for(box: float, molarity: float = 0.15) -> int:
    return int(round(molarity * box ** 3 * 1e-27 * AVOGADRO))


def water_box(n_waters: int, seed: int = 0, ion_pairs: int | None = 0,
              temperature: float = 300.0, box: float | None = None) -> System:
    """Flexible 3-site water on a jittered cubic lattice, optional NaCl.

    ``ion_pairs=None`` means 0.15 M NaCl for the box volume.  Ions replace
    randomly chosen waters (the ion sits at the oxygen site).  Orientations
    are uniformly random, redrawn where a hydrogen would sit within 1.6 A of
    another molecule.
    """
    rng = np.random.default_rng(seed)
    if box is None:
        box = (n_waters * WATER_VOLUME_A3) ** (1.0 / 3.0)
    if ion_pairs is None:
        ion_pairs = ion_pairs_for(box)
    n_side = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    spacing = box / n_side
    sites = np.sort(rng.permutation(n_side ** 3)[:n_waters])
    ix, rem = np.divmod(sites, n_side * n_side)
    iy, iz = np.divmod(rem, n_side)
    o_pos = (np.stack([ix, iy, iz], 1) + 0.5) * spacing
    o_pos += rng.uniform(-0.3, 0.3, size=o_pos.shape)
    kind = np.zeros(n_waters, np.int8)          # 0 water, 1 Na, 2 Cl
    if ion_pairs:
        pick = rng.choice(n_waters, size=2 * ion_pairs, replace=False)
        kind[pick[:ion_pairs]] = 1
        kind[pick[ion_pairs:]] = 2
    h_pos = _orient_waters(rng, o_pos, kind, box)

    crd, typ, chg, mass = [], [], [], []
    excl = []
    bonds, angles = [], []
    for m in range(n_waters):
        base = len(crd)
        if kind[m] == 0:
            crd.extend([o_pos[m], h_pos[m, 0], h_pos[m, 1]])
            typ.extend([0, 1, 1])
            chg.extend([CHARGE_E["O"], CHARGE_E["H"], CHARGE_E["H"]])
            mass.extend([MASS[0], MASS[1], MASS[1]])
            excl.extend([[base + 1, base + 2], [base + 2], []])
            bonds.extend([[base, base + 1], [base, base + 2]])
            angles.append([base + 1, base, base + 2])
        else:
            t = 2 if kind[m] == 1 else 3
            crd.append(o_pos[m])
            typ.append(t)
            chg.append(CHARGE_E["Na"] if t == 2 else CHARGE_E["Cl"])
            mass.append(MASS[t])
            excl.append([])
    n = len(crd)
    crd = np.asarray(crd, np.float32)
    charge = (np.asarray(chg, np.float32) * CHARGE_SCALE).astype(np.float32)
    mass = np.asarray(mass, np.float32)
    numbers = np.array([len(e) for e in excl], np.int32)
    start = np.zeros(n, np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    flat = np.array([j for e in excl for j in e], np.int32)
    # Maxwell-Boltzmann velocities in internal units (kcal/mol, g/mol -> A/unit)
    sigma = np.sqrt(KB * temperature / mass.astype(np.float64))
    vel = rng.normal(size=(n, 3)) * sigma[:, None]
    vel -= (vel * mass[:, None]).sum(0) / mass.sum()
    A, B = lj_tables(4)
    return System(crd=crd, vel=vel.astype(np.float32), charge=charge,
                  lj_type=np.asarray(typ, np.int32), lj_A=A, lj_B=B, mass=mass,
                  excl_start=start, excl_numbers=numbers, excl_list=flat,
                  bonds=np.asarray(bonds, np.int32).reshape(-1, 2),
                  angles=np.asarray(angles, np.int32).reshape(-1, 3),
                  box=float(box))


def _subset(s: System, keep: np.ndarray) -> System:
    """The atoms of `s` where `keep` (whole molecules only), re-indexed."""
    idx = np.flatnonzero(keep)
    new = -np.ones(s.n, np.int64)
    new[idx] = np.arange(len(idx))
    excl = []
    for i in idx:
        a, c = s.excl_start[i], s.excl_numbers[i]
        excl.append([int(new[j]) for j in s.excl_list[a:a + c]])
    numbers = np.array([len(e) for e in excl], np.int32)
    start = np.zeros(len(idx), np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    flat = np.array([j for e in excl for j in e], np.int32)
    bonds = s.bonds[keep[s.bonds[:, 0]]] if len(s.bonds) else s.bonds
    angles = s.angles[keep[s.angles[:, 1]]] if len(s.angles) else s.angles
    return dataclasses.replace(
        s, crd=s.crd[idx], vel=s.vel[idx], charge=s.charge[idx],
        lj_type=s.lj_type[idx], mass=s.mass[idx], excl_start=start,
        excl_numbers=numbers, excl_list=flat,
        bonds=new[bonds].astype(np.int32).reshape(-1, 2),
        angles=new[angles].astype(np.int32).reshape(-1, 3))


@dataclasses.dataclass
class SoftCore:
    """LJ_SOFT_CORE inputs of a box with an alchemical solute: end-state types
    and A'/B' tables (same stored form as the plain tables), subsystem masks
    and the charge difference B - A (scaled by 18.2223)."""
    type_A: np.ndarray
    type_B: np.ndarray
    n_types_A: int
    n_types_B: int
    AA: np.ndarray
    AB: np.ndarray
    BA: np.ndarray
    BB: np.ndarray
    mask: np.ndarray
    charge_B_A: np.ndarray


def soft_core_box(n_waters: int, n_solute: int = 64, seed: int = 0,
                  ion_pairs: int | None = None, clearance: float = 2.5):
    """A water/NaCl box with a seeded compact cluster of `n_solute` LJ sites at
    its centre (rejection-sampled at >= 2.5 A separations inside a sphere;
    sigma ~ U[3, 4] A, epsilon ~ U[0.05, 0.2] kcal/mol, charges ~ N(0, 0.3) e
    re-centred to sum 0).  Waters and ions within `clearance` of a site are
    removed.  State A has the solute's LJ sites on (one type per site,
    Lorentz-Berthelot mixing); state B turns them into a type without LJ and
    their charges off.  Returns (System, SoftCore)."""
    s = water_box(n_waters, seed=seed, ion_pairs=ion_pairs)
    rng = np.random.default_rng(50_000 + seed)
    radius = max(4.0, 1.4 * (n_solute ** (1.0 / 3.0)) * 2.5 / 1.6)
    centre = np.full(3, s.box / 2)
    sites = []
    while len(sites) < n_solute:
        p = rng.uniform(-radius, radius, 3)
        if np.linalg.norm(p) > radius:
            continue
        if all(np.linalg.norm(p - q) >= 2.5 for q in sites):
            sites.append(p)
    sites = np.asarray(sites) + centre
    # drop whole molecules near the cluster (water = O followed by its two H)
    # only atoms within radius + clearance of the centre can be near a site
    dc = s.crd.astype(np.float64) - centre
    dc -= np.round(dc / s.box) * s.box
    cand = np.nonzero(np.linalg.norm(dc, axis=1) < radius + clearance)[0]
    d = s.crd[cand][:, None, :].astype(np.float64) - sites[None]
    d -= np.round(d / s.box) * s.box
    near = np.zeros(s.n, bool)
    near[cand] = (np.linalg.norm(d, axis=2) < clearance).any(1)
    mol = np.cumsum(s.lj_type != 1) - 1  # a new molecule at every non-H atom
    m = int(mol[-1])
    drop_mol = np.zeros(m + 1, bool)
    drop_mol[mol[near]] = True
    w = _subset(s, ~drop_mol[mol])
    sig = rng.uniform(3.0, 4.0, n_solute)
    eps = rng.uniform(0.05, 0.2, n_solute)
    q = rng.normal(0.0, 0.3, n_solute)
    q -= q.mean()
    # A-state types: 0..3 water/ions, 4 + k solute site k
    nA = 4 + n_solute
    sigA = np.concatenate([LJ_SIGMA, sig])
    epsA = np.concatenate([LJ_EPS, eps])
    npA = nA * (nA + 1) // 2
    AA = np.zeros(npA, np.float32)
    AB = np.zeros(npA, np.float32)
    for a in range(nA):
        for b in range(a + 1):
            e = math.sqrt(epsA[a] * epsA[b])
            if e == 0.0:
                continue
            sg = 0.5 * (sigA[a] + sigA[b])
            k = lj_pair_index(a, b)
            AA[k] = np.float32(4.0 * e * sg ** 12) * np.float32(12.0)
            AB[k] = np.float32(4.0 * e * sg ** 6) * np.float32(6.0)
    # B-state types: 0..3 as in A, 4 a site without LJ
    nB = 5
    BA = np.zeros(nB * (nB + 1) // 2, np.float32)
    BB = np.zeros_like(BA)
    A4, B4 = lj_tables(4)
    BA[:len(A4)] = A4
    BB[:len(B4)] = B4
    n0 = w.n
    n = n0 + n_solute
    crd = np.concatenate([w.crd, sites.astype(np.float32)])
    charge = np.concatenate([w.charge, (q * CHARGE_SCALE).astype(np.float32)])
    typeA = np.concatenate([w.lj_type, 4 + np.arange(n_solute, dtype=np.int32)])
    typeB = np.concatenate([w.lj_type, np.full(n_solute, 4, np.int32)])
    mass = np.concatenate([w.mass, np.full(n_solute, 12.011, np.float32)])
    sol_vel = rng.normal(size=(n_solute, 3)) * np.sqrt(KB * 300.0 / 12.011)
    vel = np.concatenate([w.vel, sol_vel.astype(np.float32)])
    sys_ = dataclasses.replace(
        w, crd=crd.astype(np.float32), vel=vel.astype(np.float32), charge=charge,
        lj_type=typeA.astype(np.int32), lj_A=AA, lj_B=AB, mass=mass.astype(np.float32),
        excl_start=np.concatenate([w.excl_start, np.full(n_solute, len(w.excl_list),
                                                         np.int32)]).astype(np.int32),
        excl_numbers=np.concatenate([w.excl_numbers, np.zeros(n_solute, np.int32)]),
        n_types=nA)
    soft = SoftCore(type_A=typeA.astype(np.int32), type_B=typeB.astype(np.int32),
                    n_types_A=nA, n_types_B=nB, AA=AA, AB=AB, BA=BA, BB=BB,
                    mask=np.concatenate([np.zeros(n0, np.int32),
                                         np.ones(n_solute, np.int32)]),
                    charge_B_A=np.concatenate([np.zeros(n0, np.float32),
                                               -charge[n0:]]).astype(np.float32))
    return sys_, soft


def config_small(seed: int = 0) -> System:
    """3,000 waters (9,000 atoms), L = 44.77 A, grid 48^3, cutoff 8, skin 2."""
    return water_box(3000, seed=seed, ion_pairs=0)


def config_100k(seed: int = 0) -> System:
    """33,333 waters with 0.15 M NaCl replacing 180 waters: 99,639 atoms,
    L = 99.90 A, grid 100^3, cutoff 10, skin 2."""
    return water_box(33333, seed=seed, ion_pairs=None)


def batch_member_waters(seed: int) -> int:
    """Water count U[200, 2000] of the batch box with this seed."""
    rng = np.random.default_rng(10_000 + seed)
    return int(rng.integers(200, 2001))


def batch_member_size(seed: int) -> tuple[int, int]:
    """(atoms, PME grid edge) of the batch box with this seed, without
    building it."""
    nw = batch_member_waters(seed)
    box = (nw * WATER_VOLUME_A3) ** (1.0 / 3.0)
    return 3 * nw - 4 * ion_pairs_for(box), fft_size(box)  # an ion replaces a water


def config_batch_member(seed: int) -> System:
    """One box of the 256-box batch: water count U[200, 2000] from the seed."""
    return water_box(batch_member_waters(seed), seed=seed, ion_pairs=None)
