"""A four-site (TIP4P-Ew-like) water box for the virtual-site tests: the
flexible 3-site box of sponge_b200.systems with a massless, LJ-free site M
per water at O + a r_OH1 + b r_OH2 (a virtual atom of type 2), carrying the
negative charge; O keeps its LJ and no charge."""

import math

import numpy as np

from sponge_b200 import systems

Q_H, Q_M = 0.52422, -1.04844          # TIP4P-Ew charges (e)
R_OM = 0.125                          # O-M distance (A)


def site_coefficient():
    """a = b placing M on the bisector at R_OM for the model's geometry."""
    half = 0.5 * systems.ANGLE_T0
    return R_OM / (2.0 * systems.BOND_R0 * math.cos(half))


def tip4p_box(n_waters, seed=0):
    """(System with 4 n sites, virtual-atom records) -- the M sites appended
    after the 3 n atoms, in water order."""
    s = systems.water_box(n_waters, seed=seed)
    n3 = s.n
    ab = np.float32(site_coefficient())
    o = np.arange(0, n3, 3)
    m_idx = n3 + np.arange(n_waters)
    crd = np.concatenate([s.crd, s.crd[o] + ab * (s.crd[o + 1] - s.crd[o]) +
                          ab * (s.crd[o + 2] - s.crd[o])]).astype(np.float32)
    charge = np.concatenate([s.charge, np.zeros(n_waters, np.float32)])
    charge[o] = 0.0
    charge[o + 1] = charge[o + 2] = np.float32(Q_H) * systems.CHARGE_SCALE
    charge[m_idx] = np.float32(Q_M) * systems.CHARGE_SCALE
    lj_type = np.concatenate([s.lj_type, np.ones(n_waters, np.int32)])
    mass = np.concatenate([s.mass, np.zeros(n_waters, np.float32)])
    vel = np.concatenate([s.vel, np.zeros((n_waters, 3), np.float32)])
    excl = [[] for _ in range(n3 + n_waters)]
    for w in range(n_waters):
        a, m = 3 * w, n3 + w
        excl[a] = [a + 1, a + 2, m]
        excl[a + 1] = [a + 2, m]
        excl[a + 2] = [m]
    numbers = np.array([len(e) for e in excl], np.int32)
    start = np.zeros(len(excl), np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    flat = np.array([j for e in excl for j in e], np.int32)
    out = systems.System(crd=crd, vel=vel.astype(np.float32), charge=charge.astype(np.float32),
                         lj_type=lj_type, lj_A=s.lj_A, lj_B=s.lj_B, mass=mass.astype(np.float32),
                         excl_start=start, excl_numbers=numbers, excl_list=flat,
                         bonds=s.bonds, angles=s.angles, box=s.box)
    records = (np.full(n_waters, 2, np.int32), m_idx.astype(np.int32),
               np.stack([o, o + 1, o + 2], 1).astype(np.int32),
               np.tile(np.array([ab, ab], np.float32), (n_waters, 1)))
    return out, records
