"""TEST INFRASTRUCTURE ONLY -- accuracy of an engine result against the FP64
oracle, as the -m gpu tests and the benchmark's accuracy keys report it.

The FP64 reference of one force evaluation is the oracle's run of the same
method on the same frame (oracle/snb_oracle.c): the direct LJ + erfc-Coulomb
sum over the oracle's own FP32 pair set at cutoff + skin
(Lennard_Jones_force.cpp:326-384 over neighbor_list.cpp:347-417), the PME
reciprocal part on the same grid (PM_force.cpp:1070-1168), the excluded-pair
correction (PM_force.cpp:1745-1817) and the long-range LJ correction
(Lennard_Jones_force.cpp:279-308).

Quantities (the metric's "force rel-err vs FP64"):
  force_rel_rms   ||F - F64||_2 / ||F64||_2 over all atoms and components
  energy_rel      |E - E64| / |E64| per component (LJ, LRC, direct Coulomb,
                  excluded correction, reciprocal, self) and for the sum
  virial_rel      max |W - W64| / max |W64| over the six virial components
  pressure_err_bar  |tr(W - W64)| / (3 V) in bar (the kinetic part is the
                  same velocities on both sides and cancels)
"""

from __future__ import annotations

import numpy as np

# kcal/mol/A^3 -> bar, the conversion the engine's pressure uses
BAR_PER_KCAL_MOL_A3 = 6.946827162543585e4

# slots of snb_engine_force's d_totals
TOTAL_SLOTS = {"lj": 0, "lrc": 1, "coul": 2, "excl": 3, "recip": 4, "self": 5}


def grid_of(s):
    from sponge_b200 import systems
    return (systems.fft_size(s.box),) * 3


def reference_totals(oracle, s, cutoff, skin=2.0, grid=None, rows=None):
    """FP64 forces (n, 3), energy components and virial (6,) of System s.
    rows: the oracle's (row_start, cols) pair set if already computed."""
    beta = oracle.get_beta(cutoff)
    rs, cols = rows if rows is not None else oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.direct_f64(s, cutoff, beta, rs, cols)
    e = oracle.excluded_f64(s, beta)
    p = oracle.pme_f64(s, grid or grid_of(s), beta)
    V = float(np.float32(s.box)) ** 3
    lrc = oracle.lrc_factor(s, cutoff)
    frc = d["frc"] + e["frc"] + p["frc"]
    energies = dict(lj=float(d["lj_energy"].sum()), lrc=lrc / V,
                    coul=float(d["coulomb_energy"].sum()),
                    excl=float(e["atom_energy"].sum()), recip=float(p["e_recip"]),
                    self=float(p["e_self"]))
    vir = d["virial"].sum(0) + e["virial"].sum(0) + p["virial"]
    vir[[0, 2, 5]] += 2 * lrc / V
    return frc, energies, vir


def soft_reference_forces(oracle, s, sc, cutoff, lam, alpha, p, sigma, sigma_min,
                          skin=2.0, grid=None):
    """FP64 forces (n, 3) of the soft-core engine's step on System s: the
    soft-core direct terms (LJ_soft_core.cpp:196-461) over the oracle's pair
    set, plus the PME reciprocal part and the excluded correction with s's
    charges."""
    beta = oracle.get_beta(cutoff)
    rs, cols = oracle.nl_pairs_system(s, cutoff, skin)
    d = oracle.soft_f64(s, sc, cutoff, beta, lam, alpha, p, sigma, sigma_min, rs, cols)
    e = oracle.excluded_f64(s, beta)
    pm = oracle.pme_f64(s, grid or grid_of(s), beta)
    return d["frc"] + e["frc"] + pm["frc"]


def force_rel_rms(got, want) -> float:
    got = np.asarray(got, np.float64).reshape(-1)
    want = np.asarray(want, np.float64).reshape(-1)
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def compare(frc, totals, reference, volume) -> dict:
    """Accuracy of one engine force evaluation (frc (n, 3) in the caller's
    order, totals = d_totals[0..13] of snb_engine_force with energy and
    virial) against reference_totals(...)."""
    f_want, en, vir = reference
    t = np.asarray(totals, np.float64)
    out = {"force_rel_rms": force_rel_rms(frc, f_want)}
    rel = {}
    for k, idx in TOTAL_SLOTS.items():
        rel[k] = abs(t[idx] - en[k]) / abs(en[k]) if en[k] != 0 else abs(t[idx])
    total = sum(en.values())
    rel["potential"] = abs(t[7] - total) / abs(total)
    out["energy_rel"] = rel
    out["energy_rel_max"] = max(rel.values())
    dv = t[8:14] - vir
    out["virial_rel"] = float(np.abs(dv).max() / np.abs(vir).max())
    out["pressure_err_bar"] = float(abs(dv[0] + dv[2] + dv[5]) / (3.0 * volume)
                                    * BAR_PER_KCAL_MOL_A3)
    out["pressure_bar_fp64_virial_part"] = float((vir[0] + vir[2] + vir[5]) / (3.0 * volume)
                                                 * BAR_PER_KCAL_MOL_A3)
    return out
