"""SETTLE (constrain/settle.cpp) on the CPU: the reference's own SETTLE
(golden vectors of tests/golden/make_settle_golden.py) against the FP64
oracle, which solves the same constraint equations by iterated SHAKE.

Case: one 2 fs step of 296 waters (284 rigid triangles, 10 waters held on
one O-H bond only, two waters tied together that SETTLE leaves to SHAKE)
and two ion pairs.  Tolerances (the reference in FP32 is at about a fifth
of each): positions 1e-5 A; velocity change 1e-4 relative RMS; stress
1e-4 of its largest component; constraint lengths 1e-5 A; atoms outside
SETTLE's groups untouched."""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TOL_CRD, TOL_VEL, TOL_STRESS, TOL_LEN = 1e-5, 1e-4, 1e-4, 1e-5


def load():
    return np.load(os.path.join(HERE, "golden", "settle_water_box.npz"))


def settled_mask(z):
    """Constraints SETTLE handles: those not left over."""
    left = set(map(tuple, z["ref_left"].tolist()))
    return np.array([(a, b) not in left for a, b in zip(z["atom_i"], z["atom_j"])])


def oracle_step(oracle, z):
    k = settled_mask(z)
    return oracle.shake_f64(z["cell"], z["rcell"], z["atom_i"][k], z["atom_j"][k],
                            z["constant_r"][k].astype(np.float64),
                            z["mass"].astype(np.float64), z["crd_old"], z["crd_new"],
                            z["vel"], float(z["dt"]))


def check_against_oracle(z, o, crd, vel, stress):
    """Assertions shared by the CPU and GPU tests."""
    crd = np.asarray(crd, np.float64)
    assert np.abs(crd - o["crd"]).max() <= TOL_CRD
    dv, dv64 = np.asarray(vel, np.float64) - z["vel"], o["vel"] - z["vel"]
    assert np.linalg.norm(dv - dv64) / np.linalg.norm(dv64) <= TOL_VEL
    V = float(np.prod(1.0 / z["rcell"][[0, 2, 5]].astype(np.float64)))
    s64 = o["virial"] / V
    assert np.abs(np.asarray(stress, np.float64) - s64).max() <= TOL_STRESS * np.abs(s64).max()
    k = settled_mask(z)
    ai, aj, r0 = z["atom_i"][k], z["atom_j"][k], z["constant_r"][k]
    length = np.linalg.norm(crd[aj] - crd[ai], axis=1)
    assert np.abs(length - r0).max() <= TOL_LEN
    # atoms of no rigid group keep the unconstrained step
    moved = np.zeros(len(crd), bool)
    moved[ai] = moved[aj] = True
    assert np.array_equal(np.asarray(crd, np.float32)[~moved], z["crd_new"][~moved])


def test_reference_settle_matches_fp64_shake(oracle):
    z = load()
    o = oracle_step(oracle, z)
    assert o["sweeps"] > 0
    assert list(z["ref_counts"]) == [284, 10, 7]
    check_against_oracle(z, o, z["ref_crd"], z["ref_vel"], z["ref_stress"])


def test_oracle_keeps_rigid_bodies_rigid(oracle):
    """The oracle's step conserves each group's momentum (the constraint
    forces are internal) and puts every length back on its target."""
    z = load()
    o = oracle_step(oracle, z)
    m = z["mass"].astype(np.float64)[:, None]
    p0 = (m * z["vel"].astype(np.float64)).sum(0)
    p1 = (m * o["vel"]).sum(0)
    assert np.abs(p1 - p0).max() <= 1e-9 * np.abs(m * o["vel"]).sum()
    k = settled_mask(z)
    d = o["crd"][z["atom_j"][k]] - o["crd"][z["atom_i"][k]]
    assert np.abs(np.linalg.norm(d, axis=1) - z["constant_r"][k]).max() <= 1e-12


def test_grouping_matches_reference():
    """snb_settle_group (host code, no GPU) sorts the case's constraint pairs
    into the reference's 284 triangles, 10 rigid pairs and 7 left-over pairs,
    the same left-over pairs as the reference's SETTLE::Initial keeps."""
    import ctypes
    from sponge_b200 import capi
    z = load()
    lib = capi.load()
    ai = np.ascontiguousarray(z["atom_i"], np.int32)
    aj = np.ascontiguousarray(z["atom_j"], np.int32)
    r0 = np.ascontiguousarray(z["constant_r"], np.float32)
    mass = np.ascontiguousarray(z["mass"], np.float32)
    counts = np.zeros(3, np.int32)
    left = np.zeros(len(ai), np.int32)
    capi.check(lib.snb_settle_group(len(mass), len(ai), ai.ctypes.data, aj.ctypes.data,
                                    r0.ctypes.data, mass.ctypes.data, counts.ctypes.data,
                                    left.ctypes.data), "settle_group")
    assert list(counts) == list(z["ref_counts"])
    k = left[:counts[2]]
    assert np.array_equal(np.stack([ai[k], aj[k]], 1), z["ref_left"])
    bad = ai.copy()
    bad[0] = len(mass)
    assert lib.snb_settle_group(len(mass), len(ai), bad.ctypes.data, aj.ctypes.data,
                                r0.ctypes.data, mass.ctypes.data, counts.ctypes.data,
                                None) == capi.SNB_ERR_BAD_INPUT
