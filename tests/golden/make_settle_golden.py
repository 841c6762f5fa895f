"""Golden vectors of SETTLE (constrain/settle.cpp) made by the reference's own
SETTLE compiled from its sources into oracle/_ref (the exact-arithmetic
build), on one step of a 300-site-water box:

  settle_water_box.npz   rigid 3-site waters (O-H 0.9572 A, H-H 1.5139 A,
      the constraints listed in varied orders), ten waters constrained on
      one O-H bond only (rigid pairs), and two waters tied together by an
      extra constraint (which SETTLE leaves to SHAKE); two ion pairs stay
      unconstrained.  The step: coordinates at the rigid geometry, then
      dt v plus 0.01 A of noise, dt = 2 fs.

The file holds the inputs and the reference's coordinates, velocities,
stress (constraint virial / V), group counts and left-over pairs.  Needs
oracle/_ref (this container):

    python tests/golden/make_settle_golden.py
"""

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

R_OH = 0.9572
R_HH = 2 * 0.9572 * math.sin(math.radians(104.52) / 2)


def settle_case(n_waters=300, seed=11):
    """(system, ai, aj, r0) of the case above."""
    from sponge_b200 import systems
    s = systems.water_box(n_waters, seed=seed, ion_pairs=2)
    rng = np.random.default_rng(seed + 1)
    waters = [i for i in range(s.n - 2) if s.lj_type[i] == 0]
    ai, aj, r0 = [], [], []
    pair_only = set(rng.choice(len(waters), 10, replace=False).tolist())
    for w, o in enumerate(waters):
        h1, h2 = o + 1, o + 2
        if w in pair_only:
            rows = [(o, h1, R_OH)]
        else:
            rows = [(o, h1, R_OH), (o, h2, R_OH), (h1, h2, R_HH)]
            rng.shuffle(rows)
            rows = [(b, a, r) if rng.random() < 0.5 else (a, b, r) for a, b, r in rows]
        for a, b, r in rows:
            ai.append(a)
            aj.append(b)
            r0.append(r)
    # tie two rigid waters together: both fall to SHAKE
    full = [w for w in range(len(waters)) if w not in pair_only]
    w1, w2 = full[5], full[6]
    ai.append(waters[w1] + 2)
    aj.append(waters[w2])
    r0.append(3.0)
    return s, np.array(ai, np.int32), np.array(aj, np.int32), np.array(r0, np.float32)


def settle_step(s, seed=13):
    """(crd_old, crd_new, vel, dt) of the step."""
    from sponge_b200 import systems
    rng = np.random.default_rng(seed)
    dt = np.float32(2e-3 * systems.TIME_CONVERSION)
    crd_old = s.crd.astype(np.float32)
    vel = s.vel.astype(np.float32)
    crd_new = (crd_old + dt * vel + rng.normal(0, 0.01, crd_old.shape)).astype(np.float32)
    return crd_old, crd_new, vel, dt


def main():
    from oracle import oracle as om
    s, ai, aj, r0 = settle_case()
    crd_old, crd_new, vel, dt = settle_step(s)
    ref = om.ReferenceCPU(exact=True)
    r = ref.settle(s.cell(), ai, aj, r0, s.mass, crd_old, crd_new, vel, float(dt))
    path = os.path.join(HERE, "settle_water_box.npz")
    np.savez_compressed(path, crd_old=crd_old, crd_new=crd_new, vel=vel, dt=dt,
                        mass=s.mass, cell=s.cell(), rcell=s.rcell(), atom_i=ai, atom_j=aj,
                        constant_r=r0, ref_crd=r["crd"], ref_vel=r["vel"],
                        ref_stress=r["stress"], ref_counts=r["counts"], ref_left=r["left"])
    print(path, os.path.getsize(path), "bytes; counts", r["counts"])


if __name__ == "__main__":
    main()
