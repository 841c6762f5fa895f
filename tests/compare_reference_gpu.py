"""The reference's own GPU path against the fixed-point engine, timed on the
same equilibrated box (test infrastructure: the reference build under
oracle/_ref is a checker, never the product).

The reference side is its neighbor_list, Lennard_Jones_force, PM_force, bond
and angle modules compiled as CUDA (FP32 arithmetic, float atomics, legacy
default stream), driven in main.cpp's order by
oracle/ref_build/ref_harness_gpu.cu. The engine side is the fixed-point
engine with one captured graph per step. Both integrate NVE leap-frog at
0.5 fs from the same coordinates and velocities, after the engine has
equilibrated the lattice start at 300 K. Prints one JSON line:

    python tests/compare_reference_gpu.py [--waters 33333] [--steps 1000]
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def reference_drift(ref, s, inv_m, first_state, total, samples, dt):
    """Total energy every total/(samples-1) steps of the reference's GPU run:
    its per-atom energies and box terms (FP32), the bonded terms on the host
    (FP64) and the kinetic energy of the mid-step velocities. Fitted drift in
    kcal/mol/ns/atom, as the bench fits the engine's."""
    import bench
    n = s.n
    ref.set_state(first_state[0], first_state[1], inv_m)
    every = max(2, total // max(1, samples - 1))
    m = s.mass.astype(np.float64)[:, None]
    step, ts, es = 0, [], []
    for _ in range(samples):
        out = ref.force(forced=False, need_energy=True, need_virial=False)
        c0, v0 = ref.get_state()
        pot = float(out["atom_energy"].astype(np.float64).sum()) + out["potential"]
        pot += bench.bonded_energy(s, c0)
        ref.md_steps(1, dt)
        _, v1 = ref.get_state()
        ke = 0.5 * (m * (0.5 * (v0.astype(np.float64) + v1)) ** 2).sum()
        ts.append(step)
        es.append(pot + ke)
        ref.md_steps(every - 1, dt)
        step += every
    ts = np.asarray(ts, np.float64)
    es = np.asarray(es, np.float64)
    slope = np.polyfit(ts, es, 1)[0]
    return {"steps": int(ts[-1] - ts[0]), "samples": len(ts),
            "kcal_per_mol_per_ns_per_atom": slope / (bench.DT_FS * 1e-6) / n,
            "e_total_std": float(es.std())}


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--waters", type=int, default=33333)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=50)
    p.add_argument("--equilibrate", type=int, default=2000)
    p.add_argument("--drift-steps", type=int, default=2000)
    args = p.parse_args()

    import torch
    import bench
    from oracle.oracle import ReferenceGPU
    from sponge_b200 import capi, systems
    from tests import gpu_helpers as g

    s = bench.make_box(args.waters, seed=0)
    n = s.n
    lib = capi.load()
    h = g.engine_create(s, bench.CUTOFF, bench.SKIN)
    g.engine_set_water_bonded(h, s)
    crd = torch.from_numpy(s.crd.reshape(-1).copy()).cuda()
    vel = torch.from_numpy(s.vel.reshape(-1).copy()).cuda()
    inv_m = (1.0 / s.mass).astype(np.float32)
    invm = torch.from_numpy(inv_m).cuda()
    dt = bench.DT_FS * 1e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731

    def steps(first, k):
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm),
                                                     ctypes.c_float(dt), first, k, sp),
                       "md_steps")

    # equilibrate at 300 K (velocity rescaling every 100 steps), as the bench
    mass = torch.from_numpy(s.mass.astype(np.float64)).cuda()
    EQ = args.equilibrate
    for c0 in range(0, EQ, 100):
        steps(c0, min(100, EQ - c0))
        with torch.cuda.stream(st):
            v = vel.view(n, 3).double()
            t_now = float((mass[:, None] * v * v).sum()) / (3.0 * n * systems.KB)
            vel.mul_(float(np.sqrt(300.0 / t_now)))
    st.synchronize()
    start = (crd.cpu().numpy().reshape(n, 3).copy(), vel.cpu().numpy().reshape(n, 3).copy())
    tuned = np.zeros(4, np.int32)
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_autotune(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                           10, tuned.ctypes.data, sp), "autotune")

    K, W = args.steps, max(3, args.warmup)
    clocks = bench.ClockSampler(torch.cuda.current_device())
    clocks.start()
    # the engine
    steps(EQ, W)
    st.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    steps(EQ + W, K)
    e1.record(st)
    st.synchronize()
    ms_ours = e0.elapsed_time(e1)
    # the reference's GPU modules from the same equilibrated state
    ref = ReferenceGPU()
    with bench.stdout_to_stderr():
        ref.init(s, bench.CUTOFF, bench.SKIN)
        ref.set_bonded(s.bonds, systems.BOND_K, systems.BOND_R0, s.angles,
                       systems.ANGLE_K, systems.ANGLE_T0)
    ref.set_state(start[0], start[1], inv_m)
    ref.md_steps(W, dt)
    ms_ref = ref.md_steps(K, dt)
    clk = clocks.stop()
    count, overflow = ref.pair_count()

    # energy drift of both from the same start
    crd.copy_(torch.from_numpy(start[0].reshape(-1)))
    vel.copy_(torch.from_numpy(start[1].reshape(-1)))
    D = args.drift_steps
    drift_ours = bench.nve_drift(lib, h, s, crd, vel, invm, EQ, D, 21, dt,
                                 lib.snb_engine_md_steps_graph, st, sp)
    drift_ref = reference_drift(ref, s, inv_m, start, D, 21, dt)
    lib.snb_engine_destroy(h)

    ours = {"ms_per_step": ms_ours / K, "ns_per_day": bench.ns_per_day(K / (ms_ours / 1e3)),
            "nve_drift": drift_ours["kcal_per_mol_per_ns_per_atom"]}
    refd = {"ms_per_step": ms_ref / K, "ns_per_day": bench.ns_per_day(K / (ms_ref / 1e3)),
            "nve_drift": drift_ref["kcal_per_mol_per_ns_per_atom"],
            "list_entries": count, "list_overflow": overflow}
    print(json.dumps({
        "workload": f"{n}-atom water + NaCl box, cutoff {bench.CUTOFF} A, skin {bench.SKIN} A, "
                    f"PME {ref.grid[0]}^3, NVE dt {bench.DT_FS} fs",
        "steps": K, "warmup": W, "equilibrate": EQ,
        "engine": ours, "reference_gpu": refd,
        "speedup": ours["ns_per_day"] / refd["ns_per_day"],
        "tuned": tuned.tolist(), "clocks": clk}))


if __name__ == "__main__":
    main()
