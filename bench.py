"""Benchmark: ns/day of NVE molecular dynamics on the 100k-atom LJ + PME water
box (33,333 TIP3P-style waters, 90 Na+ / 90 Cl-, L = 99.90 A, PME grid 100^3,
cutoff 10 A, skin 2 A, dt = 0.5 fs) through this package's fused engine.

A step is one full MD step: conditional neighbor update (forced every 100
steps as in the reference loop), LJ + direct Coulomb pair kernel, excluded
correction, PME reciprocal, water bonds/angles and the leap-frog update, all
in one CUDA graph with 64-bit fixed-point force accumulation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
independent replica box (replicas only: one box does not shard across GPUs);
value = total simulated ns of all replicas per day, timed as the max over
ranks.  `--impl reference` times the reference's own CPU implementation of
the same path (its neighbor_list / Lennard_Jones_force / PM_force code built
from source into oracle/_ref) on the host cores.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ns/day at 100k-atom LJ+PME water; batched steps/s; force rel-err vs FP64"
DT_FS = 0.5
# the launch shapes snb_engine_autotune reports, in its h_choice order
TUNED_KEYS = ["pair_unroll", "pair_blocks_per_sm", "search_blocks_per_sm", "gather_threads",
              "pair_warps", "spread_tile_edge", "spread_warps", "pair_hit_stash", "own_fft"]
CUTOFF = 10.0
SKIN = 2.0


def ns_per_day(steps_per_s: float) -> float:
    return steps_per_s * DT_FS * 1e-6 * 86400.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--waters", type=int, default=33333,
                   help="box size (default: the 100k-atom configuration)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-steps", type=int, default=30)
    p.add_argument("--equilibrate", type=int, default=2000,
                   help="untimed NVE steps from the lattice start before warm-up")
    p.add_argument("--no-graph", action="store_true",
                   help="launch the step kernels on the stream instead of replaying "
                        "the captured step graph (for kernel profilers)")
    p.add_argument("--no-tune", action="store_true",
                   help="keep the default launch shapes (skip the autotuner)")
    p.add_argument("--batch-systems", type=int, default=256,
                   help="boxes in the batched measurement (0: skip)")
    p.add_argument("--batch-steps", type=int, default=200)
    p.add_argument("--drift-steps", type=int, default=10000,
                   help="NVE steps after the timed region over which the total-energy "
                        "drift is fitted (0: skip)")
    p.add_argument("--no-small-box", action="store_true",
                   help="skip the 9,000-atom box")
    p.add_argument("--soft-core-waters", type=int, default=333333,
                   help="waters of the soft-core box (about 1M atoms; 0: skip)")
    p.add_argument("--soft-core-equilibrate", type=int, default=1000)
    p.add_argument("--soft-core-grid150", type=int, default=1,
                   help="also run the soft-core box's lambda 0.5 window with PME 150^3 (0: skip)")
    p.add_argument("--no-accuracy", action="store_true",
                   help="skip the FP64 accuracy checks (outside the timed regions)")
    p.add_argument("--plain-gpu-steps", type=int, default=1000,
                   help="steps of the reference's own GPU path and of this engine from "
                        "the same state (0: skip)")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_box(n_waters: int, seed: int):
    from sponge_b200 import systems
    return systems.water_box(n_waters, seed=seed, ion_pairs=None)


# --------------------------------------------------------------------------
class ClockSampler:
    """SM clock, power and throttle reasons sampled every ~1 ms through NVML
    while the timed region runs (a background thread; the main thread waits
    in CUDA calls that release the GIL), so that even a window of a few
    milliseconds gets samples.  Falls back to `nvidia-smi -lms 20` into a
    temporary file when NVML is unavailable."""

    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown"}
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_device: int):
        self.dev = cuda_device
        self.samples = []
        self.thread = None
        self.proc = None
        self.mode = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())

    def start(self):
        import threading
        self.samples = []
        try:
            nv, h = self._handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
        except Exception:  # noqa: BLE001
            return self._start_smi()
        self.mode = "nvml"
        self.stop_flag = threading.Event()

        def loop():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append((time.perf_counter(),
                                         float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(get_reasons(h)),
                                         nv.nvmlDeviceGetPowerUsage(h) / 1000.0))
                except Exception:  # noqa: BLE001
                    pass
                time.sleep(0.001)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def _start_smi(self):
        import tempfile
        self.mode = "nvidia-smi"
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self, window=None):
        """Summary of the samples (those inside window = (t0, t1) of
        time.perf_counter when given and any fall inside it)."""
        if self.mode == "nvml" and self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=2)
            rows = self.samples
            inside = [r for r in rows if window and window[0] <= r[0] <= window[1]]
            use = inside or rows
            if not use:
                return None
            reasons = sorted({nm for r in use for bit, nm in self.REASONS.items()
                              if r[2] & bit})
            return {"sm_mhz": statistics.median(r[1] for r in use),
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "power_w_max": max(r[3] for r in use), "samples": len(use),
                    "samples_in_timed_window": len(inside), "source": "nvml 1 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"samples": 0, "source": "nvidia-smi 20 ms",
                    "note": "no sample fell in the timed window"}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi 20 ms"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per pair-kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "pair_kernel_traffic.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d
    return None


def bonded_energy(s, crd):
    """Water bonds and angles at crd (host, FP64), the same harmonic forms
    the engine integrates: k (r - r0)^2 and k (theta - theta0)^2."""
    from sponge_b200 import systems
    crd = crd.astype(np.float64)
    b = s.bonds
    d = crd[b[:, 0]] - crd[b[:, 1]]
    d -= np.round(d / s.box) * s.box
    r = np.linalg.norm(d, axis=1)
    e = systems.BOND_K * ((r - systems.BOND_R0) ** 2).sum()
    a = s.angles
    u = crd[a[:, 0]] - crd[a[:, 1]]
    w = crd[a[:, 2]] - crd[a[:, 1]]
    u -= np.round(u / s.box) * s.box
    w -= np.round(w / s.box) * s.box
    c = (u * w).sum(1) / np.linalg.norm(u, axis=1) / np.linalg.norm(w, axis=1)
    return e + systems.ANGLE_K * ((np.arccos(np.clip(c, -1, 1)) - systems.ANGLE_T0) ** 2).sum()


def nve_drift(lib, h, s, crd, vel, invm, first, total, samples, dt, run_steps, st, sp):
    """Total energy every total/(samples-1) steps: the engine's nonbonded
    potential (FP64 sums), the bonded terms on the host, and the kinetic
    energy from the average of the leap-frog half-step velocities around the
    sample.  Returns the fitted drift in kcal/mol/ns/atom."""
    import torch
    from sponge_b200 import capi, systems
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    n = s.n
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    every = max(2, total // max(1, samples - 1))
    step, ts, es, kes = first, [], [], []
    m = s.mass.astype(np.float64)[:, None]
    for _ in range(samples):
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_force(h, P(crd), P(frc), step, 1, 0, P(tot), sp),
                       "engine_force")
        st.synchronize()
        c0 = crd.cpu().numpy().reshape(n, 3)
        v0 = vel.cpu().numpy().reshape(n, 3).astype(np.float64)
        pot = float(tot[7].item()) + bonded_energy(s, c0)
        with torch.cuda.stream(st):
            capi.check(run_steps(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                 step, 1, sp), "md_steps")
        st.synchronize()
        v1 = vel.cpu().numpy().reshape(n, 3).astype(np.float64)
        ke = 0.5 * (m * (0.5 * (v0 + v1)) ** 2).sum()
        ts.append(step)
        es.append(pot + ke)
        kes.append(ke)
        step += 1
        with torch.cuda.stream(st):
            capi.check(run_steps(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                 step, every - 1, sp), "md_steps")
        step += every - 1
    st.synchronize()
    ts = np.asarray(ts, np.float64)
    es = np.asarray(es, np.float64)
    slope = np.polyfit(ts, es, 1)[0]  # kcal/mol per step
    per_ns = slope / (DT_FS * 1e-6)
    return {"steps": int(ts[-1] - ts[0]), "samples": len(ts),
            "kcal_per_mol_per_ns_per_atom": per_ns / n,
            "e_total_first": es[0], "e_total_last": es[-1],
            "e_total_std": float(es.std()),
            "temperature_K": float(2.0 * np.mean(kes) / (3.0 * n * systems.KB))}



# --------------------------------------------------------------------------
class stdout_to_stderr:
    """Sends file descriptor 1 to stderr for the duration: the reference's
    modules print their initialisation reports with C stdio, which Python's
    own redirection does not catch, and stdout must carry only the result
    line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        try:
            import ctypes.util
            libc = ctypes.CDLL(ctypes.util.find_library("c"))
            libc.fflush(None)
        except OSError:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def cpu_reference_run(s, evals: int, warmup: int, rebuild_rate: float = 0.01):
    """Time the reference's own CPU path (oracle/_ref) on box `s`: per MD step
    the conditional neighbor update, excluded correction, LJ + direct Coulomb
    and PME reciprocal, plus `rebuild_rate` full rebuilds (the rate our own
    run saw; the reference loop forces at least one every 100 steps)."""
    from oracle.oracle import REF_SO, ReferenceCPU
    if not os.path.exists(REF_SO):
        return None, "oracle/_ref/libsponge_ref.so not built"
    ref = ReferenceCPU(exact=False)
    with stdout_to_stderr():
        ref.init(s, CUTOFF, SKIN)
        cores = ref.max_threads()
        t0 = time.perf_counter()
        ref.nl_update_only(forced=True)
        t_rebuild = time.perf_counter() - t0
        for k in range(warmup):
            ref.force_step(k)
        t0 = time.perf_counter()
        for k in range(evals):
            ref.force_step(warmup + k)
        t_step = (time.perf_counter() - t0) / evals + t_rebuild * rebuild_rate
    return dict(value=ns_per_day(1.0 / t_step), unit="ns/day", cores=cores,
                kind="reference",
                sample=(f"{evals} force evaluations (conditional neighbor update, "
                        f"excluded correction, LJ + direct Coulomb, PME reciprocal) of "
                        f"the {s.n}-atom box after {warmup} warm-up, plus "
                        f"{rebuild_rate:.3f} neighbor rebuilds per step; "
                        f"{t_step * 1e3:.1f} ms/step on {cores} threads"),
                ms_per_step=t_step * 1e3), None


WORK_OURS = ("full NVE MD step: conditional neighbor update (forced every 100 steps), "
             "LJ + direct Coulomb, excluded correction, PME reciprocal, water bonds and "
             "angles, leap-frog")
WORK_REFERENCE = ("force evaluation: conditional neighbor update, excluded correction, "
                  "LJ + direct Coulomb, PME reciprocal (no bonded terms, no integration), "
                  "plus the observed neighbor rebuild rate")


def bench_config(n: int) -> dict:
    """The workload description both arms print, identical in each."""
    return {"workload": f"{n}-atom water + NaCl NVE MD, cutoff 10 A, skin 2 A, "
                        f"PME 100^3 order 4, dt 0.5 fs",
            "atoms": n, "cutoff_A": CUTOFF, "skin_A": SKIN, "pme_grid": [100, 100, 100],
            "dt_fs": DT_FS,
            "l2": "working set > L2 (neighbor list alone ~140 MB), no flush needed"}


# Neighbor rebuilds per step of this box in NVE at 300 K (the engine's
# 10,000-step drift runs see one about every 25 steps: the 1 A trigger of
# half the skin); the reference arm, which evaluates forces without moving
# atoms, amortises its rebuild at this rate.
NVE_REBUILD_RATE = 0.04


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    s = make_box(args.waters, seed=0)
    K, W = args.steps, max(args.warmup, 3)
    res, why = cpu_reference_run(s, K, W, rebuild_rate=NVE_REBUILD_RATE)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    line = {
        "metric": METRIC, "value": res["value"], "unit": "ns/day", "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": res["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded water/NaCl box)",
        "config": bench_config(s.n),
        "work": WORK_REFERENCE,
        "parallelism": "host threads (OpenMP) on rank 0",
        "impl": "reference",
        "cpu_baseline": {"value": res["value"], "unit": "ns/day", "cores": res["cores"],
                         "kind": "reference", "sample": res["sample"]},
        "e2e": {"value": res["value"], "unit": "ns/day", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
def _batch_member(seed):
    from sponge_b200 import systems
    return systems.config_batch_member(seed)


def make_batch(seeds):
    """The batch boxes (water count U[200, 2000] from each seed), generated in
    a pool of spawned worker processes."""
    import concurrent.futures as cf
    import multiprocessing as mp
    workers = max(1, min(16, os.cpu_count() or 1, len(seeds)))
    with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_batch_member, seeds))


def run_batch(args, lib, world, rank, dist):
    """Batched steps/s: this rank's share of the boxes (cost-balanced by
    sponge_b200.sharding) advanced by one engine, one launch per phase per
    step, against the same
    boxes each advanced by its own single-box engine (one captured step graph
    launched per box per step).  Both with water bonds/angles, NVE, 0.5 fs,
    cutoff 8 A, skin 2 A, PME grid per box from 1 A spacing, fixed point."""
    import torch
    from sponge_b200 import capi, sharding, systems
    sizes = [systems.batch_member_size(s) for s in range(args.batch_systems)]
    seeds = sharding.shard([sharding.box_cost(n, k) for n, k in sizes], world)[rank]
    boxes = make_batch(seeds)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    dt = DT_FS * 1e-3 * systems.TIME_CONVERSION
    cut = 8.0
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)

    def bonded(h, bonds, angles):
        nb, na = len(bonds), len(angles)
        arr = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
        ba, bb = arr(bonds[:, 0]), arr(bonds[:, 1])
        aa, ab, ac = arr(angles[:, 0]), arr(angles[:, 1]), arr(angles[:, 2])
        bk = np.full(nb, systems.BOND_K, np.float32)
        br = np.full(nb, systems.BOND_R0, np.float32)
        ak = np.full(na, systems.ANGLE_K, np.float32)
        at = np.full(na, systems.ANGLE_T0, np.float32)
        capi.check(lib.snb_engine_set_bonded(h, nb, ba.ctypes.data, bb.ctypes.data,
                                             bk.ctypes.data, br.ctypes.data, na,
                                             aa.ctypes.data, ab.ctypes.data, ac.ctypes.data,
                                             ak.ctypes.data, at.ctypes.data), "set_bonded")

    # ---- the batch in one engine
    offs = np.cumsum([0] + [b.n for b in boxes])
    cat = lambda name, dt_: np.ascontiguousarray(  # noqa: E731
        np.concatenate([getattr(b, name) for b in boxes]), dt_)
    es = np.concatenate([b.excl_start + sum(len(x.excl_list) for x in boxes[:k])
                         for k, b in enumerate(boxes)]).astype(np.int32)
    el = np.concatenate([b.excl_list + offs[k] for k, b in enumerate(boxes)]).astype(np.int32)
    en = cat("excl_numbers", np.int32)
    typ, q = cat("lj_type", np.int32), cat("charge", np.float32)
    A = np.ascontiguousarray(boxes[0].lj_A, np.float32)
    B = np.ascontiguousarray(boxes[0].lj_B, np.float32)
    counts = np.array([b.n for b in boxes], np.int32)
    lens = np.array([[b.box] * 3 for b in boxes], np.float32).reshape(-1)
    opts = capi.options(cutoff=cut, skin=SKIN)
    h = ctypes.c_void_p()
    capi.check(lib.snb_batch_create(ctypes.byref(opts), len(boxes), counts.ctypes.data,
                                    lens.ctypes.data, boxes[0].n_types, typ.ctypes.data,
                                    A.ctypes.data, B.ctypes.data, q.ctypes.data,
                                    es.ctypes.data, en.ctypes.data, el.ctypes.data, len(el),
                                    ctypes.byref(h)), "batch_create")
    bonded(h, np.concatenate([b.bonds + offs[k] for k, b in enumerate(boxes)]),
           np.concatenate([b.angles + offs[k] for k, b in enumerate(boxes)]))
    crd = torch.from_numpy(cat("crd", np.float32).reshape(-1).copy()).cuda()
    vel = torch.from_numpy(cat("vel", np.float32).reshape(-1).copy()).cuda()
    invm = torch.from_numpy((1.0 / cat("mass", np.float32)).astype(np.float32)).cuda()
    KB, WB = max(1, args.batch_steps), 3
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                                 0, 100, sp), "batch warm-up")
    tuned = np.zeros(9, np.int32)
    if not args.no_tune:
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_autotune(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                               5, tuned.ctypes.data, sp), "batch autotune")
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                                 100, WB, sp), "batch warm-up")
    st.synchronize()
    rb0, rb1 = ctypes.c_longlong(0), ctypes.c_longlong(0)
    capi.check(lib.snb_engine_stats(h, ctypes.byref(rb0), None, sp), "stats")
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                                 100 + WB, KB, sp), "batch steps")
    e1.record(st)
    st.synchronize()
    ms_b = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    capi.check(lib.snb_engine_stats(h, ctypes.byref(rb1), None, sp), "stats")
    kn, libk, bodyk = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    capi.check(lib.snb_engine_graph_info(h, ctypes.byref(kn), ctypes.byref(libk),
                                         ctypes.byref(bodyk), sp), "graph_info")
    # accuracy of every box at the frame the timed steps left, against the
    # FP64 oracle run of that box alone (outside the timed region)
    batch_acc = None
    if not args.no_accuracy:
        frc = torch.zeros_like(crd)
        tot = torch.zeros(16, dtype=torch.float64, device="cuda")
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_force(h, P(crd), P(frc), 100 + WB + KB, 1, 1, P(tot),
                                            sp), "batch force")
        st.synchronize()
        batch_acc = batch_accuracy(boxes, crd.cpu().numpy().reshape(-1, 3),
                                   frc.cpu().numpy().reshape(-1, 3), tot.cpu().numpy(), cut)
    lib.snb_engine_destroy(h)

    # ---- one engine per box, one step graph launched per box per step
    singles = []
    for b in boxes:
        hs = ctypes.c_void_p()
        bes, ben = np.ascontiguousarray(b.excl_start, np.int32), np.ascontiguousarray(
            b.excl_numbers, np.int32)
        bel = np.ascontiguousarray(b.excl_list if len(b.excl_list) else np.zeros(1), np.int32)
        bt, bq = np.ascontiguousarray(b.lj_type, np.int32), np.ascontiguousarray(b.charge,
                                                                                 np.float32)
        capi.check(lib.snb_engine_create(ctypes.byref(opts), b.n,
                                         capi.boundary(b.cell(), b.rcell()), b.n_types,
                                         bt.ctypes.data, A.ctypes.data, B.ctypes.data,
                                         bq.ctypes.data, bes.ctypes.data, ben.ctypes.data,
                                         bel.ctypes.data, len(b.excl_list), ctypes.byref(hs)),
                   "engine_create")
        bonded(hs, b.bonds, b.angles)
        c = torch.from_numpy(b.crd.reshape(-1).copy()).cuda()
        v = torch.from_numpy(b.vel.reshape(-1).copy()).cuda()
        m = torch.from_numpy((1.0 / b.mass).astype(np.float32)).cuda()
        singles.append((hs, c, v, m))
    KS = KB  # the same step count as the batch, so both windows see the same phases
    with torch.cuda.stream(st):
        for hs, c, v, m in singles:
            capi.check(lib.snb_engine_md_steps_graph(hs, P(c), P(v), P(m), ctypes.c_float(dt),
                                                     0, 100 + WB, sp), "single warm-up")
    st.synchronize()
    if dist:
        dist.barrier()
    e0.record(st)
    with torch.cuda.stream(st):  # each box's KS steps back to back, box after box
        for hs, c, v, m in singles:
            capi.check(lib.snb_engine_md_steps_graph(hs, P(c), P(v), P(m), ctypes.c_float(dt),
                                                     100 + WB, KS, sp), "single steps")
    e1.record(st)
    st.synchronize()
    ms_s = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    for hs, _, _, _ in singles:
        lib.snb_engine_destroy(hs)
    if dist:
        dist.all_reduce(ms_b, op=dist.ReduceOp.MAX)
        dist.all_reduce(ms_s, op=dist.ReduceOp.MAX)
    sps_b = KB / (float(ms_b.item()) / 1e3)
    sps_s = KS / (float(ms_s.item()) / 1e3)
    K = [systems.fft_size(b.box) for b in boxes]
    return {"systems": args.batch_systems, "systems_per_rank": len(boxes),
            "atoms_per_rank": int(offs[-1]), "steps": KB,
            "steps_per_s": sps_b, "ms_per_step": float(ms_b.item()) / KB,
            # steps of the timed window on which at least one box rebuilt its list
            "steps_with_rebuild": int(rb1.value - rb0.value),
            "one_system_per_launch_steps_per_s": sps_s,
            "one_system_per_launch_steps": KS,
            "speedup_vs_one_system_per_launch": sps_b / sps_s,
            "accuracy": batch_acc,
            "kernels_per_step": kn.value - libk.value, "library_kernels_per_step": libk.value,
            "pme_grids": f"{min(K)}^3..{max(K)}^3",
            "tuned": (None if args.no_tune else dict(zip(TUNED_KEYS, [int(x) for x in tuned]))),
            "workload": "256 water+NaCl boxes (seeds 0-255, 200-2000 waters each, 1 g/cm^3), "
                        "cutoff 8 A, skin 2 A, PME order 4 at 1 A spacing, NVE 0.5 fs, "
                        "fixed-point accumulation"}


def batch_accuracy(boxes, crd, frc, totals, cutoff):
    """Per-box force rel-RMS of a batch force evaluation (caller-order crd,
    frc of all boxes) against each box's FP64 oracle run, and the summed
    energy components against the sum of the boxes' FP64 components."""
    import copy

    from oracle import accuracy
    from oracle.oracle import Oracle
    o = Oracle()
    base, errs, en_sum = 0, [], {}
    for b in boxes:
        f = copy.copy(b)
        f.crd = np.ascontiguousarray(crd[base:base + b.n])
        want, en, _ = accuracy.reference_totals(o, f, cutoff, SKIN)
        errs.append(accuracy.force_rel_rms(frc[base:base + b.n], want))
        for k, v in en.items():
            en_sum[k] = en_sum.get(k, 0.0) + v
        base += b.n
    rel = {k: abs(totals[i] - en_sum[k]) / abs(en_sum[k])
           for k, i in accuracy.TOTAL_SLOTS.items()}
    return {"boxes": len(boxes), "force_rel_rms_max": max(errs),
            "force_rel_rms_median": float(np.median(errs)),
            "energy_rel": rel, "energy_rel_max": max(rel.values()),
            "reference": "FP64 oracle per box (direct over its FP32 pair set, PME on the "
                         "box's grid, excluded correction, tail term)"}


def headline_accuracy(lib, h, s, crd, step, st, sp):
    """Forces, energies, virial and pressure of one engine force evaluation at
    the current frame against the FP64 oracle run of the same frame."""
    import copy

    import torch
    from oracle import accuracy
    from oracle.oracle import Oracle
    from sponge_b200 import capi
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    frc = torch.zeros_like(crd)
    tot = torch.zeros(16, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_force(h, P(crd), P(frc), step, 1, 1, P(tot), sp),
                   "engine_force")
    st.synchronize()
    f = copy.copy(s)
    f.crd = crd.cpu().numpy().reshape(-1, 3).copy()
    ref = accuracy.reference_totals(Oracle(), f, CUTOFF, SKIN)
    out = accuracy.compare(frc.cpu().numpy().reshape(-1, 3), tot.cpu().numpy(), ref,
                           float(np.float32(s.box)) ** 3)
    out["reference"] = ("FP64 oracle of the same frame: direct over its FP32 pair set, "
                        "PME 100^3, excluded correction, tail term")
    return out


def plain_gpu_run(s, crd0, vel0, steps, warmup):
    """The reference's own GPU path (its neighbor_list, Lennard_Jones_force,
    PM_force, bond and angle modules compiled as CUDA for sm_100a: FP32 with
    float atomics, main.cpp's order) from the given state: device time of
    `steps` NVE steps after `warmup`."""
    from oracle.oracle import REF_GPU_SO, ReferenceGPU
    from sponge_b200 import systems
    if not os.path.exists(REF_GPU_SO):
        return {"unavailable": "oracle/_ref/libsponge_ref_gpu.so not built"}
    dt = DT_FS * 1e-3 * systems.TIME_CONVERSION
    ref = ReferenceGPU()
    with stdout_to_stderr():
        ref.init(s, CUTOFF, SKIN)
        ref.set_bonded(s.bonds, systems.BOND_K, systems.BOND_R0, s.angles,
                       systems.ANGLE_K, systems.ANGLE_T0)
    ref.set_state(crd0, vel0, (1.0 / s.mass).astype(np.float32))
    ref.md_steps(warmup, dt)
    ms = ref.md_steps(steps, dt)
    return {"ms_per_step": ms / steps, "ns_per_day": ns_per_day(steps / (ms / 1e3)),
            "steps": steps, "warmup": warmup,
            "what": "the reference's own GPU modules (neighbor_list, Lennard_Jones_force, "
                    "PM_force, bond, angle) compiled for sm_100a with its CUDA flags, FP32 "
                    "float atomics, driven in main.cpp's order; NVE leap-frog"}


def soft_accuracy(lib, h, s, sc, crd, lam, step, st, sp, grid=None):
    """Force rel-RMS of the soft-core engine at the current frame against the
    FP64 oracle (soft-core direct terms, PME, excluded correction) over all
    atoms; the windows' charges are state B's (solute charges off)."""
    import copy

    import torch
    from oracle import accuracy
    from oracle.oracle import Oracle
    from sponge_b200 import capi
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    frc = torch.zeros_like(crd)
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_force(h, P(crd), P(frc), step, 0, 0, None, sp),
                   "soft force")
    st.synchronize()
    f = copy.copy(s)
    f.crd = crd.cpu().numpy().reshape(-1, 3).copy()
    f.charge = (s.charge.astype(np.float64) + sc.charge_B_A).astype(np.float32)
    scb = copy.copy(sc)
    scb.charge_B_A = np.zeros_like(sc.charge_B_A)
    want = accuracy.soft_reference_forces(Oracle(), f, scb, CUTOFF, lam, 0.5, 1.0, 3.0, 0.0,
                                          SKIN, grid=None if grid is None else (grid,) * 3)
    return {"lambda": lam, "force_rel_rms": accuracy.force_rel_rms(
        frc.cpu().numpy().reshape(-1, 3), want),
        "reference": "FP64 oracle over all atoms at the frame after the window"}


def make_engine(lib, s, cutoff, **keys):
    """Single-box engine over System `s` with its water bonds and angles
    (`keys`: more input keys, e.g. PM_fftx)."""
    from sponge_b200 import capi, systems
    opts = capi.options(cutoff=cutoff, skin=SKIN, **keys)
    h = ctypes.c_void_p()
    arr = np.ascontiguousarray
    t, A, B = arr(s.lj_type, np.int32), arr(s.lj_A, np.float32), arr(s.lj_B, np.float32)
    q = arr(s.charge, np.float32)
    es, en = arr(s.excl_start, np.int32), arr(s.excl_numbers, np.int32)
    el = arr(s.excl_list if len(s.excl_list) else np.zeros(1), np.int32)
    capi.check(lib.snb_engine_create(ctypes.byref(opts), s.n, capi.boundary(s.cell(), s.rcell()),
                                     s.n_types, t.ctypes.data, A.ctypes.data, B.ctypes.data,
                                     q.ctypes.data, es.ctypes.data, en.ctypes.data,
                                     el.ctypes.data, len(s.excl_list), ctypes.byref(h)),
               "engine_create")
    nb, na = len(s.bonds), len(s.angles)
    ba, bb = arr(s.bonds[:, 0], np.int32), arr(s.bonds[:, 1], np.int32)
    aa, ab, ac = (arr(s.angles[:, k], np.int32) for k in range(3))
    bk, br = np.full(nb, systems.BOND_K, np.float32), np.full(nb, systems.BOND_R0, np.float32)
    ak, at = np.full(na, systems.ANGLE_K, np.float32), np.full(na, systems.ANGLE_T0, np.float32)
    capi.check(lib.snb_engine_set_bonded(h, nb, ba.ctypes.data, bb.ctypes.data, bk.ctypes.data,
                                         br.ctypes.data, na, aa.ctypes.data, ab.ctypes.data,
                                         ac.ctypes.data, ak.ctypes.data, at.ctypes.data),
               "set_bonded")
    return h


def _equilibrate(lib, h, s, crd, vel, invm, dt, steps, st, sp):
    """Untimed NVE steps with the velocities rescaled to 300 K every 100."""
    import torch
    from sponge_b200 import capi, systems
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    mass = torch.from_numpy(s.mass.astype(np.float64)).cuda()
    for c0 in range(0, steps, 100):
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm),
                                                     ctypes.c_float(dt), c0,
                                                     min(100, steps - c0), sp), "md_steps")
            v = vel.view(s.n, 3).double()
            t_now = float((mass[:, None] * v * v).sum()) / (3.0 * s.n * systems.KB)
            vel.mul_(float(np.sqrt(300.0 / t_now)))
    st.synchronize()


def _timed_steps(lib, h, crd, vel, invm, dt, first, steps, st, sp):
    """Device time (ms) of `steps` graph-replayed steps."""
    import torch
    from sponge_b200 import capi
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.synchronize()
    e0.record(st)
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_md_steps_graph(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                                 first, steps, sp), "md_steps")
    e1.record(st)
    st.synchronize()
    return e0.elapsed_time(e1)


def run_small_box(lib):
    """The 9,000-atom box (3,000 waters, cutoff 8 A, PME 48^3): 200 NVE steps
    from the Maxwell-Boltzmann start after 20 untimed ones, and the total-energy
    drift fitted over the next 200 steps."""
    import torch
    from sponge_b200 import systems
    s = systems.config_small(seed=0)
    h = make_engine(lib, s, 8.0)
    crd = torch.from_numpy(s.crd.reshape(-1).copy()).cuda()
    vel = torch.from_numpy(s.vel.reshape(-1).copy()).cuda()
    invm = torch.from_numpy((1.0 / s.mass).astype(np.float32)).cuda()
    dt = DT_FS * 1e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    ms = _timed_steps(lib, h, crd, vel, invm, dt, 0, 200, st, sp)
    # the drift after 1,000 steps at 300 K (the lattice start releases
    # potential energy into the first few hundred steps)
    _equilibrate(lib, h, s, crd, vel, invm, dt, 1000, st, sp)
    drift = nve_drift(lib, h, s, crd, vel, invm, 1200, 200, 21, dt,
                      lib.snb_engine_md_steps_graph, st, sp)
    lib.snb_engine_destroy(h)
    return {"workload": f"{s.n}-atom water box, cutoff 8 A, skin 2 A, "
                        f"PME {systems.fft_size(s.box)}^3, NVE 0.5 fs",
            "steps": 200, "ms_per_step": ms / 200, "ns_per_day": ns_per_day(200 / (ms / 1e3)),
            "timed_from": "Maxwell-Boltzmann 300 K lattice start (first 200 steps)",
            "nve_drift": drift}


def run_soft_core_box(args, lib):
    """The large soft-core workload: a water + 0.15 M NaCl box with a 64-site
    alchemical solute (soft-core LJ, alpha 0.5, p 1, sigma 3 A), cutoff 10 A,
    PME by the reference's grid rule.  The windows are the LJ stage of a
    decoupling: the solute's charges are off in every window (state B's
    charges; with them on, water H atoms, which carry no LJ, fall onto the
    charged sites once their LJ is softened, and the box blows up), and lambda
    takes the solute's LJ from state A to state B through the soft core.
    Each window runs its own engine with the soft-core tables at its lambda.
    Untimed equilibration in the lambda 0 window with 300 K velocity
    rescaling; each window then runs 10 untimed and 500 timed graph-replayed
    NVE steps from the state the previous window left."""
    import copy

    import torch
    from sponge_b200 import capi, systems
    s, sc = systems.soft_core_box(args.soft_core_waters, n_solute=64, seed=0)
    crd = torch.from_numpy(s.crd.reshape(-1).copy()).cuda()
    vel = torch.from_numpy(s.vel.reshape(-1).copy()).cuda()
    invm = torch.from_numpy((1.0 / s.mass).astype(np.float32)).cuda()
    dt = DT_FS * 1e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    arr = np.ascontiguousarray
    tA, tB = arr(sc.type_A, np.int32), arr(sc.type_B, np.int32)
    AA, AB = arr(sc.AA, np.float32), arr(sc.AB, np.float32)
    BA, BB = arr(sc.BA, np.float32), arr(sc.BB, np.float32)
    mask = arr(sc.mask, np.int32)

    def window(lam, grid=None):
        w = copy.copy(s)
        w.charge = (s.charge.astype(np.float64) + sc.charge_B_A).astype(np.float32)
        keys = {} if grid is None else {"PM_fftx": grid, "PM_ffty": grid, "PM_fftz": grid}
        h = make_engine(lib, w, CUTOFF, **keys)
        o = capi.options(cutoff=CUTOFF, skin=SKIN, lambda_lj=lam, soft_core_alpha=0.5,
                         soft_core_powfer=1.0, soft_core_sigma=3.0, soft_core_sigma_min=0.0)
        hs = ctypes.c_void_p()
        capi.check(lib.snb_lj_soft_create(ctypes.byref(o), s.n, sc.n_types_A, sc.n_types_B,
                                          tA.ctypes.data, tB.ctypes.data, AA.ctypes.data,
                                          AB.ctypes.data, BA.ctypes.data, BB.ctypes.data,
                                          mask.ctypes.data, CUTOFF, ctypes.byref(hs)),
                   "lj_soft_create")
        capi.check(lib.snb_engine_set_soft_core(h, hs), "set_soft_core")
        return h, hs

    def close(h, hs):
        lib.snb_engine_destroy(h)
        lib.snb_lj_soft_destroy(hs)

    acc = None
    EQ = max(0, args.soft_core_equilibrate)
    h, hs = window(0.0)
    _equilibrate(lib, h, s, crd, vel, invm, dt, EQ, st, sp)
    # launch shapes tuned once, in the first window, and set in every window
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    tuned = np.zeros(9, np.int32)
    if not args.no_tune:
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_autotune(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                               5, tuned.ctypes.data, sp), "soft-core autotune")
    close(h, hs)
    runs = []
    step = EQ
    for lam in (0.0, 0.25, 0.5, 0.75, 1.0):
        h, hs = window(lam)
        if not args.no_tune:
            capi.check(lib.snb_engine_set_launch_shapes(h, tuned.ctypes.data), "shapes")
        _timed_steps(lib, h, crd, vel, invm, dt, step, 10, st, sp)
        r0, r1 = ctypes.c_longlong(0), ctypes.c_longlong(0)
        capi.check(lib.snb_engine_stats(h, ctypes.byref(r0), None, sp), "stats")
        ms = _timed_steps(lib, h, crd, vel, invm, dt, step + 10, 500, st, sp)
        capi.check(lib.snb_engine_stats(h, ctypes.byref(r1), None, sp), "stats")
        if lam == 0.5 and not args.no_accuracy:
            acc = soft_accuracy(lib, h, s, sc, crd, lam, step + 510, st, sp)
        close(h, hs)
        step += 510
        v = vel.view(-1, 3).double()
        ke = 0.5 * (torch.from_numpy(s.mass).cuda().double()[:, None] * v * v).sum(1)
        runs.append({"lambda": lam, "ms_per_step": ms / 500,
                     "ns_per_day": ns_per_day(500 / (ms / 1e3)),
                     "nl_rebuilds": int(r1.value - r0.value),
                     "temperature_K": float(2.0 * ke.sum() / (3.0 * s.n * systems.KB)),
                     "hottest_atom_kcal_per_mol": float(ke.max())})
    # the stated grid variant: PME 150^3 set explicitly (the reference's
    # PM_fftx/y/z keys) in the lambda 0.5 window, from the state the windows
    # left
    g150 = None
    if args.soft_core_grid150:
        h, hs = window(0.5, grid=150)
        if not args.no_tune:
            capi.check(lib.snb_engine_set_launch_shapes(h, tuned.ctypes.data), "shapes")
        _timed_steps(lib, h, crd, vel, invm, dt, step, 10, st, sp)
        ms = _timed_steps(lib, h, crd, vel, invm, dt, step + 10, 500, st, sp)
        g150 = {"lambda": 0.5, "pme_grid": [150, 150, 150], "steps": 500,
                "ms_per_step": ms / 500, "ns_per_day": ns_per_day(500 / (ms / 1e3))}
        if not args.no_accuracy:
            a150 = soft_accuracy(lib, h, s, sc, crd, 0.5, step + 510, st, sp, grid=150)
            g150["force_rel_rms"] = a150["force_rel_rms"]
        close(h, hs)
    ok = bool(torch.isfinite(crd).all().item())
    return {"accuracy": acc, "grid_150": g150,
            "workload": f"{s.n}-atom water + NaCl box with a 64-site soft-core solute, "
                        f"L = {s.box:.2f} A, cutoff 10 A, skin 2 A, "
                        f"PME {systems.fft_size(s.box)}^3, NVE 0.5 fs, alpha 0.5, p 1, "
                        "LJ decoupling windows (solute charges off)",
            "atoms": s.n, "equilibration_steps": EQ, "steps_per_lambda": 500,
            "tuned": (None if args.no_tune else dict(zip(TUNED_KEYS, [int(x) for x in tuned]))),
            "lambdas": runs, "finite": ok}


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from sponge_b200 import capi, systems
    lib = capi.load()
    s = make_box(args.waters, seed=rank)
    n = s.n
    opts = capi.options(cutoff=CUTOFF, skin=SKIN)
    h = ctypes.c_void_p()
    t = np.ascontiguousarray(s.lj_type, np.int32)
    A = np.ascontiguousarray(s.lj_A, np.float32)
    B = np.ascontiguousarray(s.lj_B, np.float32)
    q = np.ascontiguousarray(s.charge, np.float32)
    es = np.ascontiguousarray(s.excl_start, np.int32)
    en = np.ascontiguousarray(s.excl_numbers, np.int32)
    el = np.ascontiguousarray(s.excl_list, np.int32)
    capi.check(lib.snb_engine_create(ctypes.byref(opts), n, capi.boundary(s.cell(), s.rcell()),
                                     s.n_types, t.ctypes.data, A.ctypes.data, B.ctypes.data,
                                     q.ctypes.data, es.ctypes.data, en.ctypes.data,
                                     el.ctypes.data, len(el), ctypes.byref(h)), "engine_create")
    nb, na = len(s.bonds), len(s.angles)
    ba = np.ascontiguousarray(s.bonds[:, 0], np.int32)
    bb = np.ascontiguousarray(s.bonds[:, 1], np.int32)
    bk = np.full(nb, systems.BOND_K, np.float32)
    br = np.full(nb, systems.BOND_R0, np.float32)
    aa = np.ascontiguousarray(s.angles[:, 0], np.int32)
    ab = np.ascontiguousarray(s.angles[:, 1], np.int32)
    ac = np.ascontiguousarray(s.angles[:, 2], np.int32)
    ak = np.full(na, systems.ANGLE_K, np.float32)
    at = np.full(na, systems.ANGLE_T0, np.float32)
    capi.check(lib.snb_engine_set_bonded(h, nb, ba.ctypes.data, bb.ctypes.data, bk.ctypes.data,
                                         br.ctypes.data, na, aa.ctypes.data, ab.ctypes.data,
                                         ac.ctypes.data, ak.ctypes.data, at.ctypes.data),
               "set_bonded")
    crd = torch.from_numpy(s.crd.reshape(-1).copy()).cuda()
    vel = torch.from_numpy(s.vel.reshape(-1).copy()).cuda()
    invm = torch.from_numpy((1.0 / s.mass).astype(np.float32)).cuda()
    dt = DT_FS * 1e-3 * systems.TIME_CONVERSION
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    K, W = args.steps, max(args.warmup, 3)

    run_steps = lib.snb_engine_md_steps if args.no_graph else lib.snb_engine_md_steps_graph

    def steps(first, k):
        capi.check(run_steps(h, P(crd), P(vel), P(invm), ctypes.c_float(dt), first, k, sp),
                   "md_steps")

    EQ = max(0, args.equilibrate)
    # Untimed equilibration from the lattice start, with the velocities
    # rescaled to 300 K every 100 steps (the start releases potential energy
    # that would otherwise heat the box far above 300 K), then plain NVE.
    mass = torch.from_numpy(s.mass.astype(np.float64)).cuda()
    for c0 in range(0, EQ, 100):
        with torch.cuda.stream(st):
            steps(c0, min(100, EQ - c0))
            v = vel.view(n, 3).double()
            ke = 0.5 * (mass[:, None] * v * v).sum()
            t_now = 2.0 * ke / (3.0 * n * systems.KB)
            vel.mul_(float(torch.sqrt(300.0 / t_now)))
    tuned = np.zeros(9, np.int32)
    if not args.no_tune:
        with torch.cuda.stream(st):
            capi.check(lib.snb_engine_autotune(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                               30, tuned.ctypes.data, sp), "autotune")
    with torch.cuda.stream(st):
        steps(EQ, W)
    st.synchronize()
    r0 = ctypes.c_longlong(0)
    capi.check(lib.snb_engine_stats(h, ctypes.byref(r0), None, sp), "stats")
    pp0, pp1 = ctypes.c_int(0), ctypes.c_int(0)
    capi.check(lib.snb_engine_prune_passes(h, ctypes.byref(pp0), None, sp), "prune passes")
    # state at the start of the timed region: the reference's GPU path
    # starts from it too (plain_gpu below)
    start_state = (crd.clone(), vel.clone())
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_win0 = time.perf_counter()
    e0.record(st)
    with torch.cuda.stream(st):
        steps(EQ + W, K)
    e1.record(st)
    st.synchronize()
    torch.cuda.synchronize()
    t_win1 = time.perf_counter()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop((t_win0, t_win1))
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * ns_per_day(K / (ms_max / 1e3))

    r1 = ctypes.c_longlong(0)
    capi.check(lib.snb_engine_stats(h, ctypes.byref(r1), None, sp), "stats")
    capi.check(lib.snb_engine_prune_passes(h, ctypes.byref(pp1), None, sp), "prune passes")
    timed_rebuilds = int(r1.value - r0.value)
    timed_prunes = int(pp1.value - pp0.value)
    # graph composition: our kernels per step
    kn, libk, bodyk = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    if not args.no_graph:  # with --no-graph no step graph exists to count
        capi.check(lib.snb_engine_graph_info(h, ctypes.byref(kn), ctypes.byref(libk),
                                             ctypes.byref(bodyk), sp), "graph_info")
    ours_per_step = kn.value - libk.value
    forced_steps = sum(1 for x in range(EQ + W, EQ + W + K) if x % 100 == 0)

    # per-phase timing (stream launches, events between phases)
    phases = np.zeros(7)
    pq0, pq1, kept = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_longlong(0)
    capi.check(lib.snb_engine_prune_passes(h, ctypes.byref(pq0), None, sp), "prune passes")
    with torch.cuda.stream(st):
        capi.check(lib.snb_engine_profile_steps(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                                EQ + W + K, args.profile_steps,
                                                phases.ctypes.data, sp), "profile")
    capi.check(lib.snb_engine_prune_passes(h, ctypes.byref(pq1), ctypes.byref(kept), sp),
               "prune passes")
    rebuilds, pairs = ctypes.c_longlong(0), ctypes.c_longlong(0)
    capi.check(lib.snb_engine_stats(h, ctypes.byref(rebuilds), ctypes.byref(pairs), sp), "stats")

    # accuracy of the step's forces, energies and virial at the frame the
    # timed steps left, against the FP64 oracle (outside every timed region)
    acc = None
    if not args.no_accuracy and rank == 0:
        acc = headline_accuracy(lib, h, s, crd, EQ + W + K, st, sp)

    # the rebuild cost (one forced rebuild step minus a plain one, medians of
    # five each) and the rate over the run, for a rebuild-amortised value
    reb_ms, plain_ms = [], []
    for k in range(5):
        reb_ms.append(_timed_steps(lib, h, crd, vel, invm, dt, 100 * (100000 + k), 1, st, sp))
        plain_ms.append(_timed_steps(lib, h, crd, vel, invm, dt, 100 * (100000 + k) + 1, 1,
                                     st, sp))
    rebuild_cost_ms = max(0.0, statistics.median(reb_ms) - statistics.median(plain_ms))

    # end-to-end through the public API with host buffers: every call copies
    # crd + vel from pinned host memory, runs one step and copies crd + vel
    # back (snb_engine_md_steps_host, one synchronisation per call)
    # (the state sits in one [crd | vel] array on each side, so each
    # direction is one copy; one untimed call captures the step graph for
    # these buffers)
    E = max(10, min(K, 200))
    host_steps = lib.snb_engine_md_steps_host if not args.no_graph else None
    if host_steps is not None:
        d_state = torch.cat([crd, vel])
        h_state = d_state.cpu().pin_memory()
        d_crd, d_vel = d_state[:3 * n], d_state[3 * n:]
        h_crd, h_vel = h_state[:3 * n], h_state[3 * n:]
        with torch.cuda.stream(st):
            capi.check(host_steps(h, P(h_crd), P(h_vel), P(d_crd), P(d_vel), P(invm),
                                  ctypes.c_float(dt), EQ + W + K + 999, 1, sp), "e2e warm-up")
    else:
        h_crd = torch.from_numpy(crd.cpu().numpy().copy()).pin_memory()
        h_vel = torch.from_numpy(vel.cpu().numpy().copy()).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(st):
        for k in range(E):
            if host_steps is not None:
                capi.check(host_steps(h, P(h_crd), P(h_vel), P(d_crd), P(d_vel), P(invm),
                                      ctypes.c_float(dt), EQ + W + K + 1000 + k, 1, sp),
                           "e2e step")
                continue
            crd.copy_(h_crd, non_blocking=True)
            vel.copy_(h_vel, non_blocking=True)
            capi.check(run_steps(h, P(crd), P(vel), P(invm), ctypes.c_float(dt),
                                 EQ + W + K + 1000 + k, 1, sp), "e2e step")
            h_crd.copy_(crd, non_blocking=True)
            h_vel.copy_(vel, non_blocking=True)
            st.synchronize()
    t_e2e = time.perf_counter() - t0
    if host_steps is not None:  # the run continues from the e2e leg's state
        crd.copy_(d_crd)
        vel.copy_(d_vel)
        torch.cuda.synchronize()
    e2e_t = torch.tensor([t_e2e], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * ns_per_day(E / float(e2e_t.item()))
    io_bytes = 2 * 3 * 4 * n

    drift = None
    # rebuilds per step of plain NVE at 300 K: over the drift run when there
    # is one, else over the timed steps (at least the forced one per 100)
    rebuild_rate_seen = max(timed_rebuilds / K, 0.01)
    if args.drift_steps > 0:
        d0, d1 = ctypes.c_longlong(0), ctypes.c_longlong(0)
        capi.check(lib.snb_engine_stats(h, ctypes.byref(d0), None, sp), "stats")
        drift = nve_drift(lib, h, s, crd, vel, invm, EQ + W + K + 2000 + E,
                          args.drift_steps, 21, dt, run_steps, st, sp)
        capi.check(lib.snb_engine_stats(h, ctypes.byref(d1), None, sp), "stats")
        rebuild_rate_seen = (d1.value - d0.value) / max(1, drift["steps"] + drift["samples"])

    # the reference's own GPU path against this engine over the same steps
    # from the same state (the timed region's start); this engine's first
    # step there is a forced rebuild (a multiple of 100), as its list was
    # built for another frame
    plain = None
    if args.plain_gpu_steps > 0 and rank == 0 and world == 1:
        PK = args.plain_gpu_steps
        crd.copy_(start_state[0])
        vel.copy_(start_state[1])
        ms_same = _timed_steps(lib, h, crd, vel, invm, dt, 100 * 200000, PK, st, sp)
        try:
            plain = plain_gpu_run(s, start_state[0].cpu().numpy().reshape(n, 3),
                                  start_state[1].cpu().numpy().reshape(n, 3), PK, W)
        except Exception as ex:  # noqa: BLE001
            plain = {"unavailable": f"{type(ex).__name__}: {ex}"}
        plain["this_engine_ms_per_step"] = ms_same / PK
        plain["this_engine_ns_per_day"] = ns_per_day(PK / (ms_same / 1e3))
        if "ns_per_day" in plain:
            plain["speedup_vs_plain"] = plain["this_engine_ns_per_day"] / plain["ns_per_day"]

    # roofline of the dominant kernel (the pair kernel), HBM view.  Per
    # launch, averaged over the profiled steps: the list entries scanned
    # (the full rows on a prune pass, the kept entries otherwise), the
    # positions, forces and row counts, and on a prune pass the kept entries
    # written with the rows' counts and positions
    pair_ms = float(phases[2])
    listed = int(pairs.value)
    prof_prunes = int(pq1.value - pq0.value)
    f_prune = prof_prunes / max(1, args.profile_steps) if kept.value > 0 else 1.0
    kept_n = int(kept.value) if kept.value > 0 else listed
    scanned = f_prune * listed + (1.0 - f_prune) * kept_n
    alg_bytes = (4 * scanned + 16 * n + 24 * n + 4 * (n + 1) + 4 * n
                 + (f_prune * (4 * kept_n + 20 * n) if kept.value > 0 else 0.0))
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (pair_ms * 1e-3) / 1e9
    traffic = committed_traffic()
    roofline = {"bound": "hbm", "kernel": "k_lj_direct", "achieved": achieved,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": (traffic["dram_bytes_per_launch"] if traffic else None),
                "algorithmic_bytes": alg_bytes, "kernel_ms": pair_ms,
                "entries_scanned_per_launch": scanned, "prune_passes_profiled": prof_prunes,
                "profiled_steps": args.profile_steps}
    # FP32-pipe view: 47 flops per in-cutoff pair (force only) + 10 per other
    # scanned entry; in-cutoff count from the oracle-free density estimate
    in_cut = listed * (CUTOFF / (CUTOFF + SKIN)) ** 3
    flops = 47 * in_cut + 10 * (scanned - in_cut)
    roofline["fp32_tflops"] = flops / (pair_ms * 1e-3) / 1e12

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            res, why = cpu_reference_run(make_box(args.waters, seed=0), 10, 3,
                                         rebuild_rate=max(rebuild_rate_seen, 0.01))
            cpu_base = ({k: res[k] for k in ("value", "unit", "cores", "kind", "sample")}
                        if res else {"unavailable": why})
        except Exception as ex:  # noqa: BLE001
            cpu_base = {"unavailable": f"{type(ex).__name__}: {ex}"}

    lib.snb_engine_destroy(h)
    batch = run_batch(args, lib, world, rank, dist) if args.batch_systems > 0 else None
    small = soft_box = None
    if world == 1:  # single-GPU measurements of the other workloads
        if not args.no_small_box:
            small = run_small_box(lib)
        if args.soft_core_waters > 0:
            soft_box = run_soft_core_box(args, lib)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # rebuild-amortised: the timed steps without their own rebuilds, plus the
    # measured rebuild cost at the rate the whole run saw
    rate = rebuild_rate_seen
    ms_amort = (ms_max - timed_rebuilds * rebuild_cost_ms) / K + rate * rebuild_cost_ms
    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded water/NaCl box, random-orientation TIP3P-style waters)",
        "config": bench_config(n),
        "work": WORK_OURS,
        "parallelism": f"replicas ({world} independent boxes)" if world > 1 else "single GPU",
        "accumulation": "64-bit fixed point (forces 2^40, energies and virials 2^32)",
        "equilibration_steps": EQ,
        "nl_rebuilds_timed": timed_rebuilds,
        # pair-kernel passes over the full rows (every rebuild, and whenever
        # an atom moved half the 0.8 A prune margin); the other steps scan
        # only the entries kept within cutoff + margin
        "prune_passes_timed": timed_prunes,
        "forced_rebuild_steps_in_timed_region": forced_steps,
        "value_rebuild_amortised": world * ns_per_day(1e3 / ms_amort),
        "rebuild_amortisation": {"rebuild_cost_ms": rebuild_cost_ms,
                                 "rebuilds_per_step": rebuild_rate_seen,
                                 "ms_per_step": ms_amort},
        "accuracy": acc,
        "plain_gpu": plain,
        "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": io_bytes,
                "d2h_bytes_per_step": io_bytes, "steps": E},
        "gpu_launches": ours_per_step * K + bodyk.value * timed_rebuilds,
        "kernels_per_step": ours_per_step,
        "rebuild_kernels": bodyk.value,
        "library_kernels_per_step": libk.value,
        "phase_ms": dict(zip(["neighbor", "pack", "pair", "excluded", "pme", "bonded",
                              "integrate"], [round(float(x), 5) for x in phases])),
        "nl_rebuilds": int(rebuilds.value), "pairs": listed,
        "nve_drift": drift,
        "tuned": (None if args.no_tune else dict(zip(TUNED_KEYS, [int(x) for x in tuned]))),
        "batch": batch,
        "small_box": small,
        "soft_core_box": soft_box,
        "roofline": roofline, "cpu_baseline": cpu_base, "clocks": clk,
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
