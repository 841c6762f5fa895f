"""Helpers for the -m gpu tests: device buffers from numpy and module handles
over the C ABI (include/sponge_nb.h)."""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from sponge_b200 import capi


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype)))
    return t.cuda()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def bnd(s):
    return capi.boundary(s.cell(), s.rcell())


class Box:
    """Device copies of a systems.System."""

    def __init__(self, s):
        self.s = s
        self.n = s.n
        self.crd = dev(s.crd.reshape(-1), np.float32)
        self.charge = dev(s.charge, np.float32)
        self.es = dev(s.excl_start, np.int32)
        self.en = dev(s.excl_numbers, np.int32)
        el = s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)
        self.el = dev(el, np.int32)
        self.b = bnd(s)


def make_nl(box: Box, cutoff, skin, **opts):
    lib = capi.load()
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, skin=skin, **opts)
    capi.check(lib.snb_nl_create(ctypes.byref(o), box.n, cutoff, skin, box.b,
                                 ctypes.byref(h)), "nl_create")
    return h


def nl_update(h, box: Box, crd=None, forced=1, step=0):
    lib = capi.load()
    capi.check(lib.snb_nl_update(h, None, box.n, 0, ptr(box.crd if crd is None else crd),
                                 box.b, step, forced, ptr(box.es), ptr(box.el),
                                 ptr(box.en), stream()), "nl_update")


def nl_pairs(h):
    """Sorted (i < j) pair array (P, 2) of the current list."""
    lib = capi.load()
    cnt = ctypes.c_longlong(0)
    capi.check(lib.snb_nl_pair_count(h, ctypes.byref(cnt), stream()), "pair_count")
    n = cnt.value
    pi = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    pj = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    capi.check(lib.snb_nl_export_pairs(h, ptr(pi), ptr(pj), n, ctypes.byref(cnt),
                                       stream()), "export_pairs")
    p = np.stack([pi[:n].cpu().numpy(), pj[:n].cpu().numpy()], 1).astype(np.int64)
    order = np.lexsort((p[:, 1], p[:, 0]))
    return p[order]


def csr_to_pairs(rs, cols):
    n = len(rs) - 1
    i = np.repeat(np.arange(n), np.diff(rs))
    return np.stack([i, cols.astype(np.int64)], 1)


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def lj_create(box: Box, cutoff, accumulation="fixed64"):
    lib = capi.load()
    s = box.s
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, accumulation=accumulation)
    t = np.ascontiguousarray(s.lj_type, np.int32)
    A = np.ascontiguousarray(s.lj_A, np.float32)
    B = np.ascontiguousarray(s.lj_B, np.float32)
    capi.check(lib.snb_lj_create(ctypes.byref(o), s.n, s.n_types, t.ctypes.data,
                                 A.ctypes.data, B.ctypes.data, cutoff, ctypes.byref(h)),
               "lj_create")
    return h


def lj_force(h, nl, box: Box, beta, energy=True, virial=True):
    lib = capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    ce = torch.zeros(n, dtype=torch.float32, device="cuda")
    capi.check(lib.snb_lj_pme_direct_force(
        h, n, n, 0, 0, ptr(box.crd), ptr(box.charge), ptr(frc), box.b, nl,
        ctypes.c_float(beta), int(energy), ptr(ae), int(virial), ptr(vir), ptr(ce),
        stream()), "lj_pme_direct_force")
    torch.cuda.synchronize()
    return dict(frc=frc.cpu().numpy().reshape(n, 3), atom_energy=ae.cpu().numpy(),
                virial=vir.cpu().numpy().reshape(n, 6), coulomb_energy=ce.cpu().numpy())


def pme_create(box: Box, cutoff, accumulation="fixed64", **opts):
    lib = capi.load()
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, accumulation=accumulation, **opts)
    L = np.array(getattr(box.s, "lengths", [box.s.box] * 3), np.float32)
    capi.check(lib.snb_pme_create(ctypes.byref(o), box.n, box.b, L.ctypes.data, cutoff,
                                  ctypes.byref(h)), "pme_create")
    beta = float(lib.snb_pme_beta(h))
    g = np.zeros(3, np.int32)
    capi.check(lib.snb_pme_grid(h, g.ctypes.data), "pme_grid")
    return h, beta, tuple(int(x) for x in g)


def pme_reciprocal(h, box: Box, energy=True, virial=True, step=0):
    lib = capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    pot = torch.zeros(1, dtype=torch.float32, device="cuda")
    capi.check(lib.snb_pme_reciprocal_force(h, ptr(box.crd), box.b, ptr(box.charge),
                                            ptr(frc), int(virial), int(energy), ptr(vir),
                                            ptr(pot), step, stream()), "pme_reciprocal")
    rec, slf = ctypes.c_double(0), ctypes.c_double(0)
    v6 = np.zeros(6)
    capi.check(lib.snb_pme_energies(h, ctypes.byref(rec), ctypes.byref(slf),
                                    v6.ctypes.data, stream()), "pme_energies")
    torch.cuda.synchronize()
    return dict(frc=frc.cpu().numpy().reshape(n, 3), virial=vir.cpu().numpy(),
                potential=float(pot.cpu()[0]), e_recip=rec.value, e_self=slf.value,
                virial64=v6)


def pme_excluded(h, box: Box, energy=True, virial=True):
    lib = capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    capi.check(lib.snb_pme_excluded_force(h, n, None, None, ptr(box.crd), box.b,
                                          ptr(box.charge), ptr(box.es), ptr(box.el),
                                          ptr(box.en), ptr(frc), int(energy), ptr(ae),
                                          int(virial), ptr(vir), stream()),
               "pme_excluded")
    torch.cuda.synchronize()
    return dict(frc=frc.cpu().numpy().reshape(n, 3), atom_energy=ae.cpu().numpy(),
                virial=vir.cpu().numpy().reshape(n, 6))


def engine_create(s, cutoff, skin=2.0, accumulation="fixed64", **opts):
    lib = capi.load()
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, skin=skin, accumulation=accumulation, **opts)
    t = np.ascontiguousarray(s.lj_type, np.int32)
    A = np.ascontiguousarray(s.lj_A, np.float32)
    B = np.ascontiguousarray(s.lj_B, np.float32)
    q = np.ascontiguousarray(s.charge, np.float32)
    es = np.ascontiguousarray(s.excl_start, np.int32)
    en = np.ascontiguousarray(s.excl_numbers, np.int32)
    el = np.ascontiguousarray(s.excl_list if len(s.excl_list) else np.zeros(1), np.int32)
    capi.check(lib.snb_engine_create(ctypes.byref(o), s.n, bnd(s), s.n_types,
                                     t.ctypes.data, A.ctypes.data, B.ctypes.data,
                                     q.ctypes.data, es.ctypes.data, en.ctypes.data,
                                     el.ctypes.data, int(len(s.excl_list)),
                                     ctypes.byref(h)), "engine_create")
    return h


def engine_set_water_bonded(h, s):
    from sponge_b200 import systems
    lib = capi.load()
    b = np.ascontiguousarray(s.bonds, np.int32)
    a = np.ascontiguousarray(s.angles, np.int32)
    nb, na = len(b), len(a)
    bk = np.full(max(nb, 1), systems.BOND_K, np.float32)
    br = np.full(max(nb, 1), systems.BOND_R0, np.float32)
    ak = np.full(max(na, 1), systems.ANGLE_K, np.float32)
    at = np.full(max(na, 1), systems.ANGLE_T0, np.float32)
    ba = np.ascontiguousarray(b[:, 0] if nb else np.zeros(1), np.int32)
    bb = np.ascontiguousarray(b[:, 1] if nb else np.zeros(1), np.int32)
    aa = np.ascontiguousarray(a[:, 0] if na else np.zeros(1), np.int32)
    ab = np.ascontiguousarray(a[:, 1] if na else np.zeros(1), np.int32)
    ac = np.ascontiguousarray(a[:, 2] if na else np.zeros(1), np.int32)
    capi.check(lib.snb_engine_set_bonded(h, nb, ba.ctypes.data, bb.ctypes.data,
                                         bk.ctypes.data, br.ctypes.data, na,
                                         aa.ctypes.data, ab.ctypes.data, ac.ctypes.data,
                                         ak.ctypes.data, at.ctypes.data),
               "engine_set_bonded")


def soft_create(box: Box, sc, cutoff, params: dict, accumulation="fixed64"):
    """snb_lj_soft handle for a SoftCore description; params are the
    reference's keys (lambda_lj, soft_core_alpha, ...)."""
    lib = capi.load()
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, accumulation=accumulation, **params)
    arr = lambda a, dt: np.ascontiguousarray(a, dt)  # noqa: E731
    tA, tB = arr(sc.type_A, np.int32), arr(sc.type_B, np.int32)
    AA, AB = arr(sc.AA, np.float32), arr(sc.AB, np.float32)
    BA, BB = arr(sc.BA, np.float32), arr(sc.BB, np.float32)
    mask = arr(sc.mask, np.int32)
    capi.check(lib.snb_lj_soft_create(ctypes.byref(o), box.n, sc.n_types_A, sc.n_types_B,
                                      tA.ctypes.data, tB.ctypes.data, AA.ctypes.data,
                                      AB.ctypes.data, BA.ctypes.data, BB.ctypes.data,
                                      mask.ctypes.data, cutoff, ctypes.byref(h)),
               "lj_soft_create")
    return h


def soft_force(h, nl, box: Box, sc, beta, energy=True, virial=True):
    lib = capi.load()
    n = box.n
    frc = torch.zeros(3 * n, dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    vir = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    ce = torch.zeros(n, dtype=torch.float32, device="cuda")
    dq = dev(sc.charge_B_A, np.float32)
    capi.check(lib.snb_lj_soft_pme_direct_force(
        h, n, n, 0, ptr(box.crd), ptr(box.charge), ptr(dq), ptr(frc), box.b, nl,
        ctypes.c_float(beta), int(energy), ptr(ae), int(virial), ptr(vir), ptr(ce),
        stream()), "lj_soft_pme_direct_force")
    sums = np.zeros(4, np.float32)
    if energy:
        capi.check(lib.snb_lj_soft_energy_sums(h, sums.ctypes.data, stream()),
                   "lj_soft_energy_sums")
    torch.cuda.synchronize()
    return dict(frc=frc.cpu().numpy().reshape(n, 3), atom_energy=ae.cpu().numpy(),
                virial=vir.cpu().numpy().reshape(n, 6), coulomb_energy=ce.cpu().numpy(),
                sums=sums)


def soft_dhdl(h, nl, box: Box, sc, beta):
    lib = capi.load()
    dq = dev(sc.charge_B_A, np.float32)
    out = ctypes.c_double(0)
    capi.check(lib.snb_lj_soft_dh_dlambda(h, ptr(box.crd), ptr(box.charge), ptr(dq), box.b,
                                          nl, ctypes.c_float(beta), 1, ctypes.byref(out),
                                          stream()), "lj_soft_dh_dlambda")
    return out.value


def batch_concat(systems):
    """Concatenated per-atom arrays of several boxes, exclusions made global."""
    cat = lambda name, dt: np.ascontiguousarray(  # noqa: E731
        np.concatenate([getattr(s, name) for s in systems]), dt)
    es, el = [], []
    atom_base = excl_base = 0
    for s in systems:
        es.append(s.excl_start + excl_base)
        el.append(s.excl_list + atom_base)
        atom_base += s.n
        excl_base += len(s.excl_list)
    return dict(
        counts=np.array([s.n for s in systems], np.int32),
        boxes=np.array([[s.box] * 3 for s in systems], np.float32).reshape(-1),
        crd=cat("crd", np.float32).reshape(-1), vel=cat("vel", np.float32).reshape(-1),
        charge=cat("charge", np.float32), lj_type=cat("lj_type", np.int32),
        mass=cat("mass", np.float32),
        excl_start=np.ascontiguousarray(np.concatenate(es), np.int32),
        excl_numbers=cat("excl_numbers", np.int32),
        excl_list=np.ascontiguousarray(np.concatenate(el) if sum(map(len, el)) else
                                       np.zeros(1), np.int32),
        n_excl=int(sum(len(x) for x in el)))


def batch_create(systems, cutoff, skin=2.0, **opts):
    lib = capi.load()
    c = batch_concat(systems)
    s0 = systems[0]
    A = np.ascontiguousarray(s0.lj_A, np.float32)
    B = np.ascontiguousarray(s0.lj_B, np.float32)
    h = ctypes.c_void_p()
    o = capi.options(cutoff=cutoff, skin=skin, **opts)
    capi.check(lib.snb_batch_create(ctypes.byref(o), len(systems), c["counts"].ctypes.data,
                                    c["boxes"].ctypes.data, s0.n_types,
                                    c["lj_type"].ctypes.data, A.ctypes.data, B.ctypes.data,
                                    c["charge"].ctypes.data, c["excl_start"].ctypes.data,
                                    c["excl_numbers"].ctypes.data, c["excl_list"].ctypes.data,
                                    c["n_excl"], ctypes.byref(h)), "batch_create")
    return h, c
