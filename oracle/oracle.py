"""TEST INFRASTRUCTURE ONLY -- Python access to the two checkers.

* ``Oracle``: the C restatement (``libsnb_oracle.so``): FP32 bit-exact neighbor
  pair set and FP64 runs of the LJ/Coulomb direct sum, PME reciprocal part,
  excluded-pair correction and long-range LJ correction.
* ``ReferenceCPU``: the reference's own CPU modules compiled from its sources
  (``oracle/_ref/libsponge_ref*.so``, built by ``make -C oracle ref``).
* ``ReferenceGPU``: the reference's own GPU modules (FP32, float atomics)
  compiled from its sources as CUDA (``oracle/_ref/libsponge_ref_gpu.so``,
  ``make -C oracle refgpu``); one box per process.
* The reference-side adapter (``ref_build/sponge_nb_adapter.*``: SPONGE's
  module structs over this library's C ABI) and its driver, built by
  ``make -C oracle adapter`` into ``oracle/_ref/libsponge_nb_adapter.so``;
  tests/test_gpu_adapter.py loads it.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  The product never does.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsnb_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsponge_ref.so")
REF_EXACT_SO = os.path.join(HERE, "_ref", "libsponge_ref_exact.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libsponge_ref_gpu.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _terms(arrays, k):
    """Contiguous arrays of a term list of k columns: the atom indices (two
    for a bond, k = 4; three for an angle, k = 5) as int32, the parameters as
    float32; padded to length 1 when empty."""
    m = len(arrays[0])
    out = []
    for t, a in enumerate(arrays):
        is_index = t < (2 if k == 4 else 3)
        dt = np.int32 if is_index else np.float32
        x = np.zeros(max(m, 1), dt)
        x[:m] = np.asarray(a, dt)
        out.append(x)
    return out


def reference_sources() -> str | None:
    """The reference's SPONGE/ source folder, from the environment variable
    SPONGE_REFERENCE (the reference checkout's root), or None when unset."""
    root = os.environ.get("SPONGE_REFERENCE")
    return os.path.join(root, "SPONGE") if root else None


def build_oracle(ref_root: str | None = None, with_reference: bool = True,
                 with_gpu: bool = True) -> None:
    """Build the checkers (``make -C oracle [ref]``).  The reference part only
    builds where its sources exist."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE, "libsnb_oracle.so"])
    ref_root = ref_root or reference_sources()
    if with_reference and ref_root and os.path.isdir(ref_root):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"])
        with open(os.path.join(HERE, "_ref", "REFERENCE_SOURCES"), "w") as f:
            f.write(os.path.abspath(ref_root) + "\n")
        if with_gpu:
            subprocess.check_call(["make", "-s", "-C", HERE, "refgpu", f"REF={ref_root}"])
            subprocess.check_call(["make", "-s", "-C", HERE, "adapter", f"REF={ref_root}"])


def built_reference_sources() -> str | None:
    """The reference source folder the last build_oracle() compiled from, when
    it is still present on this machine (absent where only the prebuilt
    checkers travelled)."""
    root = reference_sources()
    if not root:
        try:
            with open(os.path.join(HERE, "_ref", "REFERENCE_SOURCES")) as f:
                root = f.read().strip()
        except OSError:
            return None
    return root if root and os.path.isdir(root) else None


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle(with_reference=False)
        L = ctypes.CDLL(path)
        self.lib = L
        L.snbo_get_beta.restype = ctypes.c_float
        L.snbo_get_beta.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.snbo_nl_pairs.restype = ctypes.c_int64
        L.snbo_nl_pairs.argtypes = [
            ctypes.c_int, _f32p, _f32p, _f32p, ctypes.c_float, ctypes.c_float,
            _i32p, _i32p, _i32p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.snbo_direct_f64.restype = None
        L.snbo_direct_f64.argtypes = [
            ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, _f32p,
            ctypes.c_float, ctypes.c_float, _i64p, _i32p, _f64p, _f64p, _f64p,
            _f64p, _f64p]
        L.snbo_excluded_f64.restype = None
        L.snbo_excluded_f64.argtypes = [
            ctypes.c_int, _f32p, _f32p, _f32p, _f32p, ctypes.c_float, _i32p,
            _i32p, _i32p, _f64p, _f64p, _f64p]
        L.snbo_nb14_f64.restype = None
        L.snbo_nb14_f64.argtypes = [
            ctypes.c_int, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
            _f64p, _f64p, _f64p, _f64p]
        L.snbo_bonded_f64.restype = None
        L.snbo_bonded_f64.argtypes = [
            ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_int, _i32p, _i32p, _i32p,
            _f32p, _f32p, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
            _f64p]
        L.snbo_vatom_f64.restype = ctypes.c_int
        L.snbo_vatom_f64.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, _f32p, _f32p,
                                     _f32p, _f64p, _f64p]
        L.snbo_shake_f64.restype = ctypes.c_int
        L.snbo_shake_f64.argtypes = [
            ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f32p, _f32p, _f64p,
            _f64p, _f64p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            _f64p]
        L.snbo_pme_f64.restype = None
        L.snbo_pme_f64.argtypes = [
            ctypes.c_int, _f32p, _f32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_float, _f64p, ctypes.POINTER(ctypes.c_double),
            ctypes.POINTER(ctypes.c_double), _f64p, ctypes.c_void_p]
        L.snbo_ewald_recip_f64.restype = ctypes.c_double
        L.snbo_ewald_recip_f64.argtypes = [
            ctypes.c_int, _f32p, _f32p, ctypes.c_float, ctypes.c_float,
            ctypes.c_int, ctypes.c_void_p]
        L.snbo_lrc_factor.restype = ctypes.c_float
        L.snbo_lrc_factor.argtypes = [ctypes.c_int, _i32p, ctypes.c_int, _f32p,
                                      ctypes.c_float]
        L.snbo_soft_f64.restype = None
        L.snbo_soft_f64.argtypes = [
            ctypes.c_int, _f32p, _f32p, _f32p, _i32p, _i32p, _i32p, ctypes.c_int,
            ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_float,
            ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
            ctypes.c_float, ctypes.c_float, _i64p, _i32p, _f64p, _f64p, _f64p,
            _f64p, _f64p, _f64p, _f64p, _f64p]
        L.snbo_soft_lrc.restype = None
        L.snbo_soft_lrc.argtypes = [
            ctypes.c_int, _i32p, _i32p, _f32p, _f32p, ctypes.c_float, ctypes.c_float,
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]

    # -- neighbor list (FP32, bit-exact contract) ---------------------------
    def nl_pairs(self, crd, cell, rcell, cutoff, skin, excl_start=None,
                 excl_numbers=None, excl_list=None):
        """Half list as CSR (row_start int64[n+1], cols int32), rows sorted."""
        crd = _c(crd, np.float32).reshape(-1)
        n = crd.size // 3
        if excl_start is None:
            excl_start = np.zeros(n, np.int32)
            excl_numbers = np.zeros(n, np.int32)
            excl_list = np.zeros(1, np.int32)
        es, en = _c(excl_start, np.int32), _c(excl_numbers, np.int32)
        el = _c(excl_list if len(excl_list) else np.zeros(1), np.int32)
        cell, rcell = _c(cell, np.float32), _c(rcell, np.float32)
        total = self.lib.snbo_nl_pairs(n, crd, cell, rcell, cutoff, skin, es,
                                       en, el, None, None, 0)
        total = abs(int(total))
        rs = np.zeros(n + 1, np.int64)
        cols = np.zeros(max(total, 1), np.int32)
        got = self.lib.snbo_nl_pairs(n, crd, cell, rcell, cutoff, skin, es, en,
                                     el, rs.ctypes.data, cols.ctypes.data, total)
        assert got == total, (got, total)
        return rs, cols[:total]

    def nl_pairs_system(self, s, cutoff, skin):
        return self.nl_pairs(s.crd, s.cell(), s.rcell(), cutoff, skin,
                             s.excl_start, s.excl_numbers, s.excl_list)

    def get_beta(self, cutoff, tol=1e-5, precision=0):
        return float(self.lib.snbo_get_beta(cutoff, tol, precision))

    # -- FP64 method runs -----------------------------------------------------
    def direct_f64(self, s, cutoff, beta, row_start, cols):
        n = s.n
        frc = np.zeros(3 * n)
        ae, le, ce, vir = (np.zeros(n), np.zeros(n), np.zeros(n),
                           np.zeros(6 * n))
        self.lib.snbo_direct_f64(
            n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            _c(s.lj_type, np.int32), _c(s.lj_A, np.float32),
            _c(s.lj_B, np.float32), s.cell(), s.rcell(), cutoff, beta,
            _c(row_start, np.int64), _c(cols if len(cols) else np.zeros(1), np.int32),
            frc, ae, le, ce, vir)
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, lj_energy=le,
                    coulomb_energy=ce, virial=vir.reshape(n, 6))

    def excluded_f64(self, s, beta):
        n = s.n
        frc, ae, vir = np.zeros(3 * n), np.zeros(n), np.zeros(6 * n)
        el = s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)
        self.lib.snbo_excluded_f64(
            n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            s.cell(), s.rcell(), beta, _c(s.excl_start, np.int32),
            _c(s.excl_numbers, np.int32), _c(el, np.int32), frc, ae, vir)
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6))

    def nb14_f64(self, s, a, b, A, B, cf):
        """1-4 terms of pairs (a[t], b[t]) with scaled LJ entries A, B and
        Coulomb scale cf, in FP64 (nb14/nb14.cpp:8-103)."""
        n, m = s.n, len(a)
        frc, ae, vir, sums = np.zeros(3 * n), np.zeros(n), np.zeros(6 * n), np.zeros(2)
        z32 = np.zeros(max(m, 1), np.float32)
        zi = np.zeros(max(m, 1), np.int32)
        self.lib.snbo_nb14_f64(
            m, _c(a, np.int32) if m else zi, _c(b, np.int32) if m else zi,
            _c(A, np.float32) if m else z32, _c(B, np.float32) if m else z32,
            _c(cf, np.float32) if m else z32, _c(s.crd, np.float32).reshape(-1),
            _c(s.charge, np.float32), s.cell(), s.rcell(), frc, ae, vir, sums)
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6),
                    lj=sums[0], ee=sums[1])

    def bonded_f64(self, crd, cell, rcell, bonds, angles):
        """Harmonic bonds and angles in FP64 (bond/bond.cpp:15-60,
        angle/angle.cpp:6-80).  bonds = (a, b, k, r0), angles = (a, b, c, k,
        theta0); returns per family the forces, per-atom energies, per-atom
        virials and the energy sum."""
        crd = _c(crd, np.float32).reshape(-1)
        n = crd.size // 3
        ba, bb, bk, br = _terms(bonds, 4)
        aa, ab, ac, ak, at = _terms(angles, 5)
        out = [np.zeros(3 * n), np.zeros(n), np.zeros(6 * n),
               np.zeros(3 * n), np.zeros(n), np.zeros(6 * n), np.zeros(2)]
        self.lib.snbo_bonded_f64(len(bonds[0]), ba, bb, bk, br, len(angles[0]), aa, ab, ac,
                                 ak, at, crd, _c(cell, np.float32), _c(rcell, np.float32),
                                 *out)
        return (dict(frc=out[0].reshape(n, 3), atom_energy=out[1],
                     virial=out[2].reshape(n, 6), energy=out[6][0]),
                dict(frc=out[3].reshape(n, 3), atom_energy=out[4],
                     virial=out[5].reshape(n, 6), energy=out[6][1]))

    def vatom_f64(self, records, cell, rcell, crd, frc):
        """Virtual atoms (types 0-3) in FP64: positions in record order from
        crd, then frc's virtual-atom forces moved onto their sources in
        reverse order.  records = (type [m], virtual [m], from [m, 3],
        param [m, 2]).  Returns (crd, frc, 1 + first bad record or 0)."""
        ty, vi, fr, pa = records
        m = len(ty)
        x = np.array(crd, np.float64).reshape(-1).copy()
        f = np.array(frc, np.float64).reshape(-1).copy()
        bad = self.lib.snbo_vatom_f64(
            m, _c(ty if m else [0], np.int32), _c(vi if m else [0], np.int32),
            _c(fr if m else [[0, 0, 0]], np.int32).reshape(-1),
            _c(pa if m else [[0, 0]], np.float32).reshape(-1), _c(cell, np.float32),
            _c(rcell, np.float32), x, f)
        return x.reshape(-1, 3), f.reshape(-1, 3), int(bad)

    def shake_f64(self, cell, rcell, ai, aj, r0, mass, crd_old, crd, vel, dt,
                  v_factor=1.0, x_factor=1.0, tol=1e-13):
        """Constraints (ai, aj, r0) solved by iterated SHAKE in FP64 from the
        unconstrained crd with the bond vectors of crd_old; returns the new
        crd, vel, the constraint virial [6] and the sweeps used."""
        n, m = len(mass), len(ai)
        x = np.array(crd, np.float64).reshape(-1).copy()
        v = np.array(vel, np.float64).reshape(-1).copy()
        vir = np.zeros(6)
        z = np.zeros(1, np.int32)
        sweeps = self.lib.snbo_shake_f64(
            n, m, _c(ai, np.int32) if m else z, _c(aj, np.int32) if m else z,
            _c(r0, np.float64) if m else np.zeros(1), _c(mass, np.float64),
            _c(cell, np.float32), _c(rcell, np.float32),
            _c(crd_old, np.float64).reshape(-1), x, v, dt, v_factor, x_factor, tol, vir)
        return dict(crd=x.reshape(n, 3), vel=v.reshape(n, 3), virial=vir, sweeps=sweeps)

    def pme_f64(self, s, grid, beta, want_phi=False):
        n = s.n
        frc = np.zeros(3 * n)
        er, es = ctypes.c_double(0), ctypes.c_double(0)
        vir = np.zeros(6)
        phi = np.zeros(int(np.prod(grid))) if want_phi else None
        self.lib.snbo_pme_f64(
            n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            s.cell(), s.rcell(), int(grid[0]), int(grid[1]), int(grid[2]), beta,
            frc, ctypes.byref(er), ctypes.byref(es), vir,
            phi.ctypes.data if want_phi else None)
        out = dict(frc=frc.reshape(n, 3), e_recip=er.value, e_self=es.value,
                   virial=vir)
        if want_phi:
            out["phi"] = phi.reshape(grid)
        return out

    def ewald_recip_f64(self, s, beta, kmax, with_force=True):
        n = s.n
        frc = np.zeros(3 * n) if with_force else None
        e = self.lib.snbo_ewald_recip_f64(
            n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            float(s.box), beta, kmax, frc.ctypes.data if with_force else None)
        return e, (frc.reshape(n, 3) if with_force else None)

    def soft_f64(self, s, sc, cutoff, beta, lam, alpha, p, sigma, sigma_min,
                 row_start, cols):
        """FP64 soft-core direct terms over the half-list rows (row_start,
        cols); sigma and sigma_min are the input lengths (sigma^6 formed in
        float as LJ_SOFT_CORE::Initial does)."""
        n = s.n
        frc = np.zeros(3 * n)
        ae, le, inter, intra, ce = (np.zeros(n) for _ in range(5))
        vir = np.zeros(6 * n)
        dudl = np.zeros(2)
        s6 = float(np.float32(sigma) ** np.float32(6))
        s6min = float(np.float32(sigma_min) ** np.float32(6))
        self.lib.snbo_soft_f64(
            n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            _c(sc.charge_B_A, np.float32), _c(sc.type_A, np.int32),
            _c(sc.type_B, np.int32), _c(sc.mask, np.int32), sc.n_types_A,
            sc.n_types_B, _c(sc.AA, np.float32), _c(sc.AB, np.float32),
            _c(sc.BA, np.float32), _c(sc.BB, np.float32), s.cell(), s.rcell(),
            cutoff, beta, lam, alpha, p, s6, s6min, _c(row_start, np.int64),
            _c(cols if len(cols) else np.zeros(1), np.int32), frc, ae, le, inter,
            intra, ce, vir, dudl)
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, lj_energy=le,
                    inter=inter, intra=intra, coulomb_energy=ce,
                    virial=vir.reshape(n, 6), dudl_lj=float(dudl[0]),
                    dudl_direct=float(dudl[1]))

    def soft_lrc(self, s, sc, lam, cutoff):
        f, fti = ctypes.c_double(0), ctypes.c_double(0)
        self.lib.snbo_soft_lrc(s.n, _c(sc.type_A, np.int32), _c(sc.type_B, np.int32),
                               _c(sc.AB, np.float32), _c(sc.BB, np.float32), lam,
                               cutoff, ctypes.byref(f), ctypes.byref(fti))
        return f.value, fti.value

    def lrc_factor(self, s, cutoff):
        return float(self.lib.snbo_lrc_factor(
            s.n, _c(s.lj_type, np.int32), s.n_types, _c(s.lj_B, np.float32),
            cutoff))


class ReferenceCPU:
    """The reference's own hot-path modules compiled for CPU (OpenMP)."""

    def __init__(self, exact: bool = False):
        path = REF_EXACT_SO if exact else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} missing: build it with `make -C oracle ref` where the "
                "reference sources are present")
        L = ctypes.CDLL(path)
        self.lib = L
        L.ref_init.restype = ctypes.c_int
        L.ref_init.argtypes = [
            ctypes.c_int, _f32p, _f32p, _i32p, ctypes.c_int, _f32p, _f32p,
            _i32p, _i32p, _i32p, ctypes.c_int, _f32p, ctypes.c_float,
            ctypes.c_float, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float)]
        L.ref_grid.argtypes = [_i32p]
        L.ref_nl_update.restype = ctypes.c_int
        L.ref_nl_update.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, _i32p,
                                    ctypes.c_void_p, ctypes.c_longlong, _i32p]
        L.ref_nl_update_only.restype = ctypes.c_int
        L.ref_nl_update_only.argtypes = [_f32p, ctypes.c_int, ctypes.c_int]
        L.ref_lj_direct.restype = ctypes.c_int
        L.ref_lj_direct.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                    ctypes.c_int, ctypes.c_int]
        L.ref_pme_reciprocal.restype = ctypes.c_int
        L.ref_pme_reciprocal.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ref_pme_excluded.restype = ctypes.c_int
        L.ref_pme_excluded.argtypes = [_f32p, _f32p, _f32p, _f32p, ctypes.c_int,
                                       ctypes.c_int]
        L.ref_lj_long_range.restype = ctypes.c_int
        L.ref_lj_long_range.argtypes = [_f32p, _f32p, ctypes.c_float]
        L.ref_lj_long_range_factor.restype = ctypes.c_float
        L.ref_box_change.restype = ctypes.c_int
        L.ref_box_change.argtypes = [_f32p]
        L.ref_soft_init.restype = ctypes.c_int
        L.ref_soft_init.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, _f32p,
                                    _f32p, _f32p, _f32p, _i32p, ctypes.c_char_p]
        L.ref_soft_direct.restype = ctypes.c_int
        L.ref_soft_direct.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                      _f32p, _f32p, ctypes.c_int, ctypes.c_int]
        L.ref_soft_dhdl.restype = ctypes.c_int
        L.ref_soft_dhdl.argtypes = [_f32p, _f32p, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_float)]
        L.ref_soft_long_range.restype = ctypes.c_int
        L.ref_soft_long_range.argtypes = [_f32p, _f32p, ctypes.c_float, _f32p]
        L.ref_nb14.restype = ctypes.c_int
        L.ref_nb14.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f32p, _f32p, _f32p,
                               _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f64p]
        L.ref_vatom.restype = ctypes.c_int
        L.ref_vatom.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _f32p,
                                _f32p, _f32p, _f32p]
        L.ref_bonded.restype = ctypes.c_int
        L.ref_bonded.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f32p, _f32p,
                                 ctypes.c_int, _i32p, _i32p, _i32p, _f32p, _f32p, _f32p,
                                 _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f64p]
        L.ref_settle.restype = ctypes.c_int
        L.ref_settle.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f32p, _f32p, _f32p,
                                 _f32p, _f32p, _f32p, ctypes.c_float, _f32p, _i32p, _i32p]
        L.ref_native_load.restype = ctypes.c_int
        L.ref_native_load.argtypes = [ctypes.c_char_p]
        L.ref_native_get.restype = ctypes.c_longlong
        L.ref_native_get.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        self.n = 0

    def set_threads(self, t: int):
        self.lib.ref_set_threads(int(t))

    def max_threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def init(self, s, cutoff, skin, commands: dict | None = None):
        cmd = ";".join(f"{k}={v}" for k, v in (commands or {}).items())
        beta = ctypes.c_float(0)
        el = s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)
        self.crd = _c(s.crd, np.float32).reshape(-1)
        rc = self.lib.ref_init(
            s.n, self.crd, _c(s.charge, np.float32), _c(s.lj_type, np.int32),
            s.n_types, _c(s.lj_A, np.float32), _c(s.lj_B, np.float32),
            _c(s.excl_start, np.int32), _c(s.excl_numbers, np.int32),
            _c(el, np.int32), int(len(s.excl_list)), s.cell(), cutoff, skin,
            cmd.encode(), ctypes.byref(beta))
        if rc != 0:
            raise RuntimeError("reference init failed")
        self.n = s.n
        self.beta = beta.value
        g = np.zeros(3, np.int32)
        self.lib.ref_grid(g)
        self.grid = tuple(int(x) for x in g)
        return self.beta

    def nl_update(self, crd=None, forced=True, step=0):
        """Half list (reference order inside each row) as (counts, rows)."""
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        counts = np.zeros(self.n, np.int32)
        ov = np.zeros(2, np.int32)
        cap = self.n * 1200
        serial = np.zeros(cap, np.int32)
        rc = self.lib.ref_nl_update(crd, int(forced), step, counts,
                                    serial.ctypes.data, cap, ov)
        if rc != 0:
            raise RuntimeError("reference NL update failed")
        total = int(counts.sum())
        return counts, serial[:total].copy(), ov

    def nl_update_only(self, crd=None, forced=False, step=0):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        if self.lib.ref_nl_update_only(crd, int(forced), step) != 0:
            raise RuntimeError("reference NL update failed")

    def force_step(self, step, crd=None):
        """One force evaluation of the reference MD loop's nonbonded part
        (main.cpp:1389-1544 order): conditional neighbor update, excluded
        correction, LJ + direct Coulomb, PME reciprocal; forces only."""
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        n = self.n
        if not hasattr(self, "_frc"):
            self._frc = np.zeros(3 * n, np.float32)
            self._e = np.zeros(n, np.float32)
            self._v = np.zeros(6 * n, np.float32)
            self._s = np.zeros(6, np.float32)
            self._p = np.zeros(1, np.float32)
            self._parts = np.zeros(2, np.float32)
        self._frc[:] = 0
        L = self.lib
        ok = L.ref_nl_update_only(crd, 0, step) == 0
        ok &= L.ref_pme_excluded(crd, self._frc, self._e, self._v, 0, 0) == 0
        ok &= L.ref_lj_direct(crd, self._frc, self._e, self._v, self._e, self._e, 0, 0) == 0
        ok &= L.ref_pme_reciprocal(crd, self._frc, self._s, self._p, self._parts, 0, 0,
                                   step) == 0
        if not ok:
            raise RuntimeError("reference force step failed")
        return self._frc

    def lj_direct(self, crd=None, need_energy=True, need_virial=True):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        n = self.n
        frc = np.zeros(3 * n, np.float32)
        ae, vir = np.zeros(n, np.float32), np.zeros(6 * n, np.float32)
        le, ce = np.zeros(n, np.float32), np.zeros(n, np.float32)
        rc = self.lib.ref_lj_direct(crd, frc, ae, vir, le, ce, int(need_energy),
                                    int(need_virial))
        if rc != 0:
            raise RuntimeError("reference LJ failed")
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6),
                    lj_energy=le, coulomb_energy=ce)

    def pme_reciprocal(self, crd=None, need_energy=True, need_virial=True, step=0):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        n = self.n
        frc = np.zeros(3 * n, np.float32)
        vir = np.zeros(6, np.float32)
        pot = np.zeros(1, np.float32)
        parts = np.zeros(2, np.float32)
        rc = self.lib.ref_pme_reciprocal(crd, frc, vir, pot, parts,
                                         int(need_energy), int(need_virial), step)
        if rc != 0:
            raise RuntimeError("reference PME failed")
        return dict(frc=frc.reshape(n, 3), virial=vir, potential=float(pot[0]),
                    e_recip=float(parts[0]), e_self=float(parts[1]))

    def pme_excluded(self, crd=None, need_energy=True, need_virial=True):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        n = self.n
        frc = np.zeros(3 * n, np.float32)
        ae, vir = np.zeros(n, np.float32), np.zeros(6 * n, np.float32)
        rc = self.lib.ref_pme_excluded(crd, frc, ae, vir, int(need_energy),
                                       int(need_virial))
        if rc != 0:
            raise RuntimeError("reference excluded correction failed")
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6))

    def native_load(self, files: dict):
        """The reference's native-input loaders on {key: path} (mass_in_file,
        charge_in_file, exclude_in_file, LJ_in_file, LJ_soft_core_in_file,
        subsys_division_in_file, nb14_in_file, nb14_extra_in_file)."""
        cmd = ";".join(f"{k}={v}" for k, v in files.items())
        if self.lib.ref_native_load(cmd.encode()) != 0:
            raise RuntimeError("reference native load failed")

    def native_get(self, name: str, dtype=np.float32):
        n = int(self.lib.ref_native_get(name.encode(), None))
        if n < 0:
            raise KeyError(name)
        out = np.zeros(max(n, 1), dtype)
        self.lib.ref_native_get(name.encode(), out.ctypes.data)
        return out[:n]

    def bonded(self, crd, cell, bonds, angles):
        """BOND and ANGLE of the reference on the given terms in the box
        cell (one force call each): per family forces, per-atom energies,
        per-atom virials and the energy sum Step_Print forms."""
        crd = _c(crd, np.float32).reshape(-1)
        n = crd.size // 3
        ba, bb, bk, br = _terms(bonds, 4)
        aa, ab, ac, ak, at = _terms(angles, 5)
        out = [np.zeros(3 * n, np.float32), np.zeros(n, np.float32),
               np.zeros(6 * n, np.float32), np.zeros(3 * n, np.float32),
               np.zeros(n, np.float32), np.zeros(6 * n, np.float32)]
        sums = np.zeros(2)
        rc = self.lib.ref_bonded(n, len(bonds[0]), ba, bb, bk, br, len(angles[0]), aa, ab,
                                 ac, ak, at, crd, _c(cell, np.float32), *out, sums)
        if rc != 0:
            raise RuntimeError("reference bonded terms failed")
        return (dict(frc=out[0].reshape(n, 3), atom_energy=out[1],
                     virial=out[2].reshape(n, 6), energy=sums[0]),
                dict(frc=out[3].reshape(n, 3), atom_energy=out[4],
                     virial=out[5].reshape(n, 6), energy=sums[1]))

    def vatom(self, records, cell, crd, frc):
        """The reference's own virtual-atom formulas record by record
        (positions in order, forces in reverse order), in FP32."""
        ty, vi, fr, pa = records
        m = len(ty)
        x = np.array(crd, np.float32).reshape(-1).copy()
        f = np.array(frc, np.float32).reshape(-1).copy()
        bad = self.lib.ref_vatom(
            len(x) // 3, m, _c(ty, np.int32), _c(vi, np.int32),
            _c(fr, np.int32).reshape(-1), _c(pa, np.float32).reshape(-1),
            _c(cell, np.float32), x, f)
        return x.reshape(-1, 3), f.reshape(-1, 3), int(bad)

    def nb14(self, s, a, b, A, B, cf):
        """NON_BOND_14 of the reference on pairs (a[t], b[t]) with scaled LJ
        entries A, B and Coulomb scale cf, in s's box (forces, per-atom
        energies and virials, the LJ and Coulomb sums)."""
        n, m = s.n, len(a)
        frc, ae, vir = (np.zeros(3 * n, np.float32), np.zeros(n, np.float32),
                        np.zeros(6 * n, np.float32))
        sums = np.zeros(2)
        pad = max(m, 1)

        def arr(x, dt):
            y = np.zeros(pad, dt)
            y[:m] = x
            return y
        rc = self.lib.ref_nb14(n, m, arr(a, np.int32), arr(b, np.int32), arr(A, np.float32),
                               arr(B, np.float32), arr(cf, np.float32),
                               _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
                               _c(s.cell(), np.float32), frc, ae, vir, sums)
        if rc != 0:
            raise RuntimeError("reference nb14 failed")
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6),
                    lj=float(sums[0]), ee=float(sums[1]))

    def settle(self, cell, ai, aj, r0, mass, crd_old, crd, vel, dt):
        """SETTLE of the reference on one step (see ref_settle): the new crd
        and vel, stress[6] (virial / V), {triangles, pairs, left over} and the
        atom pairs of the constraints left over."""
        n, m = len(mass), len(ai)
        x = np.array(crd, np.float32).reshape(-1).copy()
        v = np.array(vel, np.float32).reshape(-1).copy()
        stress = np.zeros(6, np.float32)
        counts = np.zeros(3, np.int32)
        left = np.zeros(2 * max(m, 1), np.int32)
        pad = lambda a, dt_: np.ascontiguousarray(a, dt_) if m else np.zeros(1, dt_)
        rc = self.lib.ref_settle(n, m, pad(ai, np.int32), pad(aj, np.int32),
                                 pad(r0, np.float32), _c(mass, np.float32),
                                 _c(cell, np.float32), _c(crd_old, np.float32).reshape(-1),
                                 x, v, dt, stress, counts, left)
        if rc != 0:
            raise RuntimeError("reference SETTLE failed")
        return dict(crd=x.reshape(n, 3), vel=v.reshape(n, 3), stress=stress,
                    counts=counts, left=left[:2 * counts[2]].reshape(-1, 2))

    def box_change(self, box):
        """Main_Box_Change for a small change to a cubic box of length `box`:
        later calls use the new boundary; PME's Update_Box has run."""
        cell = np.array([box, 0, box, 0, 0, box], np.float32)
        if self.lib.ref_box_change(cell) != 0:
            raise RuntimeError("reference box change failed")

    def lj_long_range(self, volume):
        vir = np.zeros(6, np.float32)
        pot = np.zeros(1, np.float32)
        self.lib.ref_lj_long_range(vir, pot, volume)
        return dict(virial=vir, potential=float(pot[0]),
                    factor=float(self.lib.ref_lj_long_range_factor()))

    # -- LJ_SOFT_CORE ---------------------------------------------------------
    def soft_init(self, sc, commands: dict):
        cmd = ";".join(f"{k}={v}" for k, v in commands.items())
        rc = self.lib.ref_soft_init(
            _c(sc.type_A, np.int32), _c(sc.type_B, np.int32), sc.n_types_A,
            sc.n_types_B, _c(sc.AA, np.float32), _c(sc.AB, np.float32),
            _c(sc.BA, np.float32), _c(sc.BB, np.float32), _c(sc.mask, np.int32),
            cmd.encode())
        if rc != 0:
            raise RuntimeError("reference soft-core init failed")

    def soft_direct(self, crd=None, need_energy=True, need_virial=True):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        n = self.n
        frc = np.zeros(3 * n, np.float32)
        ae, vir = np.zeros(n, np.float32), np.zeros(6 * n, np.float32)
        le, inter, intra, ce = (np.zeros(n, np.float32) for _ in range(4))
        rc = self.lib.ref_soft_direct(crd, frc, ae, vir, le, inter, intra, ce,
                                      int(need_energy), int(need_virial))
        if rc != 0:
            raise RuntimeError("reference soft-core force failed")
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, virial=vir.reshape(n, 6),
                    lj_energy=le, inter=inter, intra=intra, coulomb_energy=ce)

    def soft_dhdl(self, charge_B_A, crd=None, charge_perturbated=1):
        crd = self.crd if crd is None else _c(crd, np.float32).reshape(-1)
        out = ctypes.c_float(0)
        rc = self.lib.ref_soft_dhdl(crd, _c(charge_B_A, np.float32),
                                    int(charge_perturbated), ctypes.byref(out))
        if rc != 0:
            raise RuntimeError("reference soft-core dH/dlambda failed")
        return float(out.value)

    def soft_long_range(self, volume):
        vir = np.zeros(6, np.float32)
        pot = np.zeros(1, np.float32)
        fac = np.zeros(2, np.float32)
        if self.lib.ref_soft_long_range(vir, pot, volume, fac) != 0:
            raise RuntimeError("reference soft-core tail failed")
        return dict(virial=vir, potential=float(pot[0]), factor=float(fac[0]),
                    factor_ti=float(fac[1]))


class ReferenceGPU:
    """The reference's own GPU modules (neighbor list, LJ + direct Coulomb,
    PME with the excluded correction, bonds, angles) driven in main.cpp's
    order by ``ref_build/ref_harness_gpu.cu``.  FP32 with float atomics on
    the legacy default stream.  The library holds one box per process."""

    def __init__(self):
        if not os.path.exists(REF_GPU_SO):
            raise FileNotFoundError(
                f"{REF_GPU_SO} missing: build it with `make -C oracle refgpu` where "
                "the reference sources are present")
        L = ctypes.CDLL(REF_GPU_SO)
        self.lib = L
        L.refg_last_error.restype = ctypes.c_char_p
        L.refg_init.restype = ctypes.c_int
        L.refg_init.argtypes = [
            ctypes.c_int, _f32p, _f32p, _i32p, ctypes.c_int, _f32p, _f32p,
            _i32p, _i32p, _i32p, ctypes.c_int, _f32p, ctypes.c_float,
            ctypes.c_float, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float)]
        L.refg_grid.argtypes = [_i32p]
        L.refg_set_bonded.restype = ctypes.c_int
        L.refg_set_bonded.argtypes = [ctypes.c_int, _i32p, _i32p, _f32p, _f32p,
                                      ctypes.c_int, _i32p, _i32p, _i32p, _f32p, _f32p]
        L.refg_set_state.restype = ctypes.c_int
        L.refg_set_state.argtypes = [_f32p, ctypes.c_void_p, ctypes.c_void_p]
        L.refg_get_state.restype = ctypes.c_int
        L.refg_get_state.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.refg_force.restype = ctypes.c_int
        L.refg_force.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p]
        L.refg_md_steps.restype = ctypes.c_int
        L.refg_md_steps.argtypes = [ctypes.c_int, ctypes.c_float,
                                    ctypes.POINTER(ctypes.c_float)]
        L.refg_pair_count.restype = ctypes.c_int
        L.refg_pair_count.argtypes = [ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_int)]
        self.n = 0

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"reference GPU {what} failed: "
                               f"{self.lib.refg_last_error().decode()}")

    def init(self, s, cutoff, skin, commands: dict | None = None):
        cmd = ";".join(f"{k}={v}" for k, v in (commands or {}).items())
        beta = ctypes.c_float(0)
        el = s.excl_list if len(s.excl_list) else np.zeros(1, np.int32)
        self._ok(self.lib.refg_init(
            s.n, _c(s.crd, np.float32).reshape(-1), _c(s.charge, np.float32),
            _c(s.lj_type, np.int32), s.n_types, _c(s.lj_A, np.float32),
            _c(s.lj_B, np.float32), _c(s.excl_start, np.int32),
            _c(s.excl_numbers, np.int32), _c(el, np.int32), int(len(s.excl_list)),
            s.cell(), cutoff, skin, cmd.encode(), ctypes.byref(beta)), "init")
        self.n = s.n
        self.beta = beta.value
        g = np.zeros(3, np.int32)
        self.lib.refg_grid(g)
        self.grid = tuple(int(x) for x in g)
        return self.beta

    def set_bonded(self, bonds, bond_k, bond_r0, angles, angle_k, angle_t0):
        b = np.ascontiguousarray(bonds, np.int32).reshape(-1, 2)
        a = np.ascontiguousarray(angles, np.int32).reshape(-1, 3)
        nb, na = len(b), len(a)
        self._keep = [np.ascontiguousarray(x) for x in (
            b[:, 0], b[:, 1], a[:, 0], a[:, 1], a[:, 2])]
        self._ok(self.lib.refg_set_bonded(
            nb, self._keep[0], self._keep[1], np.full(nb, bond_k, np.float32),
            np.full(nb, bond_r0, np.float32), na, self._keep[2], self._keep[3],
            self._keep[4], np.full(na, angle_k, np.float32),
            np.full(na, angle_t0, np.float32)), "set_bonded")

    def set_state(self, crd, vel=None, inv_mass=None):
        crd = _c(crd, np.float32).reshape(-1)
        v = None if vel is None else _c(vel, np.float32).reshape(-1)
        m = None if inv_mass is None else _c(inv_mass, np.float32)
        self._ok(self.lib.refg_set_state(
            crd, None if v is None else v.ctypes.data,
            None if m is None else m.ctypes.data), "set_state")

    def get_state(self):
        crd = np.zeros(3 * self.n, np.float32)
        vel = np.zeros(3 * self.n, np.float32)
        self._ok(self.lib.refg_get_state(crd.ctypes.data, vel.ctypes.data), "get_state")
        return crd.reshape(-1, 3), vel.reshape(-1, 3)

    def force(self, forced=True, need_energy=True, need_virial=True):
        """Nonbonded forces, per-atom energies (LJ + direct + excluded),
        the box-level potential (reciprocal + self + tail) and the summed
        virial of one evaluation on the current coordinates."""
        n = self.n
        frc = np.zeros(3 * n, np.float32)
        ae = np.zeros(n, np.float32)
        pot = np.zeros(1, np.float32)
        vir = np.zeros(6, np.float32)
        self._ok(self.lib.refg_force(int(forced), int(need_energy), int(need_virial),
                                     frc.ctypes.data, ae.ctypes.data, pot.ctypes.data,
                                     vir.ctypes.data), "force")
        return dict(frc=frc.reshape(n, 3), atom_energy=ae, potential=float(pot[0]),
                    virial=vir)

    def md_steps(self, steps, dt):
        """NVE steps; returns their device time in ms."""
        ms = ctypes.c_float(0)
        self._ok(self.lib.refg_md_steps(int(steps), float(dt), ctypes.byref(ms)),
                 "md_steps")
        return float(ms.value)

    def pair_count(self):
        c = ctypes.c_longlong(0)
        ov = ctypes.c_int(0)
        self._ok(self.lib.refg_pair_count(ctypes.byref(c), ctypes.byref(ov)), "pair_count")
        return int(c.value), int(ov.value)
