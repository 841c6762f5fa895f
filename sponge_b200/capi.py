"""ctypes binding of the C ABI in include/sponge_nb.h.

The library is ``sponge_b200/libsponge_nb.so`` built in-tree by
``sponge_b200/build.py``.  Loading fails loudly when it is missing: there is no
CPU fallback for any entry point.  Device buffers are passed as raw pointers
(``torch.Tensor.data_ptr()``), streams as ``torch.cuda.Stream.cuda_stream``.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsponge_nb.so")

_lib = None


class SnbError(RuntimeError):
    pass


class snb_boundary(ctypes.Structure):
    _fields_ = [("policy", ctypes.c_int), ("cell", ctypes.c_float * 6),
                ("rcell", ctypes.c_float * 6)]


class snb_options(ctypes.Structure):
    _fields_ = [
        ("cutoff", ctypes.c_float), ("skin", ctypes.c_float),
        ("nl_refresh_interval", ctypes.c_int), ("nl_skin_permit", ctypes.c_float),
        ("nl_max_neighbor_numbers", ctypes.c_int),
        ("nl_max_atom_in_grid_numbers", ctypes.c_int),
        ("nl_max_ghost_in_grid_numbers", ctypes.c_int),
        ("nl_check_overflow_interval", ctypes.c_int),
        ("nl_throw_error_when_overflow", ctypes.c_int),
        ("pm_fftx", ctypes.c_int), ("pm_ffty", ctypes.c_int), ("pm_fftz", ctypes.c_int),
        ("pm_grid_spacing", ctypes.c_float), ("pm_direct_tolerance", ctypes.c_float),
        ("pme_update_interval", ctypes.c_int),
        ("pme_calculate_reciprocal_part", ctypes.c_int),
        ("pme_calculate_excluded_part", ctypes.c_int),
        ("lambda_lj", ctypes.c_float), ("soft_core_alpha", ctypes.c_float),
        ("soft_core_powfer", ctypes.c_float), ("soft_core_sigma", ctypes.c_float),
        ("soft_core_sigma_min", ctypes.c_float), ("accumulation", ctypes.c_int),
        ("dom_dec_update_interval", ctypes.c_int),
    ]


EXPORTED = [
    "snb_version", "snb_last_error", "snb_options_default", "snb_options_set",
    "snb_check_erfc_exp",
    "snb_nl_create", "snb_nl_update", "snb_nl_check_overflow", "snb_nl_pair_count",
    "snb_nl_export_pairs", "snb_nl_export_atom_groups", "snb_nl_destroy",
    "snb_lj_create", "snb_lj_get_local", "snb_lj_pme_direct_force", "snb_solvent_lj_pme_direct_force",
    "snb_lj_long_range_correction", "snb_lj_energy_sum", "snb_lj_long_range_factor",
    "snb_lj_destroy",
    "snb_lj_soft_create", "snb_lj_soft_pme_direct_force", "snb_lj_soft_dh_dlambda",
    "snb_lj_soft_long_range_correction", "snb_lj_soft_energy_sums", "snb_lj_soft_destroy",
    "snb_pme_create", "snb_pme_beta", "snb_pme_grid", "snb_pme_reciprocal_force",
    "snb_pme_excluded_force", "snb_pme_energies", "snb_pme_spread_wide_tiles", "snb_pme_update_box", "snb_pme_destroy",
    "snb_pme_excluded_force_noalloc",
    "snb_engine_create", "snb_batch_create", "snb_engine_force", "snb_engine_set_bonded",
    "snb_engine_set_soft_core", "snb_engine_update_box", "snb_engine_set_nb14",
    "snb_nb14_create", "snb_nb14_force", "snb_nb14_energy_sums", "snb_nb14_destroy",
    "snb_engine_set_settle", "snb_engine_pressure", "snb_settle_create", "snb_settle_group", "snb_settle_counts",
    "snb_settle_remember_last_coordinates", "snb_settle_do", "snb_settle_status",
    "snb_settle_destroy",
    "snb_engine_md_steps", "snb_engine_md_steps_graph", "snb_engine_md_steps_host",
    "snb_engine_profile_steps",
    "snb_engine_autotune", "snb_engine_set_launch_shapes", "snb_engine_graph_info",
    "snb_engine_stats",
    "snb_engine_spread_wide_tiles", "snb_engine_set_list_form", "snb_engine_list_form",
    "snb_engine_set_prune_margin", "snb_engine_prune_passes",
    "snb_engine_export_pairs",
    "snb_engine_destroy",
    "snb_bond_create", "snb_bond_force", "snb_bond_energy", "snb_bond_destroy",
    "snb_angle_create", "snb_angle_force", "snb_angle_energy", "snb_angle_destroy",
    "snb_read_bond_in_file", "snb_read_angle_in_file", "snb_read_virtual_atom_in_file",
    "snb_vatom_create", "snb_vatom_levels", "snb_vatom_coordinate_refresh",
    "snb_vatom_force_redistribute", "snb_vatom_status", "snb_vatom_destroy",
    "snb_engine_set_virtual_atoms",
    "snb_read_lj_in_file", "snb_read_lj_soft_core_in_file", "snb_read_subsys_division_in_file",
    "snb_read_charge_in_file", "snb_read_mass_in_file", "snb_read_exclude_in_file",
    "snb_read_nb14_in_file", "snb_append_frc_traj",
]

# status codes of include/sponge_nb.h
SNB_OK = 0
SNB_ERR_BAD_INPUT = 1
SNB_ERR_CUDA = 2
SNB_ERR_OVERFLOW = 3
SNB_ERR_TIMEOUT = 4
SNB_ERR_NOT_SUPPORTED = 5

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_LL = ctypes.c_longlong

_SIGS = {
    "snb_version": (_I, []),
    "snb_last_error": (ctypes.c_char_p, []),
    "snb_options_default": (None, [ctypes.POINTER(snb_options)]),
    "snb_options_set": (_I, [ctypes.POINTER(snb_options), ctypes.c_char_p,
                             ctypes.c_char_p]),
    "snb_nl_create": (_I, [ctypes.POINTER(snb_options), _I, _F, _F, snb_boundary,
                           ctypes.POINTER(_P)]),
    "snb_nl_update": (_I, [_P, _P, _I, _I, _P, snb_boundary, _I, _I, _P, _P, _P, _P]),
    "snb_nl_check_overflow": (_I, [_P, ctypes.POINTER(_I), _P]),
    "snb_nl_pair_count": (_I, [_P, ctypes.POINTER(_LL), _P]),
    "snb_nl_export_pairs": (_I, [_P, _P, _P, _LL, ctypes.POINTER(_LL), _P]),
    "snb_nl_export_atom_groups": (_I, [_P, _P, _P, _I, _P]),
    "snb_nl_destroy": (_I, [_P]),
    "snb_lj_create": (_I, [ctypes.POINTER(snb_options), _I, _I, _P, _P, _P, _F,
                           ctypes.POINTER(_P)]),
    "snb_lj_get_local": (_I, [_P, _P, _I, _I, _P]),
    "snb_lj_pme_direct_force": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, snb_boundary, _P,
                                     _F, _I, _P, _I, _P, _P, _P]),
    "snb_solvent_lj_pme_direct_force": (_I, [_P, _P, _I, _I, _P, _P, _P, snb_boundary, _F,
                                             _I, _P, _I, _P, _P, _P]),
    "snb_lj_long_range_correction": (_I, [_P, _I, _P, _I, _P, _F, _P]),
    "snb_lj_energy_sum": (_I, [_P, ctypes.POINTER(_F), _P]),
    "snb_lj_long_range_factor": (_F, [_P]),
    "snb_lj_destroy": (_I, [_P]),
    "snb_lj_soft_create": (_I, [ctypes.POINTER(snb_options), _I, _I, _I, _P, _P, _P,
                                _P, _P, _P, _P, _F, ctypes.POINTER(_P)]),
    "snb_lj_soft_pme_direct_force": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, snb_boundary,
                                          _P, _F, _I, _P, _I, _P, _P, _P]),
    "snb_lj_soft_dh_dlambda": (_I, [_P, _P, _P, _P, snb_boundary, _P, _F, _I,
                                    ctypes.POINTER(ctypes.c_double), _P]),
    "snb_lj_soft_long_range_correction": (_I, [_P, _I, _P, _I, _P, _F, _P]),
    "snb_lj_soft_energy_sums": (_I, [_P, _P, _P]),
    "snb_lj_soft_destroy": (_I, [_P]),
    "snb_pme_create": (_I, [ctypes.POINTER(snb_options), _I, snb_boundary, _P, _F,
                            ctypes.POINTER(_P)]),
    "snb_pme_beta": (_F, [_P]),
    "snb_pme_grid": (_I, [_P, _P]),
    "snb_pme_reciprocal_force": (_I, [_P, _P, snb_boundary, _P, _P, _I, _I, _P, _P, _I,
                                      _P]),
    "snb_pme_excluded_force": (_I, [_P, _I, _P, _P, _P, snb_boundary, _P, _P, _P, _P, _P,
                                    _I, _P, _I, _P, _P]),
    "snb_pme_update_box": (_I, [_P, snb_boundary, _P, _F]),
    "snb_pme_energies": (_I, [_P, _P, _P, _P, _P]),
    "snb_pme_spread_wide_tiles": (_I, [_P, ctypes.POINTER(ctypes.c_int), _P]),
    "snb_check_erfc_exp": (_I, [_I, _P, _P, _P]),
    "snb_pme_destroy": (_I, [_P]),
    "snb_pme_excluded_force_noalloc": (_I, [_I, _P, snb_boundary, _P, _F, _P, _P, _P, _P,
                                            _I, _P, _I, _P, _P]),
    "snb_engine_create": (_I, [ctypes.POINTER(snb_options), _I, snb_boundary, _I, _P,
                               _P, _P, _P, _P, _P, _P, _I, ctypes.POINTER(_P)]),
    "snb_batch_create": (_I, [ctypes.POINTER(snb_options), _I, _P, _P, _I, _P, _P, _P, _P,
                              _P, _P, _P, _I, ctypes.POINTER(_P)]),
    "snb_engine_force": (_I, [_P, _P, _P, _I, _I, _I, _P, _P]),
    "snb_engine_set_bonded": (_I, [_P, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "snb_engine_set_soft_core": (_I, [_P, _P]),
    "snb_engine_update_box": (_I, [_P, snb_boundary]),
    "snb_engine_set_nb14": (_I, [_P, _P]),
    "snb_nb14_create": (_I, [_I, _I, _P, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "snb_nb14_force": (_I, [_P, _P, _P, snb_boundary, _P, _I, _P, _I, _P, _P]),
    "snb_nb14_energy_sums": (_I, [_P, _P, _P, _P]),
    "snb_nb14_destroy": (_I, [_P]),
    "snb_engine_set_settle": (_I, [_P, _P]),
    "snb_engine_pressure": (_I, [_P, _P, _P, _P, _P, _P]),
    "snb_settle_create": (_I, [_I, _I, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "snb_settle_group": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "snb_settle_counts": (_I, [_P, _P, _P, _P, _P]),
    "snb_settle_remember_last_coordinates": (_I, [_P, _P, snb_boundary, _P]),
    "snb_settle_do": (_I, [_P, _P, snb_boundary, _P, _F, _F, _F, _I, _P, _P]),
    "snb_settle_status": (_I, [_P, _P, _P]),
    "snb_settle_destroy": (_I, [_P]),
    "snb_read_nb14_in_file": (_I, [ctypes.c_char_p, ctypes.c_char_p, _I, _P, _P, _P, _P,
                                   _P, _P, _P, _P, _P]),
    "snb_read_lj_in_file": (_I, [ctypes.c_char_p, _P, _P, _P, _P, _P]),
    "snb_read_lj_soft_core_in_file": (_I, [ctypes.c_char_p, _P, _P, _P, _P, _P, _P, _P,
                                           _P, _P]),
    "snb_read_subsys_division_in_file": (_I, [ctypes.c_char_p, _P, _P]),
    "snb_read_charge_in_file": (_I, [ctypes.c_char_p, _P, _P]),
    "snb_read_mass_in_file": (_I, [ctypes.c_char_p, _P, _P]),
    "snb_read_exclude_in_file": (_I, [ctypes.c_char_p, _P, _P, _P, _P, _P]),
    "snb_append_frc_traj": (_I, [ctypes.c_char_p, _P, _I, _P]),
    "snb_engine_md_steps": (_I, [_P, _P, _P, _P, _F, _I, _I, _P]),
    "snb_engine_md_steps_graph": (_I, [_P, _P, _P, _P, _F, _I, _I, _P]),
    "snb_engine_md_steps_host": (_I, [_P, _P, _P, _P, _P, _P, _F, _I, _I, _P]),
    "snb_engine_profile_steps": (_I, [_P, _P, _P, _P, _F, _I, _I, _P, _P]),
    "snb_engine_autotune": (_I, [_P, _P, _P, _P, _F, _I, _P, _P]),
    "snb_engine_set_launch_shapes": (_I, [_P, _P]),
    "snb_engine_graph_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I),
                                   ctypes.POINTER(_I), _P]),
    "snb_engine_stats": (_I, [_P, ctypes.POINTER(_LL), ctypes.POINTER(_LL), _P]),
    "snb_engine_spread_wide_tiles": (_I, [_P, ctypes.POINTER(ctypes.c_int), _P]),
    "snb_engine_set_list_form": (_I, [_P, _I]),
    "snb_engine_set_prune_margin": (_I, [_P, _F]),
    "snb_engine_prune_passes": (_I, [_P, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_longlong), _P]),
    "snb_bond_create": (_I, [_I, _I, _P, _P, _P, _P, _P]),
    "snb_bond_force": (_I, [_P, _P, snb_boundary, _P, _I, _P, _I, _P, _P]),
    "snb_bond_energy": (_I, [_P, ctypes.POINTER(ctypes.c_float), _P]),
    "snb_bond_destroy": (_I, [_P]),
    "snb_angle_create": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "snb_angle_force": (_I, [_P, _P, snb_boundary, _P, _I, _P, _I, _P, _P]),
    "snb_angle_energy": (_I, [_P, ctypes.POINTER(ctypes.c_float), _P]),
    "snb_angle_destroy": (_I, [_P]),
    "snb_read_bond_in_file": (_I, [ctypes.c_char_p, ctypes.POINTER(_I), _P, _P, _P, _P]),
    "snb_read_virtual_atom_in_file": (_I, [ctypes.c_char_p, ctypes.POINTER(_I), _P, _P, _P,
                                           _P]),
    "snb_vatom_create": (_I, [_I, _I, _P, _P, _P, _P, _P]),
    "snb_vatom_levels": (_I, [_P, ctypes.POINTER(_I)]),
    "snb_vatom_coordinate_refresh": (_I, [_P, _P, snb_boundary, _P]),
    "snb_vatom_force_redistribute": (_I, [_P, _P, snb_boundary, _P, _P]),
    "snb_vatom_status": (_I, [_P, ctypes.POINTER(_I), _P]),
    "snb_vatom_destroy": (_I, [_P]),
    "snb_engine_set_virtual_atoms": (_I, [_P, _P]),
    "snb_read_angle_in_file": (_I, [ctypes.c_char_p, ctypes.POINTER(_I), _P, _P, _P, _P,
                                    _P]),
    "snb_engine_list_form": (_I, [_P, ctypes.POINTER(ctypes.c_int)]),
    "snb_engine_export_pairs": (_I, [_P, _P, _P, _LL, ctypes.POINTER(_LL), _P]),
    "snb_engine_destroy": (_I, [_P]),
}


def load(path: str = LIB_PATH):
    """Load the CUDA library (once).  Raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SnbError(
            f"{path} is missing: build it with `python -m sponge_b200.build`; "
            "this package has no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = load().snb_last_error()
        raise SnbError(f"{what} failed with status {rc}: "
                       f"{msg.decode() if msg else ''}")


def boundary(cell6, rcell6) -> snb_boundary:
    b = snb_boundary()
    b.policy = 1
    for k in range(6):
        b.cell[k] = float(cell6[k])
        b.rcell[k] = float(rcell6[k])
    return b


def options(**kv) -> snb_options:
    lib = load()
    o = snb_options()
    lib.snb_options_default(ctypes.byref(o))
    for k, v in kv.items():
        check(lib.snb_options_set(ctypes.byref(o), k.encode(), str(v).encode()),
              f"options_set({k})")
    return o
