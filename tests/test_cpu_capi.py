"""The C ABI library: it loads without a GPU, exports every entry point that
include/sponge_nb.h declares, and its option parser accepts the reference's
input keys (no compute calls here)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sponge_nb.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(snb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from sponge_b200 import build, capi
    if not os.path.exists(capi.LIB_PATH):
        build.build()
    return capi.load()


def test_header_declares_the_module_entry_points():
    syms = declared_symbols()
    for must in ("snb_nl_create", "snb_nl_update", "snb_lj_pme_direct_force",
                 "snb_lj_soft_pme_direct_force", "snb_pme_reciprocal_force",
                 "snb_pme_excluded_force", "snb_engine_force"):
        assert must in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from sponge_b200 import capi
    assert sorted(capi.EXPORTED) == declared_symbols()


def test_options_accept_reference_keys(lib):
    from sponge_b200 import capi
    o = capi.options(cutoff=8, skin=1.5, neighbor_list_refresh_interval=10,
                     neighbor_list_skin_permit=0.25,
                     neighbor_list_max_neighbor_numbers=800,
                     neighbor_list_max_atom_in_grid_numbers=64,
                     neighbor_list_check_overflow_interval=50,
                     neighbor_list_throw_error_when_overflow="true",
                     PM_fftx=64, PM_ffty=48, PM_fftz=40, PM_grid_spacing=0.9,
                     PM_Direct_Tolerance=1e-6, PME_update_interval=2,
                     PME_calculate_reciprocal_part=0, PME_calculate_excluded_part=1,
                     lambda_lj=0.25, soft_core_alpha=0.5, soft_core_powfer=1,
                     soft_core_sigma=3.5, soft_core_sigma_min=2.0,
                     accumulation="float")
    assert o.cutoff == 8.0 and o.skin == 1.5
    assert o.nl_refresh_interval == 10 and o.nl_skin_permit == 0.25
    assert o.nl_max_neighbor_numbers == 800 and o.nl_throw_error_when_overflow == 1
    assert (o.pm_fftx, o.pm_ffty, o.pm_fftz) == (64, 48, 40)
    assert o.pme_update_interval == 2 and o.pme_calculate_reciprocal_part == 0
    assert o.lambda_lj == 0.25 and o.soft_core_sigma == 3.5
    assert o.accumulation == 1


def test_options_defaults_are_the_reference_defaults(lib):
    from sponge_b200 import capi
    o = capi.options()
    assert o.cutoff == 10.0 and o.skin == 2.0          # MD_core/nb.hpp:14-27
    assert o.nl_skin_permit == 0.5                      # neighbor_list.cpp:286
    assert o.nl_max_neighbor_numbers == 1200            # neighbor_list.cpp:894
    assert o.nl_check_overflow_interval == 150          # neighbor_list.cpp:916
    assert (o.pm_fftx, o.pm_ffty, o.pm_fftz) == (-1, -1, -1)
    assert o.pm_grid_spacing == 1.0                     # PM_force.cpp:379
    assert abs(o.pm_direct_tolerance - 1e-5) < 1e-12   # PM_force.cpp:316
    assert o.pme_update_interval == 1                   # PM_force.cpp:405
    assert o.soft_core_alpha == 0.5 and o.soft_core_powfer == 1.0  # LJ_soft_core.cpp
    assert o.soft_core_sigma == 3.0 and o.soft_core_sigma_min == 0.0
    assert o.accumulation == 0


def test_unknown_key_is_an_error(lib):
    from sponge_b200 import capi
    o = capi.snb_options()
    lib.snb_options_default(ctypes.byref(o))
    rc = lib.snb_options_set(ctypes.byref(o), b"no_such_key", b"1")
    assert rc == 1
    assert b"no_such_key" in lib.snb_last_error()


def test_null_handles_are_rejected_without_a_gpu(lib):
    from sponge_b200 import capi
    b = capi.snb_boundary()
    assert lib.snb_nl_update(None, None, 1, 0, None, b, 0, 1, None, None, None,
                             None) == 1
    assert lib.snb_engine_force(None, None, None, 0, 0, 0, None, None) == 1
    assert lib.snb_version() == 1


def test_product_path_has_no_oracle_dependency():
    """Nothing under sponge_b200/ imports or links the oracle."""
    pkg = os.path.join(ROOT, "sponge_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                text = open(os.path.join(dirpath, f), errors="ignore").read()
                assert "oracle" not in text.lower(), f
