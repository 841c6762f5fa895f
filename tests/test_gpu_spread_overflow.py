"""The PME spread's int32 fixed-point tile sums and their guard.

The spread sums each grid point's charge in int32 at 2^22 units per
(18.2223-scaled) charge unit, which holds |Q| < 512 at a point.  Each tile
keeps, per 4x4x4 octant, a bound on its points' sums (the atoms' |q| times the
largest weight product (2/3)^3); a liquid stays far below the range (the
100k water box's largest octant bound is about 0.4 of it).  A host-built
cluster of highly charged sites goes beyond it: twelve sites of +30 e within
half an Angstrom put about 12 x 547 x 0.3 ~ 2,000 units on the points at the
cluster's centre.  Such tiles are taken again with int64 sums, so the
reciprocal forces and energy stay within the usual FP64 tolerances, and they
are counted.  The plain 216-water box takes no tile again.
"""

import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


def _clustered(small_box):
    from sponge_b200 import systems
    s = copy.deepcopy(small_box)
    rng = np.random.default_rng(7)
    pos_sites = np.arange(0, 36, 3)        # twelve water O atoms
    neg_sites = np.arange(300, 336, 3)     # twelve others
    c1 = np.full(3, 0.3 * s.box, np.float32)
    c2 = np.full(3, 0.75 * s.box, np.float32)
    s.crd[pos_sites] = c1 + rng.uniform(-0.25, 0.25, (12, 3)).astype(np.float32)
    s.crd[neg_sites] = c2 + rng.uniform(-0.25, 0.25, (12, 3)).astype(np.float32)
    s.charge[pos_sites] = np.float32(30.0) * systems.CHARGE_SCALE
    s.charge[neg_sites] = np.float32(-30.0) * systems.CHARGE_SCALE
    return s


def _wide(g, h):
    import ctypes
    c = ctypes.c_int(-1)
    g.capi.check(g.capi.load().snb_pme_spread_wide_tiles(h, ctypes.byref(c), g.stream()),
                 "pme_spread_wide_tiles")
    return c.value


def test_dense_charge_cluster_is_summed_exactly(g, oracle, small_box):
    s = _clustered(small_box)
    box = g.Box(s)
    h, beta, grid = g.pme_create(box, 8.0)
    try:
        got = g.pme_reciprocal(h, box)
        wide = _wide(g, h)
    finally:
        g.capi.load().snb_pme_destroy(h)
    want = oracle.pme_f64(s, grid, beta)
    assert wide > 0
    assert g.rel_rms(got["frc"], want["frc"]) <= 1e-5
    assert abs(got["e_recip"] - want["e_recip"]) <= 2e-6 * abs(want["e_recip"])


def test_liquid_takes_no_tile_again(g, oracle, small_box):
    box = g.Box(small_box)
    h, beta, grid = g.pme_create(box, 8.0)
    try:
        got = g.pme_reciprocal(h, box)
        wide = _wide(g, h)
    finally:
        g.capi.load().snb_pme_destroy(h)
    assert wide == 0
    want = oracle.pme_f64(small_box, grid, beta)
    assert g.rel_rms(got["frc"], want["frc"]) <= 1e-5
