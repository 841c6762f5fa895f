import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def small_box():
    """216 waters (648 atoms), L = 18.63 A, grid 20^3: the golden-vector box."""
    from sponge_b200 import systems
    return systems.water_box(216, seed=1)


@pytest.fixture(scope="session")
def box_9k():
    """3,000 waters (9,000 atoms), L = 44.77 A, grid 48^3."""
    from sponge_b200 import systems
    return systems.config_small(seed=0)
