import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libvoxrt.so")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle
    return pyoracle.load()


@pytest.fixture(scope="session")
def c1_oracle_world():
    """The c1 benchmark world generated by the oracle (CPU)."""
    from oracle import pyoracle
    from voxelg_b200.configs import CONFIGS
    cfg = CONFIGS["c1"]
    w = pyoracle.World(*cfg.bricks)
    w.generate(cfg.terrain)
    return w
