import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda_block_factory():
    """Builds chimera Blocks; fails loudly (no CPU fallback) when CUDA is absent."""
    from chimera_comp_les_b200 import Block
    return Block
