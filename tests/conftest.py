"""Shared fixtures. GPU tests carry @pytest.mark.gpu and call the sm_100a library through its C ABI;
everything else runs on the CPU (oracle, scene generation, host logic, library symbol checks)."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libdfsph_b200.so")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    return oracle.build()


@pytest.fixture(scope="session")
def cuda_lib():
    from splishsplash_for_cuda_b200 import _capi
    from splishsplash_for_cuda_b200.build import build

    build()
    return _capi.load()
