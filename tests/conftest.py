import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU or GPU cases")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    from oracle.build import build
    build()
    return oracle.lib()


@pytest.fixture(scope="session")
def native_lib():
    from polyswift_plusplus_b200 import _abi
    if not _abi.LIB_PATH.exists():
        from polyswift_plusplus_b200 import build_native
        build_native.build()
    return _abi.load_library()


@pytest.fixture(scope="session")
def gpu(native_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return native_lib
