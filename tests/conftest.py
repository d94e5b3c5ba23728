import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def kernels():
    """The CUDA library; GPU tests fail (not skip) when it is missing."""
    import cuda_pf_localization_b200 as pkg
    lib = pkg.kernels()
    assert lib.pfc_device_available() == 1, "no CUDA device visible to libpf_kernels.so"
    return lib


@pytest.fixture(scope="session")
def ref():
    """The reference library built from its own source (oracle/_ref)."""
    import oracle
    r = oracle.ref_lib()
    if r is None:
        pytest.skip("oracle/_ref/libpf_kernels_ref.so not built")
    return r
