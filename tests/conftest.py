import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def reference_module():
    """The compiled reference CPU module (oracle/_ref), or None."""
    if not any(f.startswith("radia") and f.endswith(".so") for f in os.listdir(REF_DIR)) if os.path.isdir(REF_DIR) else True:
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import radia  # noqa: WPS433
    return radia


@pytest.fixture(scope="session")
def ref():
    m = reference_module()
    if m is None:
        pytest.skip("compiled reference module (oracle/_ref) not present")
    return m


@pytest.fixture(scope="session")
def rad():
    from radiacuda_b200 import rad as R
    return R


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
