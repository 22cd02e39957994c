import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the device library")


@pytest.fixture(scope="session")
def ref_bin():
    """The reference's own code, compiled by oracle/Makefile (skip if absent)."""
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/pk_ref not built")
    return oracle.REF_BIN


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a GPU")
    return torch.device("cuda:0")
