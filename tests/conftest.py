"""Shared test setup: the `gpu` marker, builds of the CUDA library and the CPU oracles."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle (and, where the reference tree exists, its reference build) and the
    CUDA library in-tree if they are missing; both builds are incremental."""
    import oracle.pyoracle as po
    from mikroptim_b200 import build as mbuild

    if not os.path.exists(po.PORT_LIB) or (
            os.path.isdir(os.path.join(po.REFERENCE_TREE, "src")) and not os.path.exists(po.REF_LIB)):
        po.build()
    if not os.path.exists(mbuild.LIB):
        mbuild.build()
    yield


def has_reference_build() -> bool:
    import oracle.pyoracle as po
    return os.path.exists(po.REF_LIB)


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
