import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    """The plain-C restatement of the reference path (oracle/gt_oracle.c)."""
    from oracle import Restatement

    return Restatement()


@pytest.fixture(scope="session")
def reference():
    """The reference's own shmem tree compiled from its sources (oracle/_ref); skipped if absent."""
    from oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("oracle/_ref not built (reference sources unavailable)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    path = os.path.join(ROOT, "tests", "golden", "golden.npz")
    return dict(np.load(path, allow_pickle=False))


@pytest.fixture(scope="session")
def gpu_ctx():
    import gizmo_shared_memory_b200 as g

    return g.Context(0)
