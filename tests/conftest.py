"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "arbor-cuda_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and runs the CUDA library")


@pytest.fixture(scope="session")
def oracle():
    from pyoracle import Oracle

    return Oracle("port")


@pytest.fixture(scope="session")
def oracle64():
    from pyoracle import Oracle

    return Oracle("port64")


@pytest.fixture(scope="session")
def ref():
    from pyoracle import Oracle, available

    if not available("reference"):
        pytest.skip("reference harness build (oracle/_ref) not available here")
    return Oracle("reference")


@pytest.fixture(scope="session")
def scenes(oracle):
    cache = {}

    def get(seed):
        if seed not in cache:
            cache[seed] = oracle.build_scene(seed)
        return cache[seed]

    return get


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import arbor_b200

    lib = arbor_b200.lib()
    assert lib.arbor_device_ready() == 1, "library loaded but device not sm_100"
    return arbor_b200


def u32(a):
    return np.ascontiguousarray(a).view(np.uint32)
