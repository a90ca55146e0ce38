"""Shared pytest configuration: the `gpu` marker and access to the oracle libraries.

GPU tests (`-m gpu`) need a CUDA device and the in-tree CUDA library; everything else runs on CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the in-tree CUDA library")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    return oracle_lib.port()


@pytest.fixture(scope="session")
def reference():
    import oracle_lib
    ref = oracle_lib.reference()
    if ref is None:
        pytest.skip("oracle/_ref/libzapref.so not built (the reference tree is not present here)")
    return ref


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    path = os.path.join(TESTS, "golden", "golden_tex.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_containers():
    """Files the reference CLI's `zap tex` wrote (tests/golden/make_containers.py): key -> (image, args, bytes)."""
    import numpy as np
    path = os.path.join(TESTS, "golden", "golden_containers.npz")
    with np.load(path) as z:
        return {k[5:]: (z["img/" + str(z["image/" + k[5:]])], tuple(z["args/" + k[5:]]), z[k])
                for k in z.files if k.startswith("file/")}


@pytest.fixture(scope="session")
def cuda_lib():
    """The product library on a real device; GPU tests only."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zap_b200
    return zap_b200
