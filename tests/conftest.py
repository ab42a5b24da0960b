"""Shared fixtures.  `-m gpu` tests need a CUDA device and libdgann.so; the
rest run on CPU (the oracle, host-side logic and the C-ABI symbol table)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdgann.so")
    config.addinivalue_line("markers", "slow: larger CPU oracle cases")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        have_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def small_data():
    """Integer-valued Gaussian-mixture data: every FP32 distance is exact."""
    from pydiskann_b200 import synth

    X = synth.mixture(4000, 128, 32, seed=7, stream=synth.STREAM_BASE)
    Q = synth.mixture(200, 128, 32, seed=7, stream=synth.STREAM_QUERY)
    return X, Q


@pytest.fixture(scope="session")
def small_graph(oracle, small_data):
    X, _ = small_data
    adj, med = oracle.build_vamana(X, R=32, L_build=64, alpha=1.2, seed=11)
    return adj, med
