"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build()
    return Oracle()


@pytest.fixture(scope="session")
def k2lib():
    """The CUDA library, built in-tree (nvcc cross-compiles without a GPU)."""
    from mertens_bound_b200 import build, _lib
    build.build_library()
    return _lib.lib()


@pytest.fixture(scope="session")
def gpu(k2lib):
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session")
def small_table():
    from mertens_bound_b200 import synth
    return synth.make_table(10_000, seed=1)


@pytest.fixture(scope="session")
def small_cands():
    from mertens_bound_b200 import synth
    return synth.make_candidates(64, seed=2)
