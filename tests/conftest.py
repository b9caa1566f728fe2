"""Shared pytest setup: the ``gpu`` marker, the package loader and fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from __graft_entry__ import load_package  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "late: run after the other tests (GPU paths not yet run on a GPU), so "
                                       "that under -x a failure there cannot stop the established tests")
    # raised inside torch.func's linear-algebra rules, not by this package
    config.addinivalue_line("filterwarnings", "ignore:`torch.jit.script` is deprecated:DeprecationWarning")


def pytest_collection_modifyitems(session, config, items):
    """Tests marked ``late`` go last, in their collected order."""
    items[:] = ([it for it in items if it.get_closest_marker("late") is None]
                + [it for it in items if it.get_closest_marker("late") is not None])


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def cuda(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg._native.load()
    return torch.device("cuda", 0)

