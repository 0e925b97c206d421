import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cf():
    """The product package (chanflow_b200)."""
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure)."""
    import orc as _orc
    _orc.lib()
    return _orc


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


import contextlib  # noqa: E402


@contextlib.contextmanager
def whole_velocity_transforms(on=True):
    """Contexts created inside keep the whole velocity (mean included) in the
    FP32 transforms, as multi-rank runs do, instead of the single-context
    mean split (CHANFLOW_NO_MEAN_SPLIT is read at cfg_create)."""
    old = os.environ.get("CHANFLOW_NO_MEAN_SPLIT")
    if on:
        os.environ["CHANFLOW_NO_MEAN_SPLIT"] = "1"
    try:
        yield
    finally:
        if old is None:
            os.environ.pop("CHANFLOW_NO_MEAN_SPLIT", None)
        else:
            os.environ["CHANFLOW_NO_MEAN_SPLIT"] = old
