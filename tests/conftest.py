import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from oracle.build_ref import reference_dir  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line('markers',
                            'gpu: needs a CUDA GPU and the built library')


@pytest.fixture(scope='session')
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


@pytest.fixture(scope='session')
def built_lib():
    from py_stoch_b200 import build
    build.build()
    from py_stoch_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope='session')
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


def reference_available():
    from oracle.build_ref import reference_present
    return reference_present()
