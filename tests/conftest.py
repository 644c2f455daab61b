"""Test configuration.

* ``gpu``-marked tests run the sm_100a kernels through the C ABI and
  compare them with the oracle (the reference's own C core built under
  oracle/_ref, or its numpy restatement oracle/port.py where that library
  is absent).
* Everything else runs on the CPU: the oracle against the golden vectors,
  host-side logic, the C-ABI symbol table, multi-process (gloo) paths.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers',
                            'gpu: needs a CUDA device (B200, sm_100a)')


@pytest.fixture(scope='session')
def golden():
    path = os.path.join(ROOT, 'tests', 'golden', 'golden.npz')
    with np.load(path) as z:
        data = {k: z[k] for k in z.files}
    cases = {}
    for key, v in data.items():
        name, field = key.split('/')
        cases.setdefault(name, {})[field] = v
    return cases


@pytest.fixture(scope='session')
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from gpaw_b200 import _lib
    _lib.load()
    return torch.device('cuda:0')
