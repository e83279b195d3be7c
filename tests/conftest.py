import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a) and the built native library')


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def pytest_collection_modifyitems(config, items):
    # a test that loops on the host without end fails after 5 minutes instead of holding the run (pytest-timeout)
    if config.pluginmanager.hasplugin('timeout'):
        for item in items:
            if item.get_closest_marker('timeout') is None:
                item.add_marker(pytest.mark.timeout(300))
    if gpu_available():
        return
    skip = pytest.mark.skip(reason='no CUDA device in this environment')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, f'{name}.npz'))
