import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


# The CTMRG path's parity and kernel tests run first; the rows built on top of
# it (front end, gradients, full update, long-range correlations) follow, so
# that a stop at the first failure (-x) still reports on the path itself.
_LATE_FILES = ("test_gpu_frontend.py", "test_gpu_grad.py", "test_gpu_full_update.py", "test_gpu_local_gauge.py",
               "test_gpu_configs.py")


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        name = os.path.basename(str(item.fspath))
        if name in _LATE_FILES:
            return 1 + _LATE_FILES.index(name)
        if item.name.startswith("test_correlation_strip"):
            return len(_LATE_FILES)
        if name == "test_zz_no_alloc.py":
            return 2 + len(_LATE_FILES)
        return 0
    items.sort(key=rank)  # stable: file and definition order within a rank
