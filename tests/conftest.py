import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vfs-geophysics-3.1_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def pytest_sessionfinish(session, exitstatus):
    """With VFS_PARITY_REPORT set, write the achieved errors that the parity tests
    recorded (helpers.report) to that file as JSON."""
    path = os.environ.get("VFS_PARITY_REPORT")
    if not path:
        return
    import json
    from helpers import REPORT
    with open(path, "w") as f:
        json.dump(REPORT, f, indent=1, sort_keys=True)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
