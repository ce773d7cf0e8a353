"""The C-ABI library loads on a machine without a GPU, exports every entry point that
include/vfs_b200.h declares, and refuses to run without a B200 instead of falling back."""
import ctypes
import os
import re

import pytest

import vfs_b200 as vfs
from conftest import ROOT


def _declared():
    with open(os.path.join(ROOT, "include", "vfs_b200.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|long long)\s*\*?\s*(vfs_\w+)\s*\(", src, re.M)))


def test_header_lists_entry_points():
    names = _declared()
    assert "vfs_formfunction2" in names and "vfs_poisson_solve" in names and "vfs_step" in names
    assert set(vfs.EXPORTS) <= set(names)


def test_library_exports_all_declared_symbols():
    lib = vfs.load_library()
    for n in _declared():
        assert hasattr(lib, n), n


def test_create_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    lib = vfs.load_library()
    cfg = vfs.make_config(9, 9, 9, [7, 7, 1, 1, 7, 7], 1, 0, 1)
    h = ctypes.c_void_p()
    rc = lib.vfs_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert rc == vfs.ERR_NO_DEVICE
    assert b"no CUDA device" in lib.vfs_last_error(None)


def test_bad_config_is_rejected_before_device_use():
    lib = vfs.load_library()
    cfg = vfs.make_config(2, 9, 9, [7, 7, 1, 1, 7, 7], 1, 0, 1)
    h = ctypes.c_void_p()
    rc = lib.vfs_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert rc in (vfs.ERR_INVALID, vfs.ERR_NO_DEVICE)
