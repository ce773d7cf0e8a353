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


def test_struct_layouts_match_the_header(tmp_path):
    """Every public struct of include/vfs_b200.h has the size and field offsets the ctypes
    mirror uses (compiled with the host C compiler: the structs hold no CUDA types)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    mirrors = {"vfs_config": vfs.VfsConfig, "vfs_solve_opts": vfs.SolveOpts, "vfs_solve_stats": vfs.SolveStats,
               "vfs_step_stats": vfs.StepStats, "vfs_adjoint_opts": vfs.AdjointOpts,
               "vfs_adjoint_stats": vfs.AdjointStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vfs_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append('  printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, fname, val = line.split()
        got[(cname, fname)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
