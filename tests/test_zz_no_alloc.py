"""vfs_contra2cart_noalloc, the allocation-free Contra2Cart for callers that cannot
allocate device memory, against the context entry point vfs_contra2cart on the same
inputs, on two calls in a row.  Both run the same kernels, so the results must be equal
bit for bit (the tolerance of the Contra2Cart parity tests).  The buffers handed to the
allocation-free call are owned by the test (torch), as they would be by such a caller."""
import ctypes

import numpy as np
import pytest

import vfs_b200 as vfs
from vfs_b200 import cases


def _soa(a):
    """(mz, my, mx, 3) host array -> three consecutive component blocks."""
    return np.ascontiguousarray(np.moveaxis(a, -1, 0))


def _cases():
    c1 = cases.channel(12, 10, 14, wavy=0.15)
    c2 = cases.open_channel_cylinders(16, 12, 24, D=0.6)
    return [c1, c2]


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1])
def test_noalloc_contra2cart_matches_context_path(which):
    import torch
    case = _cases()[which]
    lib = vfs.load_library()
    lib.vfs_contra2cart_noalloc.argtypes = [ctypes.POINTER(vfs.VfsConfig)] + [ctypes.c_void_p] * 8
    cfg = case.config()
    ctx = vfs.Context(cfg)
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    m = {k: ctx.get_field(f) for k, f in vfs.METRIC_FIELDS.items()}
    dev = torch.device("cuda", 0)
    d_csi = torch.from_numpy(_soa(m["csi"])).to(dev)
    d_eta = torch.from_numpy(_soa(m["eta"])).to(dev)
    d_zet = torch.from_numpy(_soa(m["zet"])).to(dev)
    d_nv = torch.from_numpy(np.ascontiguousarray(case.nvert, dtype=np.float64)).to(dev)
    for seed in (0, 1):   # two calls in a row on different inputs
        u = cases.initial_ucat(case, seed=seed)
        uc = cases.ucont_from_ucat(case, u, m)
        uo = cases.initial_ucat(case, seed=seed + 10)
        ctx.set_field(vfs.UCONT, uc)
        ctx.set_field(vfs.UCAT, u)
        ctx.set_field(vfs.UCAT_O, uo)
        ctx.contra2cart()
        want_u = ctx.get_field(vfs.UCAT)
        want_uc = ctx.get_field(vfs.UCONT)
        d_uc = torch.from_numpy(_soa(uc)).to(dev)
        d_u = torch.from_numpy(_soa(u)).to(dev)
        d_uo = torch.from_numpy(_soa(uo)).to(dev)
        for t in (d_uc, d_csi, d_eta, d_zet, d_nv, d_uo, d_u):
            assert t.dtype == torch.float64 and t.is_contiguous()
        torch.cuda.synchronize()
        rc = lib.vfs_contra2cart_noalloc(ctypes.byref(cfg), d_uc.data_ptr(), d_csi.data_ptr(), d_eta.data_ptr(),
                                         d_zet.data_ptr(), d_nv.data_ptr(), d_uo.data_ptr(), d_u.data_ptr(), None)
        assert rc == 0, lib.vfs_last_error(None)
        got_u = np.moveaxis(d_u.cpu().numpy(), 0, -1)
        got_uc = np.moveaxis(d_uc.cpu().numpy(), 0, -1)
        np.testing.assert_array_equal(got_u, want_u)
        np.testing.assert_array_equal(got_uc, want_uc)
    ctx.close()


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = vfs.load_library()
    lib.vfs_contra2cart_noalloc.argtypes = [ctypes.POINTER(vfs.VfsConfig)] + [ctypes.c_void_p] * 8
    cfg = vfs.make_config(200, 200, 200, [7, 7, 1, 1, 7, 7], 1, 0, 1)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.vfs_contra2cart_noalloc(ctypes.byref(cfg), dummy, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == vfs.ERR_INVALID
    assert b"exceeds" in lib.vfs_last_error(None)
