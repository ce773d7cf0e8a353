"""nvert classification of closed triangulated bodies (ibm_search_advanced, ibm.c:85) on the
B200 against the reference's own ray test (point_cell_advanced, ibm.c:1068, driven by
oracle/_ref) and the committed fixture: integer flags, compared bit for bit, at the
wavy-channel test size, at 64^3 and at 128x96x128 with a 20480-triangle sphere (the
curvilinear sphere configuration), and for two bodies in a row."""
import os

import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from vfs_b200 import cases

HERE = os.path.dirname(os.path.abspath(__file__))


def _ctx(case):
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, np.zeros(case.da_shape))
    return ctx


@pytest.mark.gpu
def test_ibm_search_matches_fixture():
    d = np.load(os.path.join(HERE, "golden", "ibm_sphere_wavy_24x20x28.npz"))
    case = cases.channel(24, 20, 28, wavy=0.1)
    np.testing.assert_array_equal(case.X, d["X"])
    np.testing.assert_array_equal(case.Y, d["Y"])
    ctx = _ctx(case)
    got = ctx.ibm_search(d["sx"], d["sy"], d["sz"], d["tri"])
    np.testing.assert_array_equal(got, d["nvert"])
    assert (got == 3).sum() > 0 and (got == 1).sum() > 0
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("size,level", [((24, 20, 28), 3), ((64, 64, 64), 4), ((128, 96, 128), 5)])
def test_ibm_search_matches_reference(size, level):
    nx, ny, nz = size
    case = cases.channel(nx, ny, nz, wavy=0.1)
    case.immersed = 1
    x, y, z, tri = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.2 if level == 5 else 0.4, level=level)
    R = ref.Reference(case)
    want = R.ibm_classify(x, y, z, tri)
    R.close()
    ctx = _ctx(case)
    got = ctx.ibm_search(x, y, z, tri)
    np.testing.assert_array_equal(got, want)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_ibm_search_two_bodies():
    """Body 1 after body 0: earlier flags are kept and the new body's added."""
    case = cases.channel(40, 32, 48, wavy=0.1)
    case.immersed = 1
    a = cases.icosphere((np.pi / 2 - 0.5, 0.9, np.pi - 1.0), 0.35, level=3)
    b = cases.icosphere((np.pi / 2 + 0.4, 1.1, np.pi + 1.0), 0.3, level=3)
    R = ref.Reference(case)
    R.ibm_classify(*a, ibi=0)
    want = R.ibm_classify(*b, ibi=1)
    R.close()
    ctx = _ctx(case)
    ctx.ibm_search(*a, ibi=0)
    got = ctx.ibm_search(*b, ibi=1)
    np.testing.assert_array_equal(got, want)
    assert (got == 3).sum() > 0
    ctx.close()
