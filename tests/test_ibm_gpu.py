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


def _immersed_pair(size=(24, 20, 28), level=3, radius=0.4, seed=0):
    """The wavy channel with an icosphere body on both sides: the reference classified and
    listed it with its own nearestcell1/InterceptionPoint, the B200 library with its own."""
    from helpers import build_pair
    nx, ny, nz = size
    case = cases.channel(nx, ny, nz, wavy=0.1)
    case.immersed = 1
    body = cases.icosphere((np.pi / 2, 1.0, np.pi), radius, level=level)
    R, ctx = build_pair(case, seed=seed)
    R.ibm_classify(*body, build_list=True)
    ctx.ibm_search(*body)
    return case, R, ctx


def _by_cell(ints, dbls):
    order = np.lexsort((ints[:, 0], ints[:, 1], ints[:, 2]))
    return ints[order], dbls[order]


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("size,level,radius", [((24, 20, 28), 3, 0.4), ((48, 40, 56), 4, 0.35)])
def test_ibm_list_matches_reference(size, level, radius):
    """The IB-node list node by node: nearest triangle, interception mode and stencil cells
    bit for bit; the weights and distances to 1e-12 relative."""
    case, R, ctx = _immersed_pair(size, level, radius)
    wi, wd = _by_cell(*R.ibm_list())
    gi, gd = _by_cell(*ctx.ibm_list())
    R.close()
    assert len(wi) > 50 and len(gi) == len(wi)
    np.testing.assert_array_equal(gi[:, :3], wi[:, :3])
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_allclose(gd, wd, rtol=1e-12, atol=1e-14)
    assert (gi[:, 4] >= 0).all() and ctx.get_scalar(vfs.S_IB_UNRESOLVED) == 0
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_ibm_interpolation_matches_reference():
    """ibm_interpolation_advanced (ibm.c:3294) on the seeded state: IB-node Ucat and P,
    the face fluxes around the nodes and the Cartesian velocity after Contra2Cart."""
    from helpers import assert_close
    case, R, ctx = _immersed_pair()
    u0 = ctx.get_field(vfs.UCAT)
    R.call("ref_ibm_interpolation", 1)
    ctx.ibm_interpolation()
    nv = ctx.get_field(vfs.NVERT)
    assert ((nv == 1) & (np.abs(ctx.get_field(vfs.UCAT) - u0).max(axis=-1) > 0)).sum() > 0
    # the device keeps one copy of each field; the reference's ghosted local copy (lUcont)
    # is the one its later operators read
    np.testing.assert_array_equal(ctx.get_field(vfs.P), R.get("P"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), R.get("lUcont"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), R.get("Ucat"))
    R.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_volume_flux_ibm_matches_reference():
    """VolumeFlux(user, &flux, &area, 0) (poisson.c:3570) after the interpolation: the
    net flux into the IB nodes spread over the fluid/IB faces."""
    from helpers import assert_close
    case, R, ctx = _immersed_pair()
    R.call("ref_ibm_interpolation", 1)
    ctx.ibm_interpolation()
    # a perturbed Ucont, so that a net flux into the IB nodes remains to be corrected
    rng = np.random.Generator(np.random.Philox(11))
    uc = R.get("lUcont") + 0.01 * rng.standard_normal(R.shape + (3,))
    R.set("Ucont", uc)
    R.set("lUcont", uc)
    ctx.set_field(vfs.UCONT, uc)
    flux, area = R.volume_flux_ibm()   # the net flux recounted after the correction
    ctx.volume_flux()
    assert abs(flux) < 1e-12
    assert np.abs(ctx.get_field(vfs.UCONT) - uc).max() > 1e-6
    assert_close(ctx.get_field(vfs.UCONT), R.get("Ucont"), rtol=1e-13, atol_frac=1e-15, what="Ucont")
    R.close()
    ctx.close()
