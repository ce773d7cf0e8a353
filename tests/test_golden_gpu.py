"""The B200 path against the committed golden fixtures (tests/golden/*.npz: outputs of
the reference's own functions, see tests/golden/make_golden.py).  These tests need no
reference build on the GPU machine."""
import numpy as np
import pytest

import vfs_b200 as vfs
from golden_cases import FIXTURES, load

NAMES = list(FIXTURES)


def _ctx(name):
    case, d = load(name)
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    ctx.set_field(vfs.UCONT, d["ucont"])
    ctx.set_field(vfs.UCAT, d["ucat"])
    ctx.set_field(vfs.UCAT_O, d["ucat"])
    ctx.set_field(vfs.P, d["p"])
    return case, d, ctx


@pytest.mark.gpu
def test_form_metrics_bitwise():
    case, d, ctx = _ctx("wavy_channel_12x10x14")
    for name, fid in vfs.METRIC_FIELDS.items():
        np.testing.assert_array_equal(ctx.get_field(fid), d["metric_" + name], err_msg=name)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_contra2cart_formfunction2_bitwise(name):
    case, d, ctx = _ctx(name)
    ctx.contra2cart()
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), d["ucat_c2c"])
    ctx.set_field(vfs.RHS, d["rhs0"])
    ctx.formfunction2(0.75)
    np.testing.assert_array_equal(ctx.get_field(vfs.RHS), d["rhs_ff2"])
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_pressure_gradient_bitwise(name):
    case, d, ctx = _ctx(name)
    ctx.set_scalar(vfs.S_MEAN_K_FLUX, 0.37)
    ctx.set_scalar(vfs.S_MEAN_K_AREA, 1.9)
    ctx.set_scalar(vfs.S_INLET_FLUX, 0.25)
    ctx.pressure_gradient()
    np.testing.assert_array_equal(ctx.get_field(vfs.DP), d["dp"])
    np.testing.assert_array_equal(ctx.get_field(vfs.P), d["p_pg"])
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_poisson_operator_and_rhs(name):
    case, d, ctx = _ctx(name)
    ctx.poisson_lhs()
    ax = ctx.poisson_apply(d["x"])
    assert np.abs(ax - d["ax"]).max() <= 1e-14 * np.abs(d["ax"]).max()
    ctx.poisson_rhs()
    b = ctx.get_field(vfs.B)
    assert np.abs(b - d["b"]).max() <= 1e-12 * np.abs(d["b"]).max()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_update_pressure_projection_bitwise(name):
    case, d, ctx = _ctx(name)
    ctx.poisson_lhs()
    ctx.set_field(vfs.P, d["p_before_up"])
    ctx.set_field(vfs.UCONT, d["ucont_before_proj"])
    ctx.set_field(vfs.UCAT, d["ucat_before_proj"])
    ctx.set_field(vfs.PHI, d["phi"])
    ctx.update_pressure()
    np.testing.assert_array_equal(ctx.get_field(vfs.P), d["p_up"])
    ctx.projection()
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), d["ucont_proj"])
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), d["ucat_proj"])
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_dynamic_smagorinsky(name):
    """Cs and nu_t of the dynamic model at ti = 5 (les.c:67, les.c:1135).  pow() is CUDA's
    on the device and the host libm's in the fixture, so the comparison allows 1e-12 of
    the largest value; zeros (solid cells, boundaries, clipping) must coincide."""
    case, d = load(name)
    case.les = 2
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    ctx.set_field(vfs.UCONT, d["ucont"])
    ctx.set_field(vfs.UCAT, d["ucat"])
    ctx.set_field(vfs.UCAT_O, d["ucat"])
    ctx.set_field(vfs.NU_T, d["nut0"])
    ctx.set_scalar(vfs.S_TI, 5)
    ctx.contra2cart()
    ctx.smagorinsky_constant()
    ctx.eddy_viscosity()
    cs = ctx.get_field(vfs.CS)
    assert np.abs(cs - d["cs_les"]).max() <= 1e-12 * np.abs(d["cs_les"]).max()
    np.testing.assert_array_equal(cs == 0.0, d["cs_les"] == 0.0)
    nut = ctx.get_field(vfs.NU_T)
    assert np.abs(nut - d["nut_les"]).max() <= 1e-12 * np.abs(d["nut_les"]).max()
    ctx.close()
