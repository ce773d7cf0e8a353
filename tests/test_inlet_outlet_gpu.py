"""Inlet and outlet faces on the B200 against the reference's own InflowFlux (bcs.c:329)
and FormBCS outlet rescaling (bcs.c:2285-2417), then whole steps with an inlet on the
k = 0 face and an outlet on the k+ face: the open channel with the cylinder array and the
channel with the Poiseuille inflow.

Face values set pointwise are compared bit for bit; the inlet and outlet flux sums are
reductions whose summation order differs from the reference's loops, so they and every
face value they rescale are compared to 1e-13 relative."""
import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from vfs_b200 import cases
from helpers import assert_close, build_pair, small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _case(name):
    if name == "cylinders100":
        c = cases.inflow_outflow(small_cylinders(), 100)
        c.immersed = 0
    elif name in ("cylinders1", "cylinders2"):
        c = cases.inflow_outflow(small_cylinders(), int(name[-1]))
        c.immersed = 0
    else:  # channel with the laminar Poiseuille inflow of inletprofile 21
        c = cases.inflow_outflow(small_channel(), 21)
    return c


def _pair(name):
    case = _case(name)
    R, ctx = build_pair(case)
    ctx.form_metrics(case.X, case.Y, case.Z)   # the node plane for inletprofile 21
    area = R.inlet_area()
    flux = 0.8 * area
    ref.set_global("inlet_flux", flux)
    ctx.calc_inlet_area()
    ctx.set_scalar(vfs.S_INLET_FLUX, flux)
    if case.inletprofile == 100:
        plane = cases.inflow_plane(case)
        R.set_inflow_plane(plane)
        ctx.set_inflow_plane(plane)
    return case, R, ctx


NAMES = ["cylinders100", "cylinders2", "poiseuille21"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_inflow_flux(name):
    case, R, ctx = _pair(name)
    R.call("ref_inflow_flux")
    got_flux = ctx.inflow_flux()
    want_flux = R.flux_in()
    assert abs(got_flux - want_flux) <= 1e-13 * abs(want_flux)
    uc_w, uc_g = R.get("Ucont"), ctx.get_field(vfs.UCONT)
    u_w, u_g = R.get("Ucat"), ctx.get_field(vfs.UCAT)
    if case.inletprofile in (2, 100):
        # inlet_flux/inletArea (2) and the flux rescaling (100) carry the rounding of the
        # area and flux sums, so the inlet plane agrees to 1e-13; the rest is untouched
        assert_close(uc_g[0], uc_w[0], rtol=1e-13, atol_frac=1e-14, what="inlet Ucont")
        assert_close(u_g[0], u_w[0], rtol=1e-13, atol_frac=1e-14, what="inlet Ucat")
        np.testing.assert_array_equal(uc_g[1:], uc_w[1:])
        np.testing.assert_array_equal(u_g[1:], u_w[1:])
    else:
        np.testing.assert_array_equal(uc_g, uc_w)
        np.testing.assert_array_equal(u_g, u_w)
    R.close()
    ctx.close()


@pytest.mark.gpu
def test_inletprofile_1_gives_zero_inflow():
    """inletprofile 1 runs with uin = 0 in the reference (bcs.c:408-466); so does the B200
    path."""
    case, R, ctx = _pair("cylinders1")
    R.call("ref_inflow_flux")
    assert ctx.inflow_flux() == R.flux_in() == 0.0
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), R.get("Ucont"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), R.get("Ucat"))
    R.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_outlet_rescaling(name):
    """InflowFlux, then FormBCS with outflow_scale: the outflow equals the inflow."""
    case, R, ctx = _pair(name)
    R.call("ref_inflow_flux")
    ctx.inflow_flux()
    R.call("ref_form_bcs_scaled", 1)
    ctx.form_bcs(1)
    uc_w, uc_g = R.get("lUcont"), ctx.get_field(vfs.UCONT)
    assert_close(uc_g, uc_w, rtol=1e-13, atol_frac=1e-14, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-13, atol_frac=1e-14, what="Ucat")
    nv = case.nvert
    fluid = nv[-2, 1:-1, 1:-1] == 0
    out = uc_g[-2, 1:-1, 1:-1, 2][fluid].sum()
    assert abs(out - ctx.get_scalar(vfs.S_FLUX_IN)) <= 1e-12 * abs(out)
    R.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_inflow_outflow_step(name):
    """One whole step (RungeKutta with InflowFlux and the outlet rescaling, Poisson,
    projection) against the reference; the reference's HYPRE solve is a dense
    least-squares solve of its own system (as in test_step_gpu)."""
    from test_step_gpu import reference_step
    case, R, ctx = _pair(name)
    reference_step(R)
    st = ctx.step(precision=0, rtol=1e-13)
    assert st.poisson.converged == 1
    assert abs(ctx.get_scalar(vfs.S_FLUX_IN) - R.flux_in()) <= 1e-12 * abs(R.flux_in())
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    assert st.max_div < 1e-8
    R.close()
    ctx.close()
