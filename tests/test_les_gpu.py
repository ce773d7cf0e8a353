"""Dynamic Smagorinsky eddy viscosity (les.c:67-1252) on the B200 against the reference's
own Compute_Smagorinsky_Constant_1 and Compute_eddy_viscosity_LES (oracle library) on
identical inputs: the periodic channel, the wavy-wall channel and the cylinder array with
immersed-boundary nodes (wall floor of Cs) and solid cells.

Every operation follows the reference's order and is IEEE-exact on both sides except pow(),
which is CUDA's on the device and the host libm's in the reference; their last-place
rounding can differ, so Cs and nu_t are compared to 1e-12 of their largest value."""
import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from helpers import assert_close, build_pair, small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

CASES = {
    "channel": lambda: small_channel(),
    "wavy": lambda: small_channel(wavy=0.15),
    "cylinders": lambda: small_cylinders(),
}


def _les_pair(name, les=2, ti=5):
    case = CASES[name]()
    case.les = les
    R, ctx = build_pair(case, les_nut=True, extra_globals={"ti": ti, "tistart": 0})
    ctx.set_scalar(vfs.S_TI, ti)
    # the model reads the Ucat that Contra2Cart produced (solvers.c:651)
    R.call("ref_contra2cart")
    ctx.contra2cart()
    return case, R, ctx


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_dynamic_smagorinsky(name):
    case, R, ctx = _les_pair(name)
    R.call("ref_les", 1)
    ctx.smagorinsky_constant()
    ctx.eddy_viscosity()
    cs_want, cs_got = R.get("lCs"), ctx.get_field(vfs.CS)
    assert cs_want.max() > 0.0                     # the model is active on this input
    assert_close(cs_got, cs_want, rtol=1e-12, atol_frac=1e-14, what="Cs")
    # clipping and masks are exact: zeros and the ceiling/floor land on the same cells
    np.testing.assert_array_equal(cs_got == 0.0, cs_want == 0.0)
    if case.immersed:
        ib = case.nvert == 1.0
        assert np.all(cs_got[ib] >= 0.001)
    nut_want, nut_got = R.get("lNu_t"), ctx.get_field(vfs.NU_T)
    assert_close(nut_got, nut_want, rtol=1e-12, atol_frac=1e-14, what="nu_t")
    R.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("les,ti,value", [(2, 1, 0.0), (1, 5, 0.01)])
def test_smagorinsky_fixed_values(les, ti, value):
    """Fresh run before ti = 2: Cs = 0 (les.c:69-72); les = 1: Cs = 0.01 (les.c:74-77)."""
    case, R, ctx = _les_pair("wavy", les=les, ti=ti)
    R.call("ref_les", 1)
    ctx.smagorinsky_constant()
    ctx.eddy_viscosity()
    cs = ctx.get_field(vfs.CS)
    np.testing.assert_array_equal(cs, R.get("lCs"))
    assert np.all(cs == value)
    assert_close(ctx.get_field(vfs.NU_T), R.get("lNu_t"), rtol=1e-12, atol_frac=1e-14, what="nu_t")
    R.close()
    ctx.close()
