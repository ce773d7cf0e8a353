"""Immersed-boundary reconstruction with a wall model and with moving bodies, on the B200
against the reference's own functions.

* ibm_interpolation_advanced (ibm.c:3405-3530) with -wallfunction from ti > 0: the node
  velocity from wall_function_roughness_a (sediment_transport-Y.c:68, compiled into the
  oracle) or, with -roughness, the rough-wall log law (wallfunction.c:71), the friction
  velocity ustar, a non-zero surface velocity of the body (ibm->u).
  The wall model's logarithms, exponentials and sine are CUDA's and glibc's, which may
  differ in the last bit, so the comparison is to 1e-12 relative.
* A body that moves between steps (movefsi): the IB search of every step with the cells
  the body uncovers marked as IB nodes (ibm.c:346-357), PoissonLHSNew and the solver set-up
  every step (poisson_hypre.c:540-553), the reconstruction without the solid-stencil
  test and Contra2Cart without the zeroing of solid cells (ibm.c:3444, rhs.c:298)."""
import numpy as np
import pytest

from oracle import ref, steps
import vfs_b200 as vfs
from vfs_b200 import cases
from helpers import assert_close, build_pair, small_channel

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _by_cell(ints, dbls):
    """The list in (k, j, i) order (the reference builds it in its own order)."""
    order = np.lexsort((ints[:, 0], ints[:, 1], ints[:, 2]))
    return ints[order], dbls[order]


def _sphere(dz=0.0):
    x, y, z, tri = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.45, level=3)
    return x, y, z + dz, tri


def _surface_velocity(x, y, z):
    """Vertex velocities of a rigid motion: a translation (0.1, 0, 0.05) plus a rotation
    about the sphere's centre."""
    cx, cy, cz = np.pi / 2, 1.0, np.pi
    return 0.1 + 0.2 * (y - cy), -0.2 * (x - cx) + 0.3 * (z - cz), 0.05 - 0.3 * (y - cy)


@pytest.mark.gpu
@pytest.mark.parametrize("roughness", [0.0, 1e-3])
def test_wall_model_reconstruction_matches_reference(roughness):
    """roughness 0: wall_function_roughness_a; > 0 (-roughness): body 0 takes the rough-wall
    log law wall_function_roughness_loglaw (wallfunction.c:71)."""
    case = small_channel(16, 14, 20, wavy=0.1)
    case.immersed = 1
    case.wallfunction = 1
    case.roughness = roughness
    R, ctx = build_pair(case)
    x, y, z, tri = _sphere()
    R.ibm_classify(x, y, z, tri, build_list=True)
    ctx.ibm_search(x, y, z, tri)
    u, v, w = _surface_velocity(x, y, z)
    R.ibm_set_velocity(u, v, w)
    ctx.ibm_set_velocity(u, v, w)
    ref.set_global("ti", 3)
    ctx.set_scalar(vfs.S_TI, 3)
    R.call("ref_ibm_interpolation", 1)
    ref.set_global("ti", 0)
    ctx.ibm_interpolation()
    nodes = ctx.get_field(vfs.NVERT) == 1
    assert nodes.sum() > 50
    want, got = R.get("Ucat"), ctx.get_field(vfs.UCAT)
    assert_close(got[nodes], want[nodes], rtol=1e-12, atol_frac=0, what="IB-node Ucat (wall model)")
    assert_close(got[~nodes], want[~nodes], rtol=0, atol_frac=0, what="Ucat elsewhere")
    ustar_w, ustar_g = R.get("lUstar"), ctx.get_field(vfs.USTAR)
    assert np.abs(ustar_w[nodes]).max() > 0
    assert_close(ustar_g[nodes], ustar_w[nodes], rtol=1e-12, atol_frac=0, what="ustar")
    np.testing.assert_array_equal(ctx.get_field(vfs.P), R.get("P"))
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-12, atol_frac=0, what="Ucont")
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("wallfunction", [0, 1])
def test_moving_body_steps_match_reference(wallfunction):
    case = small_channel(16, 14, 24, wavy=0.1)
    case.immersed = 1
    case.moving = 1
    case.wallfunction = wallfunction
    case.inlet_flux = 5.0
    R, ctx = build_pair(case)
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    dz = 0.4 * (2 * np.pi / 24)          # 0.4 of a cell per step along the stream
    stepper = None
    uncovered = 0
    for s in range(4):
        x, y, z, tri = _sphere(dz * s)
        u, v, w = _surface_velocity(x, y, z)
        before = ctx.get_field(vfs.NVERT)
        R.ibm_classify(x, y, z, tri, build_list=True)
        ctx.ibm_search(x, y, z, tri)
        R.ibm_set_velocity(u, v, w)
        ctx.ibm_set_velocity(u, v, w)
        after = ctx.get_field(vfs.NVERT)
        np.testing.assert_array_equal(after, R.get("lNvert"), err_msg="nvert after the search of step %d" % s)
        ints_r, dbl_r = _by_cell(*R.ibm_list())
        ints_g, dbl_g = _by_cell(*ctx.ibm_list())
        np.testing.assert_array_equal(ints_g, ints_r)
        if s > 0:
            uncovered += int(((before > 2.5) & (after == 1)).sum())
        if stepper is None:
            R.call("ref_calc_inlet_area")
            stepper = steps.ReferenceStepper(R, rtol=1e-13)
        stepper.step()
        st = ctx.step(precision=1, rtol=1e-13)
        assert st.poisson.converged == 1
    assert uncovered > 0   # the moving body uncovered cells, which became IB nodes
    for f, name in ((vfs.P, "P"), (vfs.UCONT, "Ucont"), (vfs.UCAT, "Ucat")):
        want = R.get({"P": "P", "Ucont": "lUcont", "Ucat": "Ucat"}[name])
        assert_close(ctx.get_field(f), want, rtol=1e-10, atol_frac=0, what=name + " after 4 moving steps")
    R.close()
