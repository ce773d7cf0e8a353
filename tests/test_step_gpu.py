"""One whole projection time step (Flow_Solver, solvers.c:562-1390, implicit = 0) on the
periodic channel, B200 library against the reference's own functions.  The reference's
HYPRE solve is replaced by a dense least-squares solve of its own matrix and right-hand
side (both mean-free, Remove_Nullspace), so the comparison is solver independent up to
the Poisson tolerance; the GPU solve runs to rtol 1e-13.

Velocity and pressure must agree within 1e-10 relative to their largest magnitude (the
FP64 contract), in both precisions of the solve's preconditioner; each test records the
error it achieved (helpers.report)."""
import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from helpers import assert_close, build_pair, small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def reference_projection(R, immersed=False):
    """Poisson set-up, a dense solve of the reference's own system, pressure update and
    projection (poisson_hypre.c:527-610, solvers.c:1341-1342)."""
    R.call("ref_poisson_lhs")                         # poisson_hypre.c:527
    if immersed:
        R.volume_flux_ibm()                           # poisson_hypre.c:564
    else:
        R.volume_flux()                               # poisson_hypre.c:566
    b = R.poisson_rhs_hypre()                         # poisson_hypre.c:568
    rp, col, val = R.poisson_csr()
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    x = np.linalg.lstsq(A, b, rcond=None)[0]
    x = R.remove_nullspace(x)                         # poisson_hypre.c:602
    R.set("Phi2", x)
    R.call("ref_convert_phi2_phi")                    # poisson_hypre.c:610
    R.call("ref_update_pressure")                     # solvers.c:1341
    R.call("ref_projection")                          # solvers.c:1342


def reference_step(R):
    R.call("ref_ib_bc")                               # solvers.c:609 (ti == tistart)
    R.set("Ucont", R.get("lUcont"))                   # DALocalToGlobal, solvers.c:610
    R.call("ref_calc_k_flux")                         # solvers.c:644
    R.call("ref_pressure_gradient")                   # solvers.c:786
    R.call("ref_runge_kutta")                         # solvers.c:1294
    reference_projection(R)
    R.call("ref_ib_bc")                               # solvers.c:1381
    R.set("Ucont", R.get("lUcont"))
    R.call("ref_contra2cart")                         # solvers.c:1385


def _blocked_cylinders():
    """The open channel with the cylinder array as blocked cells (immersed = 0): bottom
    no-slip, top free-slip, spanwise and streamwise periodic."""
    c = small_cylinders()
    c.immersed = 0
    return c


STEP_CASES = {"channel": lambda: small_channel(), "wavy": lambda: small_channel(wavy=0.15),
              "cylinders": _blocked_cylinders}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(STEP_CASES))
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_one_step_matches_reference(name, precision):
    case = STEP_CASES[name]()
    case.inlet_flux = 5.0
    R, ctx = build_pair(case)
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    reference_step(R)
    st = ctx.step(precision=precision, rtol=1e-13)
    assert st.poisson.converged == 1
    flux, area = R.kflux()
    assert abs(st.mean_k_flux - flux) <= 1e-13 * abs(flux)
    assert abs(ctx.get_scalar(vfs.S_MEAN_K_AREA) - area) <= 1e-13 * area
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    assert st.max_div < 1e-8
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("faces", [(1, 2), (1, 10), (1, -10), (1, 12), (12, 1), (1, 13), (1, 14), (1, 4)])
def test_one_step_boundary_codes(faces):
    """One step of the wavy channel with the j- and j+ faces set to the other wall codes
    FormBCS and Contra2Cart handle (bcs.c:1841-2936, rhs.c:291-675): 2 moving lid (j+),
    10 / -10 free slip, 12 moving wall, 13 and 14 slip lids, 4 outlet on j+."""
    case = small_channel(wavy=0.15)
    case.bctype[2], case.bctype[3] = faces
    case.inlet_flux = 5.0
    R, ctx = build_pair(case)
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    reference_step(R)
    st = ctx.step(precision=1, rtol=1e-13)
    assert st.poisson.converged == 1
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(13, 11, 15), (9, 14, 7), (16, 9, 10)])
@pytest.mark.parametrize("precision", [0, 1])
def test_one_step_odd_grids(dims, precision):
    """Grids whose cell counts are odd in one or more directions: the multigrid hierarchy
    stops coarsening early, and a level with an odd periodic dimension is smoothed by damped
    line Jacobi instead of the zebra sweep; the step must still match the reference."""
    case = small_channel(*dims, wavy=0.1)
    case.inlet_flux = 5.0
    R, ctx = build_pair(case)
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    reference_step(R)
    st = ctx.step(precision=precision, rtol=1e-13)
    assert st.poisson.converged == 1
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    R.close()


@pytest.mark.gpu
def test_ten_steps_stay_divergence_free():
    """Ten steps on the 64^3 channel: every step ends with max|div| below 1e-8 in both
    precisions (the Divergence() gate of main.c:1083-1090)."""
    from vfs_b200 import cases
    case = cases.channel(32, 32, 32)
    case.inlet_flux = 5.0
    R = ref.Reference(case)
    m = R.metrics()
    u = cases.initial_ucat(case)
    uc = cases.ucont_from_ucat(case, u, m)
    for prec in (0, 1):
        ctx = vfs.Context(case.config())
        ctx.set_metrics(m)
        ctx.set_field(vfs.NVERT, case.nvert)
        ctx.set_field(vfs.UCONT, uc)
        ctx.set_field(vfs.UCAT, u)
        ctx.set_field(vfs.UCAT_O, u)
        ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
        for s in range(10):
            st = ctx.step(precision=prec, rtol=1e-10)
            assert st.poisson.converged == 1
            assert st.max_div < 1e-8, (prec, s, st.max_div)
        ctx.close()
    R.close()


def reference_les_step(R, ti):
    """The same step with the eddy viscosity of solvers.c:648-654 before the momentum.
    The reference's step index is ti only for the model (les.c:69 reads it); the rest runs
    as the first step, whose Poisson set-up (setup_lidx2, poisson.c:207-280) allocates its
    vectors only when ti == tistart."""
    R.call("ref_ib_bc")
    R.set("Ucont", R.get("lUcont"))
    R.call("ref_calc_k_flux")
    R.call("ref_contra2cart")
    ref.set_global("ti", ti)
    R.call("ref_les", 1)
    ref.set_global("ti", 0)
    R.call("ref_pressure_gradient")
    R.call("ref_runge_kutta")
    reference_projection(R)
    R.call("ref_ib_bc")
    R.set("Ucont", R.get("lUcont"))
    R.call("ref_contra2cart")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wavy", "cylinders"])
def test_one_les_step_matches_reference(name):
    """A step with the dynamic Smagorinsky model (les = 2) at ti = 2, when Cs is first
    computed on a fresh run."""
    case = STEP_CASES[name]()
    case.les = 2
    case.inlet_flux = 5.0
    R, ctx = build_pair(case, les_nut=True)
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    ctx.set_scalar(vfs.S_TI, 2)
    reference_les_step(R, 2)
    st = ctx.step(precision=0, rtol=1e-13)
    assert st.poisson.converged == 1
    assert R.get("lCs").max() > 0.0
    assert_close(ctx.get_field(vfs.CS), R.get("lCs"), rtol=1e-12, atol_frac=1e-14, what="Cs")
    assert_close(ctx.get_field(vfs.NU_T), R.get("lNu_t"), rtol=1e-12, atol_frac=1e-14, what="nu_t")
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    assert st.max_div < 1e-8
    assert ctx.get_scalar(vfs.S_TI) == 3
    R.close()


def reference_immersed_step(R):
    """The first step with an immersed body (immersed = 1): the IB-node interpolation
    before IB_BC (solvers.c:603-610), inside RungeKutta (rhs.c:1610-1614) and after the
    projection (solvers.c:1366-1370), the immersed VolumeFlux in the Poisson set-up."""
    R.call("ref_calc_inlet_area")                     # main.c:3488, after the IB search
    R.call("ref_ibm_interpolation", 1)                # solvers.c:607
    R.call("ref_ib_bc")
    R.set("Ucont", R.get("lUcont"))
    R.call("ref_calc_k_flux")
    R.call("ref_pressure_gradient")
    R.call("ref_runge_kutta")
    reference_projection(R, immersed=True)
    R.call("ref_ibm_interpolation", 1)                # solvers.c:1368
    R.call("ref_ib_bc")                               # solvers.c:1382
    R.set("Ucont", R.get("lUcont"))
    R.call("ref_contra2cart")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_one_immersed_step_matches_reference(precision):
    """A step of the wavy channel with an icosphere body, classified and listed on each
    side by its own search (the lists agree node for node, test_ibm_gpu.py)."""
    from vfs_b200 import cases
    case = small_channel(16, 14, 20, wavy=0.1)
    case.immersed = 1
    case.inlet_flux = 5.0
    body = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.45, level=3)
    R, ctx = build_pair(case)
    R.ibm_classify(*body, build_list=True)
    ctx.ibm_search(*body)
    assert ctx.ibm_list()[0].shape[0] == R.ibm_list()[0].shape[0] > 0
    ref.set_global("inlet_flux", case.inlet_flux)
    ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    reference_immersed_step(R)
    st = ctx.step(precision=precision, rtol=1e-13)
    assert st.poisson.converged == 1
    assert_close(ctx.get_field(vfs.P), R.get("P"), rtol=1e-10, atol_frac=0, what="P")
    assert_close(ctx.get_field(vfs.UCONT), R.get("lUcont"), rtol=1e-10, atol_frac=0, what="Ucont")
    assert_close(ctx.get_field(vfs.UCAT), R.get("Ucat"), rtol=1e-10, atol_frac=0, what="Ucat")
    assert st.max_div < 1e-8
    R.close()
