"""Operator-by-operator parity of the B200 kernels against the reference's own functions
(compiled into the oracle library) on identical inputs.

Pointwise operators must agree bit for bit (the library is built without FMA
contraction, in the reference's operation order); reductions and the Poisson solve are
compared with the tolerances stated in each test.
"""
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


def _pair(name, les=False):
    case = CASES[name]()
    if les:
        case.les = 2
    return case, build_pair(case, les_nut=les)


def _interior(a):
    return a[1:-1, 1:-1, 1:-1]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_contra2cart_bitwise(name):
    case, (R, ctx) = _pair(name)
    R.call("ref_contra2cart")
    ctx.contra2cart()
    want = R.get("Ucat")
    got = ctx.get_field(vfs.UCAT)
    np.testing.assert_array_equal(got, want)
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,les", [("channel", False), ("wavy", False), ("cylinders", False),
                                      ("wavy", True), ("cylinders", True)])
def test_formfunction2_bitwise(name, les):
    case, (R, ctx) = _pair(name, les)
    # Formfunction_2 reads the Ucat that Contra2Cart produced (rhs.c:1642)
    R.call("ref_contra2cart")
    ctx.contra2cart()
    rng = np.random.Generator(np.random.Philox(5))
    rhs0 = rng.standard_normal(R.shape + (3,))
    R.set("Rhs", rhs0)
    ctx.set_field(vfs.RHS, rhs0)
    R.call("ref_formfunction2", 0.75)
    ctx.formfunction2(0.75)
    want = R.get("Rhs")
    got = ctx.get_field(vfs.RHS)
    np.testing.assert_array_equal(got, want)
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_pressure_gradient_bitwise(name):
    case, (R, ctx) = _pair(name)
    flux, area = 0.37, 1.9
    R.set_kflux(flux, area)
    ref.set_global("inlet_flux", 0.25)
    ctx.set_scalar(vfs.S_MEAN_K_FLUX, flux)
    ctx.set_scalar(vfs.S_MEAN_K_AREA, area)
    ctx.set_scalar(vfs.S_INLET_FLUX, 0.25)
    R.call("ref_pressure_gradient")
    ctx.pressure_gradient()
    np.testing.assert_array_equal(ctx.get_field(vfs.DP), R.get("dP"))
    np.testing.assert_array_equal(ctx.get_field(vfs.P), R.get("P"))
    R.close()


def _blocked(case):
    case.immersed = 0
    return case


RK_CASES = {"channel": lambda: small_channel(), "wavy": lambda: small_channel(wavy=0.15),
            "cylinders": lambda: _blocked(small_cylinders())}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(RK_CASES))
def test_runge_kutta_bitwise(name):
    """RungeKutta (rhs.c:1578-1700): InflowFlux, FormBCS, four stages of Contra2Cart +
    Formfunction_2 - dP + stage update, final FormBCS.  With the same dP on both sides
    (Pressure_Gradient from the same k-flux) every operation is pointwise, so Ucont and
    Ucat must agree bit for bit."""
    case = RK_CASES[name]()
    R, ctx = build_pair(case)
    flux, area = 0.37, 1.9
    R.set_kflux(flux, area)
    ref.set_global("inlet_flux", 0.25)
    ctx.set_scalar(vfs.S_MEAN_K_FLUX, flux)
    ctx.set_scalar(vfs.S_MEAN_K_AREA, area)
    ctx.set_scalar(vfs.S_INLET_FLUX, 0.25)
    R.call("ref_pressure_gradient")
    ctx.pressure_gradient()
    np.testing.assert_array_equal(ctx.get_field(vfs.DP), R.get("dP"))
    R.call("ref_runge_kutta")
    ctx.runge_kutta()
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), R.get("lUcont"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), R.get("Ucat"))
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_calc_k_flux(name):
    case, (R, ctx) = _pair(name)
    R.call("ref_calc_k_flux")
    want, _ = R.kflux()
    got = ctx.calc_k_flux()
    assert abs(got - want) <= 1e-13 * max(abs(want), 1e-300) + 1e-15
    R.close()


def _csr_apply(R, x_grid):
    rp, col, val = R.poisson_csr()
    gid = R.gid()
    n = len(rp) - 1
    # interior owners only (the periodic ghost copies of Gid name the same unknowns)
    inner = np.zeros(R.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    m = (gid >= 0) & inner
    xc = np.zeros(n)
    xc[gid[m]] = x_grid[m]
    y = np.zeros(n)
    for r in range(n):
        y[r] = np.dot(val[rp[r]:rp[r + 1]], xc[col[rp[r]:rp[r + 1]]])
    out = np.zeros(R.shape)
    out[m] = y[gid[m]]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_poisson_operator(name):
    """The 19-point operator of PoissonLHSNew: A x on random x, against the recorded CSR."""
    case, (R, ctx) = _pair(name)
    R.call("ref_poisson_lhs")
    ctx.poisson_lhs()
    rng = np.random.Generator(np.random.Philox(11))
    x = rng.standard_normal(R.shape)
    gid = R.gid()
    inner = np.zeros(R.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    x[~((gid >= 0) & inner)] = 0.0
    want = _csr_apply(R, x)
    got = ctx.poisson_apply(x)
    assert_close(got, want, rtol=1e-14, atol_frac=1e-14, what="A x")
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_poisson_rhs(name):
    case, (R, ctx) = _pair(name)
    R.call("ref_poisson_lhs")
    want_c = R.poisson_rhs_hypre()
    gid = R.gid()
    inner = np.zeros(R.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    m = (gid >= 0) & inner
    want = np.zeros(R.shape)
    want[m] = want_c[gid[m]]
    ctx.poisson_rhs()
    got = ctx.get_field(vfs.B)
    assert_close(got, want, rtol=1e-12, atol_frac=1e-12, what="Poisson RHS")
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_update_pressure_projection_divergence(name):
    """Same Phi on both sides: UpdatePressure and Projection bit for bit."""
    case, (R, ctx) = _pair(name)
    R.call("ref_poisson_lhs")
    rng = np.random.Generator(np.random.Philox(3))
    n = lib_n = len(R.poisson_csr()[0]) - 1
    phi2 = rng.standard_normal(n) * 1e-2
    R.set("Phi2", phi2)
    R.call("ref_convert_phi2_phi")
    phi = R.get("Phi")
    ctx.set_field(vfs.PHI, phi)
    R.call("ref_update_pressure")
    ctx.update_pressure()
    np.testing.assert_array_equal(ctx.get_field(vfs.P), R.get("P"))
    R.call("ref_projection")
    ctx.projection()
    # the device keeps one Ucont array, equal to the reference's local lUcont (the copy
    # every consumer reads after its periodic refresh); the global Ucont differs from it
    # only on periodic ghost planes in the components tangential to them
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), R.get("lUcont"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), R.get("Ucat"))
    # Divergence (main.c:1083-1090) recomputed from the reference's fields
    uc, aj, nv = R.get("lUcont"), R.get("lAj"), R.get("lNvert")
    d = np.abs((uc[1:-1, 1:-1, 1:-1, 0] - uc[1:-1, 1:-1, :-2, 0] + uc[1:-1, 1:-1, 1:-1, 1] -
                uc[1:-1, :-2, 1:-1, 1] + uc[1:-1, 1:-1, 1:-1, 2] - uc[:-2, 1:-1, 1:-1, 2]) * aj[1:-1, 1:-1, 1:-1])
    s = (nv[1:-1, 1:-1, 1:-1] + nv[2:, 1:-1, 1:-1] + nv[:-2, 1:-1, 1:-1] + nv[1:-1, 2:, 1:-1] +
         nv[1:-1, :-2, 1:-1] + nv[1:-1, 1:-1, 2:] + nv[1:-1, 1:-1, :-2])
    d[s > 0.1] = 0
    assert ctx.divergence() == d.max()
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_poisson_solve_matches_direct(name, precision):
    """Solve to rtol 1e-13 (mixed, FP64, and FP32 inner FGMRES in FP64 refinement) and compare Phi with a dense least-squares
    solve of the reference's own matrix and right-hand side, both mean-free, to 1e-10
    relative to max |Phi|."""
    case, (R, ctx) = _pair(name)
    R.call("ref_poisson_lhs")
    b = R.poisson_rhs_hypre()
    rp, col, val = R.poisson_csr()
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        A[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    x = np.linalg.lstsq(A, b, rcond=None)[0]
    x = R.remove_nullspace(x)
    R.set("Phi2", x)
    R.call("ref_convert_phi2_phi")
    want = R.get("Phi")
    ctx.poisson_rhs()
    st = ctx.poisson_solve(precision=precision, rtol=1e-13)
    assert st.converged == 1
    got = ctx.get_field(vfs.PHI)
    assert_close(got, want, rtol=1e-10, atol_frac=0, what="phi")
    R.close()


@pytest.mark.gpu
def test_poisson_solve_starts_from_the_previous_solution():
    """The solve's initial guess follows the reference's persistent Phi2 (zero when the
    unknowns are numbered, poisson.c:280-282; the previous solution afterwards,
    poisson_hypre.c:571): the first solve after PoissonLHSNew starts from 0 (initial
    residual = |b|), a second solve of the same system starts at its solution and stops
    at once, zero_guess = 1 reaches the same Phi from 0, and a Phi set through the ABI is
    the next solve's starting point."""
    case, (R, ctx) = _pair("cylinders")
    ctx.poisson_lhs()
    ctx.poisson_rhs()
    first = ctx.poisson_solve(precision=1, rtol=1e-12)
    assert first.converged == 1 and first.iterations > 0
    b = ctx.get_field(vfs.B)
    assert first.r0 == pytest.approx(np.linalg.norm(b), rel=1e-12)
    phi = ctx.get_field(vfs.PHI)
    again = ctx.poisson_solve(precision=1, rtol=1e-12)
    # the first solve stops within twice the target on its true residual
    assert again.converged == 1 and again.iterations <= 1
    assert again.r0 <= 2.0001e-12 * first.r0
    assert_close(ctx.get_field(vfs.PHI), phi, rtol=1e-10, atol_frac=1e-12, what="phi again")
    cold = ctx.poisson_solve(precision=1, rtol=1e-12, zero_guess=1)
    assert cold.r0 == pytest.approx(first.r0, rel=1e-12) and cold.iterations > 0
    assert_close(ctx.get_field(vfs.PHI), phi, rtol=1e-8, atol_frac=1e-9, what="phi from 0")
    ctx.set_field(vfs.PHI, 0.5 * phi)
    half = ctx.poisson_solve(precision=1, rtol=1e-12)
    assert half.r0 == pytest.approx(0.5 * first.r0, rel=1e-6)
    assert_close(ctx.get_field(vfs.PHI), phi, rtol=1e-8, atol_frac=1e-9, what="phi from the set guess")
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_form_metrics_bitwise(name):
    """FormMetrics on the device from the grid.dat nodes equals the reference's metrics,
    ghost planes and periodic images included."""
    case = CASES[name]()
    R = ref.Reference(case)
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    for key, fid in vfs.METRIC_FIELDS.items():
        want = R.get(ref.METRIC_VECS[key])
        got = ctx.get_field(fid)
        np.testing.assert_array_equal(got, want, err_msg=key)
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_formfunction2_forms_agree(name):
    """The three forms of Formfunction_2 on the same inputs: the three-kernel form
    (diagnostic id 7), the one-pass k-marching kernel (id 11) and the form a step runs
    (id 8) give identical right-hand sides."""
    case, (R, ctx) = _pair(name)
    ctx.contra2cart()
    rhs0 = np.random.Generator(np.random.Philox(9)).standard_normal(R.shape + (3,))
    ctx.set_field(vfs.RHS, rhs0)
    ctx.run_kernel(7, 1)
    want = ctx.get_field(vfs.RHS)
    for kid in (11, 8):
        ctx.set_field(vfs.RHS, rhs0)
        ctx.run_kernel(kid, 1)
        np.testing.assert_array_equal(ctx.get_field(vfs.RHS), want, err_msg="kernel id %d" % kid)
    R.close()
