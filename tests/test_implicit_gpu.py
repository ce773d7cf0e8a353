"""Implicit momentum (implicit = 4) on the B200 against the reference's own
residual, FormFunction_SNES (momentum.c:2197-2300, compiled into oracle/_ref).

* The residual F(Ucont) = -Ucont/dt + Ucont_o/dt + 0.5 Formfunction_2(Ucont) + 0.5 RHS_o
  - dP, with the reference's wall faces and Contra2Cart / IB_BC, is bit-identical.
* The Newton-Krylov solve (Implicit_MatrixFree, implicitsolver.c:4196): the reference
  hands F to PETSc's SNES, which is not in this image, so its iterates cannot be compared;
  the solution is checked against the reference's equations instead: the reference's own
  F at the library's solution is below imp_tol times F at the start.
* A few implicit time steps (vfs_step with implicit = 4) keep the projection's divergence
  bound."""
import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from vfs_b200 import cases
from helpers import build_pair, report, small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

CASES = {
    "channel": lambda: small_channel(12, 10, 14),
    "wavy": lambda: small_channel(12, 10, 14, wavy=0.15),
    "cylinders": lambda: small_cylinders(),
}


def _old_level(R, ctx, seed):
    """Ucont_o, RHS_o and dP: the same seeded values on both sides."""
    rng = np.random.Generator(np.random.Philox(seed))
    uc = ctx.get_field(vfs.UCONT)
    uo = uc * (1.0 + 0.01 * rng.standard_normal(uc.shape))
    ro = 0.1 * rng.standard_normal(uc.shape)
    dp = 0.1 * rng.standard_normal(uc.shape)
    for n in ("Ucont_o", "lUcont_o"):
        R.set(n, uo)
    R.set("RHS_o", ro)
    R.set("dP", dp)
    ctx.set_field(vfs.UCONT_O, uo)
    ctx.set_field(vfs.RHS_O, ro)
    ctx.set_field(vfs.DP, dp)
    return uo, ro, dp


def _step_old_level(R, ctx, seed):
    """Ucont_o seeded, dP and RHS_o as a step forms them (Pressure_Gradient; Formfunction_2
    of the initial state, solvers.c:1284-1286): zero where the faces are masked, so that
    F = 0 has a solution."""
    rng = np.random.Generator(np.random.Philox(seed))
    uc = ctx.get_field(vfs.UCONT)
    uo = uc * (1.0 + 0.01 * rng.standard_normal(uc.shape))
    for n in ("Ucont_o", "lUcont_o"):
        R.set(n, uo)
    ctx.set_field(vfs.UCONT_O, uo)
    ctx.calc_inlet_area()      # the mean k-face area of the k-periodic forcing (main.c:3488)
    ctx.pressure_gradient()
    ctx.set_field(vfs.RHS, np.zeros(uc.shape))
    ctx.formfunction2(1.0)
    ro, dp = ctx.get_field(vfs.RHS), ctx.get_field(vfs.DP)
    ctx.set_field(vfs.RHS_O, ro)
    R.set("RHS_o", ro)
    R.set("dP", dp)


def _ref_residual(R, U):
    R.set("Uin", U)
    R.call("ref_formfunction_snes")
    return R.get("Rhs")


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_residual_bitwise(name):
    case = CASES[name]()
    R, ctx = build_pair(case)
    _old_level(R, ctx, 5)
    rng = np.random.Generator(np.random.Philox(11))
    U = ctx.get_field(vfs.UCONT) + 0.01 * rng.standard_normal(R.shape + (3,))
    want = _ref_residual(R, U)
    ctx.set_field(vfs.UCONT, U)
    ctx.implicit_residual()
    assert np.isfinite(want).all()
    np.testing.assert_array_equal(ctx.get_field(vfs.RHS), want)
    np.testing.assert_array_equal(ctx.get_field(vfs.UCONT), R.get("lUcont"))
    np.testing.assert_array_equal(ctx.get_field(vfs.UCAT), R.get("lUcat"))
    R.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_newton_solution_satisfies_the_reference_equations(name):
    """The library's Newton-Krylov solution U*: |F_ref(U*)| <= imp_tol |F_ref(U0)|, and the
    reference's F at U* is the library's final residual (the same function)."""
    case = CASES[name]()
    case.implicit = 4
    case.imp_tol = 1e-6
    R, ctx = build_pair(case)
    _step_old_level(R, ctx, 7)
    f0_ref = np.linalg.norm(_ref_residual(R, ctx.get_field(vfs.UCONT)))
    assert np.isfinite(f0_ref) and f0_ref > 0
    st = ctx.implicit_momentum()
    assert st.converged == 1 and st.newton_iterations >= 1
    # the solve starts after InflowFlux and FormBCS, which leave these Ucont unchanged
    assert abs(st.f0 - f0_ref) <= 1e-12 * f0_ref
    f_ref = np.linalg.norm(_ref_residual(R, ctx.get_field(vfs.UCONT)))
    report("|F_ref(U*)| / |F_ref(U0)|", f_ref / f0_ref)
    assert f_ref <= case.imp_tol * f0_ref * (1 + 1e-9)
    assert abs(f_ref - st.ffinal) <= 1e-10 * st.f0
    R.close()


@pytest.mark.gpu
def test_implicit_steps_keep_the_divergence_bound():
    case = cases.channel(16, 14, 20, wavy=0.1)
    case.implicit = 4
    case.inlet_flux = 5.0
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    m = {n: ctx.get_field(f) for n, f in vfs.METRIC_FIELDS.items()}
    u = cases.initial_ucat(case)
    uc = cases.ucont_from_ucat(case, u, m)
    ctx.set_field(vfs.UCONT, uc)
    ctx.set_field(vfs.UCONT_O, uc)
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    for _ in range(3):
        st = ctx.step(precision=1, rtol=1e-12)
        assert st.poisson.converged == 1
        assert st.max_div < 1e-9
    assert np.isfinite(ctx.get_field(vfs.UCAT)).all()
    ctx.close()
