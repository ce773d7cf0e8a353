"""Tangent-linear and discrete adjoint of a window of projection steps (no counterpart in the
reference, which has no adjoint): the measured operator matrices against the forward
kernels, the tangent against central finite differences of the forward step, the adjoint
against the tangent (dot-product test), the gradient against central differences at 32
seeded control entries, and checkpointing that does not change the gradient.

Cases: the periodic channel with the k-flux forcing (initial-Ucont control, kinetic
energy), the open channel with an inlet plane and blocked cylinders (inflow-plane control,
drag: pressure force plus viscous traction), and the wavy channel with an immersed sphere
(initial-Ucont control, drag on the body's cells)."""
import numpy as np
import pytest

import vfs_b200 as vfs
from vfs_b200 import cases
from helpers import report

NSTEPS = 2


def _case(name):
    if name == "channel":
        c = cases.channel(12, 10, 14)
        c.inlet_flux = 5.0
        return c, vfs.OBJ_KINETIC_ENERGY, vfs.CTRL_INITIAL_UCONT, None
    if name == "inlet":
        c = cases.open_channel_cylinders(16, 12, 24, D=0.6, Lx=3.2, Lz=8.0, Ly=1.0)
        c.immersed = 0
        cases.inflow_outflow(c, 100)
        return c, vfs.OBJ_DRAG, vfs.CTRL_INFLOW_PLANE, None
    c = cases.channel(16, 14, 20, wavy=0.1)
    c.immersed = 1
    c.inlet_flux = 5.0
    body = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.45, level=3)
    return c, vfs.OBJ_DRAG, vfs.CTRL_INITIAL_UCONT, body


def _context(name, seed=0):
    case, obj, ctrl, body = _case(name)
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    if body is not None:
        ctx.ibm_search(*body)
    m = {n: ctx.get_field(f) for n, f in vfs.METRIC_FIELDS.items()}
    case.nvert = ctx.get_field(vfs.NVERT)
    u = cases.initial_ucat(case, seed=seed)
    uc = cases.ucont_from_ucat(case, u, m)
    ctx.set_field(vfs.UCONT, uc)
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    rng = np.random.Generator(np.random.Philox(seed + 3))
    ctx.set_field(vfs.P, 0.1 * rng.standard_normal(ctx.shape))
    if case.bctype[4] == 5:
        ctx.set_scalar(vfs.S_INLET_FLUX, 0.0)
        ctx.calc_inlet_area()
        ctx.set_scalar(vfs.S_INLET_FLUX, 0.8 * ctx.get_scalar(vfs.S_INLET_AREA))
        ctx.set_inflow_plane(cases.inflow_plane(case))
    else:
        ctx.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    return ctx, case, obj, ctrl


def _control(ctx, case, ctrl):
    if ctrl == vfs.CTRL_INITIAL_UCONT:
        return ctx.get_field(vfs.UCONT)
    return cases.inflow_plane(case)


def _set_control(ctx, ctrl, x):
    if ctrl == vfs.CTRL_INITIAL_UCONT:
        ctx.set_field(vfs.UCONT, x)
    else:
        ctx.set_inflow_plane(x)


def _direction(ctx, case, ctrl, seed):
    rng = np.random.Generator(np.random.Philox(seed + 101))
    d = rng.standard_normal(ctx.control_shape(ctrl))
    if ctrl == vfs.CTRL_INFLOW_PLANE:
        d[0, :, :] = 0; d[-1, :, :] = 0; d[:, 0, :] = 0; d[:, -1, :] = 0
    return d


def _fd(ctx, case, obj, ctrl, d, x0, rel=1e-6, rtol=1e-12):
    eps = rel * np.abs(x0).max() / np.abs(d).max()
    _set_control(ctx, ctrl, x0 + eps * d)
    jp = ctx.objective(NSTEPS, obj, ctrl, rtol=rtol, max_iter=400)
    _set_control(ctx, ctrl, x0 - eps * d)
    jm = ctx.objective(NSTEPS, obj, ctrl, rtol=rtol, max_iter=400)
    _set_control(ctx, ctrl, x0)
    return (jp - jm) / (2 * eps)


NAMES = ["channel", "inlet", "sphere"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_measured_operators_match_kernels(name):
    """Dot-product test of every operator: <y, L x> by its forward kernels equals <L^T y, x>
    by the transpose the adjoint sweep applies (hand-written or measured)."""
    ctx, case, obj, ctrl = _context(name)
    rng = np.random.Generator(np.random.Philox(7))
    N = int(np.prod(ctx.shape))
    checked = 0
    for op in range(len(vfs.OP_NAMES)):
        slots, nnz = ctx.adjoint_op_info(op)
        if not slots:
            continue
        x = rng.standard_normal((len(slots), N))
        y = rng.standard_normal((len(slots), N))
        lx, lty = ctx.adjoint_op_check(op, x, y)
        a, b = float((y * lx).sum()), float((lty * x).sum())
        scale = float(np.abs(y * lx).sum())
        assert abs(a - b) <= 1e-12 * scale, (vfs.OP_NAMES[op], a, b, nnz)
        checked += 1
    assert checked >= 8
    ctx.close()


def _handwritten_check(ctx, seed):
    """Each hand-written transpose against the measured matrix (element-wise, relative to
    the largest entry) and in the dot-product test against the forward kernels."""
    rng = np.random.Generator(np.random.Philox(seed))
    N = int(np.prod(ctx.shape))
    worst = 0.0
    for name in vfs.OP_HANDWRITTEN:
        op = vfs.OP_NAMES.index(name)
        slots, nnz = ctx.adjoint_op_info(op)
        if not slots:
            continue
        x = rng.standard_normal((len(slots), N))
        y = rng.standard_normal((len(slots), N))
        lx, lty = ctx.adjoint_op_check(op, x, y)
        lm = ctx.adjoint_op_measured(op, y)
        err = float(np.abs(lty - lm).max() / np.abs(lm).max())
        assert err <= 1e-13, (name, err)
        a, b = float((y * lx).sum()), float((lty * x).sum())
        assert abs(a - b) <= 1e-12 * float(np.abs(y * lx).sum()), (name, a, b)
        worst = max(worst, err)
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_handwritten_transposes_match_measured(name):
    ctx, case, obj, ctrl = _context(name)
    _handwritten_check(ctx, 17)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", ["ik", "ijk", "none", "slip"])
def test_handwritten_transposes_random_nvert(periodic):
    """Every branch of the stencils and boundary rules: nvert drawn from {0, 1, 2, 3} on a
    wavy grid (one-sided cross differences next to IB nodes and solids, Projection's j-face
    nvert sum 5), with periodic directions i and k, all three, or none (walls all round), or
    none with slip walls on both i faces and on top (their ghosts mirror Ucat_o), a no-slip
    bottom and k- wall, and an outflow face at k+."""
    case = cases.channel(10, 9, 12, wavy=0.1)
    case.i_periodic = int("i" in periodic)
    case.j_periodic = int("j" in periodic)
    case.k_periodic = int("k" in periodic)
    case.bctype = [7 if case.i_periodic else 1] * 2 + [7 if case.j_periodic else 1] * 2 + \
                  [7 if case.k_periodic else 1] * 2
    if periodic == "slip":
        case.bctype = [10, 10, 1, 10, 1, 4]
    rng = np.random.Generator(np.random.Philox(23))
    nv = np.zeros(case.da_shape)
    nv[1:-1, 1:-1, 1:-1] = rng.choice([0, 0, 0, 0, 1, 2, 3], size=nv[1:-1, 1:-1, 1:-1].shape)
    case.nvert = nv
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, nv)
    ctx.set_scalar(vfs.S_INLET_FLUX, 0.0)
    report("hand-written vs measured transposes, random nvert " + periodic, _handwritten_check(ctx, 29))
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_tangent_matches_finite_differences(name):
    """Central differences of J over two steps (FP64 Poisson solves to rtol 1e-12)."""
    ctx, case, obj, ctrl = _context(name)
    x0 = _control(ctx, case, ctrl)
    d = _direction(ctx, case, ctrl, 0)
    J, dJ = ctx.tangent(d, NSTEPS, obj, ctrl)
    assert J == pytest.approx(ctx.objective(NSTEPS, obj, ctrl), rel=1e-13)
    fd = _fd(ctx, case, obj, ctrl, d, x0)
    assert abs(dJ - fd) <= 1e-6 * abs(fd), (J, dJ, fd)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_adjoint_matches_tangent(name):
    """<dJ/dcontrol, d> from the adjoint equals the tangent's dJ along d."""
    ctx, case, obj, ctrl = _context(name)
    g, st = ctx.adjoint_gradient(NSTEPS, obj, ctrl)
    for seed in (0, 1):
        d = _direction(ctx, case, ctrl, seed)
        J, dJ = ctx.tangent(d, NSTEPS, obj, ctrl)
        assert st.J == pytest.approx(J, rel=1e-12)
        assert abs(float((g * d).sum()) - dJ) <= 1e-9 * abs(dJ) + 1e-12 * np.abs(g).sum() * np.abs(d).max(), \
            (float((g * d).sum()), dJ)
    ctx.close()


@pytest.mark.gpu
def test_gradient_matches_finite_differences_at_32_inlet_nodes():
    """dJ/d(inflow plane) at 32 seeded inlet entries against central differences, along a
    random combination of the 32 entries and entry by entry.  The differences use a step of
    1e-4 of the plane's largest value: with the step of 1e-6 the change of J from a single
    entry (about 1e-11) is of the order of the rounding noise of the forward window itself,
    while the truncation error of the 1e-4 step stays near 1e-8 relative.  Agreement: 1e-6
    relative along the combination, 1e-6 of the largest gradient entry entry by entry."""
    ctx, case, obj, ctrl = _context("inlet")
    g, st = ctx.adjoint_gradient(NSTEPS, obj, ctrl)
    x0 = _control(ctx, case, ctrl)
    rng = np.random.Generator(np.random.Philox(32))
    my, mx = ctx.shape[1], ctx.shape[2]
    picks = set()
    while len(picks) < 32:
        picks.add((int(rng.integers(1, my - 1)), int(rng.integers(1, mx - 1)), int(rng.integers(0, 3))))
    picks = sorted(picks)
    d = np.zeros_like(x0)
    for (j, i, c) in picks:
        d[j, i, c] = rng.standard_normal()
    fd = _fd(ctx, case, obj, ctrl, d, x0, rel=1e-4)
    gd = float((g * d).sum())
    assert abs(gd - fd) <= 1e-6 * abs(fd), (gd, fd)
    gmax = np.abs(g).max()
    for (j, i, c) in picks:
        e = np.zeros_like(x0)
        e[j, i, c] = 1.0
        fd = _fd(ctx, case, obj, ctrl, e, x0, rel=1e-4)
        assert abs(g[j, i, c] - fd) <= 1e-6 * gmax, ((j, i, c), g[j, i, c], fd, gmax)
    ctx.close()


@pytest.mark.gpu
def test_checkpointing_does_not_change_the_gradient():
    ctx, case, obj, ctrl = _context("channel")
    g1, s1 = ctx.adjoint_gradient(3, obj, ctrl, checkpoint_every=1)
    g3, s3 = ctx.adjoint_gradient(3, obj, ctrl, checkpoint_every=3)
    assert s1.checkpoints == 3 and s3.checkpoints == 1
    assert s1.recomputed_steps == 3 and s3.recomputed_steps == 3
    np.testing.assert_allclose(g1, g3, rtol=1e-10, atol=1e-12 * np.abs(g3).max())
    ctx.close()


@pytest.mark.gpu
def test_drag_objective_adds_the_viscous_traction():
    """OBJ_DRAG - OBJ_PRESSURE_DRAG after one step equals the viscous traction summed on the
    host from the state of the same step: 2/ren |csi|^2 aj w per i-face (|eta|^2 per j-face)
    that a fluid cell shares with a body cell."""
    ctx, case, obj, ctrl = _context("inlet")
    jd = ctx.objective(1, objective=vfs.OBJ_DRAG, control=ctrl)
    jp = ctx.objective(1, objective=vfs.OBJ_PRESSURE_DRAG, control=ctrl)
    ctx.step(precision=1, rtol=1e-12)
    u = ctx.get_field(vfs.UCAT)
    nv = ctx.get_field(vfs.NVERT)
    csi, eta, aj = ctx.get_field(vfs.CSI), ctx.get_field(vfs.ETA), ctx.get_field(vfs.AJ)
    kz, jz, iz = nv.shape
    jv = 0.0
    for k in range(1, kz - 1):
        for j in range(1, jz - 1):
            for i in range(1, iz - 1):
                if nv[k, j, i] != 0:
                    continue
                ni = int(i + 1 <= iz - 2 and nv[k, j, i + 1] > 0) + int(i - 1 >= 1 and nv[k, j, i - 1] > 0)
                nj = int(j + 1 <= jz - 2 and nv[k, j + 1, i] > 0) + int(j - 1 >= 1 and nv[k, j - 1, i] > 0)
                if ni or nj:
                    ci = float(np.dot(csi[k, j, i], csi[k, j, i]))
                    cj = float(np.dot(eta[k, j, i], eta[k, j, i]))
                    jv += 2.0 / case.ren * (ni * ci + nj * cj) * aj[k, j, i] * u[k, j, i, 2]
    ctx.close()
    assert jv != 0.0
    assert abs((jd - jp) - jv) <= 1e-9 * abs(jv), (jd - jp, jv)
