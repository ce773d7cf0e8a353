"""The gradient-check harness's torch binding of the adjoint: a torch.autograd.Function
whose forward is the objective of a window of steps as a function of the inflow plane and
whose backward is the library's discrete adjoint (vfs_adjoint_gradient).  Used only here:
the library itself has no torch dependency."""
import numpy as np
import pytest

import vfs_b200 as vfs

torch = pytest.importorskip("torch")

NSTEPS = 2


class WindowObjective(torch.autograd.Function):
    """J(plane) after NSTEPS steps; backward by the adjoint."""

    @staticmethod
    def forward(fctx, plane, vctx, objective):
        vctx.set_inflow_plane(plane.detach().cpu().numpy())
        g, st = vctx.adjoint_gradient(NSTEPS, objective, vfs.CTRL_INFLOW_PLANE)
        fctx.save_for_backward(torch.from_numpy(g))
        return torch.tensor(st.J, dtype=torch.float64)

    @staticmethod
    def backward(fctx, grad_out):
        (g,) = fctx.saved_tensors
        return grad_out * g, None, None


@pytest.mark.gpu
def test_autograd_binding_matches_tangent_and_differences():
    from test_adjoint_gpu import _context, _control
    ctx, case, obj, ctrl = _context("inlet")
    x0 = _control(ctx, case, ctrl)
    plane = torch.tensor(x0, dtype=torch.float64, requires_grad=True)
    J = WindowObjective.apply(plane, ctx, obj)
    J.backward()
    g = plane.grad.numpy()
    rng = np.random.Generator(np.random.Philox(5))
    d = rng.standard_normal(x0.shape)
    d[0], d[-1], d[:, 0], d[:, -1] = 0, 0, 0, 0
    Jt, dJ = ctx.tangent(d, NSTEPS, obj, ctrl)
    assert float(J.detach()) == pytest.approx(Jt, rel=1e-12)
    assert float((g * d).sum()) == pytest.approx(dJ, rel=1e-9)
    # central differences with a step of 1e-4 of the plane's largest value: at 1e-6 the
    # change of J (about 1e-6 relative) is within a few decades of the forward window's own
    # solver noise (rtol 1e-12 on each Poisson solve, whose warm start from the previous
    # step's Phi shifts where each solve stops), while the truncation error of the 1e-4
    # step stays near 1e-8 relative
    eps = 1e-4 * np.abs(x0).max() / np.abs(d).max()
    with torch.no_grad():
        jp = WindowObjective.apply(torch.tensor(x0 + eps * d), ctx, obj)
        jm = WindowObjective.apply(torch.tensor(x0 - eps * d), ctx, obj)
    fd = float(jp - jm) / (2 * eps)
    assert abs(fd - dJ) <= 1e-6 * abs(dJ), (fd, dJ)
    ctx.close()
