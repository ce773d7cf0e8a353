"""The whole time step as one CUDA graph (vfs_solve_opts.graph = 1): captured once, replayed
every step, the Poisson solve's restart and Arnoldi loops as conditional WHILE nodes whose
conditions the solver's control kernels set on the device.  The replay runs the same
kernels as the step launched one by one, so every field must agree bit for bit, and the
solve must take the same iterations."""
import numpy as np
import pytest

import vfs_b200 as vfs
from vfs_b200 import cases
from helpers import small_channel, small_cylinders


def _cases():
    def inout():
        c = cases.inflow_outflow(small_cylinders(), 100)
        c.immersed = 0
        return c

    def les():
        c = small_channel(16, 12, 18, wavy=0.1)
        c.les = 2
        return c

    def sphere():
        c = small_channel(16, 14, 20, wavy=0.1)
        c.immersed = 1
        return c
    return {"inflow_outflow": inout, "les": les, "sphere": sphere}


def _context(case):
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    if case.immersed:
        ctx.ibm_search(*cases.icosphere((np.pi / 2, 1.0, np.pi), 0.45, level=3))
    m = {k: ctx.get_field(f) for k, f in vfs.METRIC_FIELDS.items()}
    u = cases.initial_ucat(case)
    ctx.set_field(vfs.UCONT, cases.ucont_from_ucat(case, u, m))
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    if case.inletprofile == 100:
        ctx.set_inflow_plane(cases.inflow_plane(case))
        _, area = ctx.calc_inlet_area()
        ctx.set_scalar(vfs.S_INLET_FLUX, 0.8 * area)
    else:
        ctx.set_scalar(vfs.S_INLET_FLUX, 5.0)
    return ctx


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["inflow_outflow", "les", "sphere"])
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_graph_step_matches_launched_step(name, precision):
    case = _cases()[name]()
    a, b = _context(case), _context(case)
    for s in range(6):
        sa = a.step(precision=precision, rtol=1e-10)
        sb = b.step(precision=precision, rtol=1e-10, graph=1)
        assert sa.poisson.iterations == sb.poisson.iterations, s
        assert sb.poisson.converged == 1
        assert sa.max_div == sb.max_div
        assert sa.mean_k_flux == sb.mean_k_flux
    for f in (vfs.UCONT, vfs.UCAT, vfs.P, vfs.PHI, vfs.UCONT_O, vfs.UCAT_O, vfs.NU_T):
        np.testing.assert_array_equal(b.get_field(f), a.get_field(f), err_msg=str(f))
    for q in (vfs.S_MEAN_K_FLUX, vfs.S_FLUX_IN, vfs.S_FLUX_OUT, vfs.S_TI):
        assert b.get_scalar(q) == a.get_scalar(q)
    a.close()
    b.close()


@pytest.mark.gpu
def test_graph_is_captured_again_after_a_setup_change():
    """A new nvert field (a new operator) invalidates the captured step: the next graph
    step is launched one by one, then captured anew, still matching the launched form."""
    case = _cases()["inflow_outflow"]()
    a, b = _context(case), _context(case)
    for s in range(3):
        a.step(precision=0, rtol=1e-10)
        b.step(precision=0, rtol=1e-10, graph=1)
    nv = case.nvert.copy()
    nv[5:7, 4:6, 6:9] = 3.0
    for ctx in (a, b):
        ctx.set_field(vfs.NVERT, nv)
    for s in range(3):
        sa = a.step(precision=0, rtol=1e-10)
        sb = b.step(precision=0, rtol=1e-10, graph=1)
        assert sa.poisson.iterations == sb.poisson.iterations
    for f in (vfs.UCONT, vfs.UCAT, vfs.P):
        np.testing.assert_array_equal(b.get_field(f), a.get_field(f))
    a.close()
    b.close()
