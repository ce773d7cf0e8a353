"""Restart through the library: a run written to restart files with
vfs_restart_write and continued in a new context with vfs_restart_read gives the same
steps as the run that never stopped, and the reference's own Ucont_P_Binary_Input
(main.c:394) reads the files the library wrote."""
import tempfile

import numpy as np
import pytest

from oracle import ref
import vfs_b200 as vfs
from helpers import assert_close, small_channel
from vfs_b200 import cases

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _context(case, m):
    ctx = vfs.Context(case.config())
    ctx.set_metrics(m)
    ctx.set_field(vfs.NVERT, case.nvert)
    return ctx


@pytest.mark.gpu
@pytest.mark.parametrize("les", [0, 2])
def test_restart_continues_the_run(les):
    case = small_channel(16, 12, 18, wavy=0.1)
    case.les = les
    case.inlet_flux = 5.0
    R = ref.Reference(case)
    m = R.metrics()
    u = cases.initial_ucat(case)
    uc = cases.ucont_from_ucat(case, u, m)
    a = _context(case, m)
    a.set_field(vfs.UCONT, uc)
    a.set_field(vfs.UCAT, u)
    a.set_field(vfs.UCAT_O, u)
    a.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
    for _ in range(3):
        a.step(precision=1, rtol=1e-13)
    with tempfile.TemporaryDirectory() as d:
        a.restart_write(d, 3)
        b = _context(case, m)
        b.set_scalar(vfs.S_INLET_FLUX, case.inlet_flux)
        b.restart_read(d, 3)
        for f in (vfs.UCONT, vfs.UCAT, vfs.P):
            np.testing.assert_array_equal(b.get_field(f), a.get_field(f))
        # the reference reads the library's files into its own vectors
        R.restart_input(d, 3)
        np.testing.assert_array_equal(R.get("lUcont"), a.get_field(vfs.UCONT))
        np.testing.assert_array_equal(R.get("Ucat"), a.get_field(vfs.UCAT))
        np.testing.assert_array_equal(R.get("P"), a.get_field(vfs.P))
        if les:
            np.testing.assert_array_equal(R.get("lCs"), a.get_field(vfs.CS))
    sa = a.step(precision=1, rtol=1e-13)
    sb = b.step(precision=1, rtol=1e-13)
    assert sa.poisson.converged == 1 and sb.poisson.converged == 1
    # the restarted run solves its first Poisson system from zero (the reference's Phi2 is
    # fresh after a restart), so the two runs agree to the solve's tolerance
    for f, name in ((vfs.P, "P"), (vfs.UCONT, "Ucont"), (vfs.UCAT, "Ucat")):
        assert_close(b.get_field(f), a.get_field(f), rtol=1e-10, atol_frac=0, what=name + " after restart")
    a.close()
    b.close()
    R.close()
