"""Multi-step parity on two workloads of their own size: the B200 step repeated against the
reference's step (oracle/_ref) repeated from the same inputs (tests/multistep.py).

* 64^3 periodic channel, 10 FP64 steps at dt = 1e-3: the reference is run
  here, and P, Ucont and Ucat are compared over the whole DA grid.
* 128x96x128 wavy-wall channel with the immersed 20480-triangle sphere and dynamic
  Smagorinsky LES, 20 steps: the reference's 20 steps take minutes on one core,
  so its result is a committed fixture (tests/golden/make_multistep.py): the fields at
  20000 seeded points, plane sums and global norms, compared with the same quantities of
  the device run.

Contract: velocity and pressure within 1e-10 relative to their largest magnitude (the
FP64 path, and the mixed path at the same tolerance); every step divergence free to 1e-8.
"""
import os

import numpy as np
import pytest

from oracle import ref
from helpers import assert_close, report
import multistep

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE2 = os.path.join(HERE, "golden", "multistep_wavy_sphere_les_128x96x128.npz")


@pytest.fixture(scope="module")
def channel_64_reference():
    run = multistep.ReferenceRun(multistep.channel_64())
    for _ in range(10):
        run.step()
    out = run.fields()
    yield run, out
    run.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [1, 0, 2])
def test_channel_64_ten_steps_match_reference(channel_64_reference, precision):
    run, want = channel_64_reference
    ctx, stats = multistep.device_run(run.case, run.m, run.u0, run.uc0, 10, precision=precision)
    for s, st in enumerate(stats):
        assert st.poisson.converged == 1, s
        assert st.max_div < 1e-8, (s, st.max_div)
    import vfs_b200 as vfs
    assert_close(ctx.get_field(vfs.P), want["P"], rtol=1e-10, atol_frac=0, what="P after 10 steps")
    assert_close(ctx.get_field(vfs.UCONT), want["Ucont"], rtol=1e-10, atol_frac=0, what="Ucont after 10 steps")
    assert_close(ctx.get_field(vfs.UCAT), want["Ucat"], rtol=1e-10, atol_frac=0, what="Ucat after 10 steps")
    report("max_div of the last step", stats[-1].max_div)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(FIXTURE2), reason="the 128x96x128 LES fixture is not generated")
@pytest.mark.parametrize("precision", [1, 0])
def test_wavy_sphere_les_twenty_steps_match_reference_fixture(precision):
    import vfs_b200 as vfs
    fx = np.load(FIXTURE2)
    case, body = multistep.wavy_sphere_les()
    nsteps = int(fx["nsteps"])
    # the reference's metrics are those FormMetrics gives bit for bit on the device
    ctx0 = vfs.Context(case.config())
    ctx0.form_metrics(case.X, case.Y, case.Z)
    m = {k: ctx0.get_field(f) for k, f in vfs.METRIC_FIELDS.items()}
    ctx0.close()
    u0 = multistep.cases.initial_ucat(case)
    uc0 = multistep.cases.ucont_from_ucat(case, u0, m)
    ctx, stats = multistep.device_run(case, m, u0, uc0, nsteps, precision=precision, body=body)
    np.testing.assert_array_equal(ctx.get_field(vfs.NVERT).ravel()[fx["idx"]], fx["nvert"])
    for s, st in enumerate(stats):
        assert st.poisson.converged == 1, s
        assert st.max_div < 1e-8, (s, st.max_div)
    idx = fx["idx"]
    for name, fid in (("P", vfs.P), ("Ucont", vfs.UCONT), ("Ucat", vfs.UCAT)):
        got = ctx.get_field(fid)
        flat = got.reshape(-1) if got.ndim == 3 else got.reshape(-1, 3)
        want = fx[name + "_pts"]
        scale = float(fx[name + "_max"])
        err = np.abs(flat[idx] - want).max() / scale
        report(name + " at 20000 points after %d steps" % nsteps, err)
        assert err <= 1e-10, (name, err)
        # plane sums along k and the global maximum
        planes = got.sum(axis=(1, 2))
        perr = np.abs(planes - fx[name + "_planes"]).max() / np.abs(fx[name + "_planes"]).max()
        report(name + " k-plane sums", perr)
        assert perr <= 1e-10, (name, perr)
        assert abs(np.abs(got).max() - scale) <= 1e-10 * scale
    ctx.close()
