"""The oracle library (the reference's own sources under the single-rank shim) builds,
reads synthetic grid.dat/bcs.dat through MG_Initial, and runs the hot-path functions."""
import numpy as np
import pytest

from oracle import ref
from helpers import small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def test_metrics_of_a_cartesian_channel():
    c = small_channel(8, 6, 10)
    R = ref.Reference(c)
    m = R.metrics()
    aj = m["aj"][1:-1, 1:-1, 1:-1]
    # aj is the inverse cell volume (metrics.c:186-252)
    dx = np.diff(c.X[0, 0, :])[None, None, :]
    dy = np.diff(c.Y[0, :, 0])[None, :, None]
    dz = np.diff(c.Z[:, 0, 0])[:, None, None]
    np.testing.assert_allclose(aj, 1.0 / (dx * dy * dz), rtol=1e-12)
    R.close()


def test_contra2cart_recovers_a_uniform_flow():
    c = small_channel(8, 6, 10)
    R = ref.Reference(c)
    m = R.metrics()
    u = np.zeros(R.shape + (3,))
    u[..., 2] = 1.0
    uc = np.zeros(R.shape + (3,))
    uc[..., 2] = m["kzet"][..., 2]
    R.set("Ucont", uc); R.set("lUcont", uc)
    R.call("ref_contra2cart")
    got = R.get("Ucat")[1:-1, 1:-1, 1:-1]
    np.testing.assert_allclose(got[..., 2], 1.0, rtol=1e-12)
    np.testing.assert_allclose(got[..., :2], 0.0, atol=1e-12)
    R.close()


def test_poisson_matrix_rows_sum_to_zero_in_the_interior():
    """PoissonLHSNew builds a Neumann Laplacian: away from walls each row sums to zero."""
    c = small_channel(8, 6, 10)
    R = ref.Reference(c)
    R.call("ref_poisson_lhs")
    rp, col, val = R.poisson_csr()
    sums = np.array([val[rp[r]:rp[r + 1]].sum() for r in range(len(rp) - 1)])
    assert np.abs(sums).max() < 1e-12 * np.abs(val).max()
    R.close()


def test_cylinder_flags_are_zero_one_three():
    c = small_cylinders()
    vals = set(np.unique(c.nvert).tolist())
    assert vals == {0.0, 1.0, 3.0}
