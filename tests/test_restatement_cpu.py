"""The C restatement oracle (oracle/vfs_oracle.c) pinned against the reference's own
functions (oracle/_ref) on the same inputs: pointwise operators bit for bit, the
divergence maximum exactly, the Poisson operator entry by entry."""
import numpy as np
import pytest

from oracle import ref, restatement
from vfs_b200 import cases
from helpers import small_channel, small_cylinders

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

CASES = {
    "channel": lambda: small_channel(),
    "wavy": lambda: small_channel(wavy=0.15),
    "cylinders": lambda: small_cylinders(),
}


def _state(name, les=False):
    case = CASES[name]()
    if les:
        case.les = 2
    R = ref.Reference(case)
    m = R.metrics()
    u = cases.initial_ucat(case)
    uc = cases.ucont_from_ucat(case, u, m)
    for n in ("Ucont", "lUcont"):
        R.set(n, uc)
    for n in ("Ucat", "lUcat", "lUcat_old"):
        R.set(n, u)
    rng = np.random.Generator(np.random.Philox(7))
    p = rng.standard_normal(R.shape) * 0.1
    R.set("P", p)
    R.set("lP", p)
    nut = rng.random(R.shape) * 1e-3 if les else None
    if les:
        R.set("lNu_t", nut)
    return case, R, restatement.State(case, m, uc, u, p=p, nut=nut)


@pytest.mark.parametrize("name", list(CASES))
def test_form_metrics(name):
    case = CASES[name]()
    R = ref.Reference(case)
    got = restatement.form_metrics(case)
    for k, v in ref.METRIC_VECS.items():
        np.testing.assert_array_equal(got[k], R.get(v), err_msg=k)
    R.close()


@pytest.mark.parametrize("name,les", [("channel", False), ("wavy", False), ("cylinders", False),
                                      ("wavy", True), ("cylinders", True)])
def test_contra2cart_and_formfunction2(name, les):
    case, R, st = _state(name, les)
    R.call("ref_contra2cart")
    restatement.contra2cart(st)
    np.testing.assert_array_equal(st.ucat, R.get("Ucat"))
    R.set("Rhs", np.zeros(R.shape + (3,)))
    R.call("ref_formfunction2", 1.0)
    rhs = restatement.formfunction2(st, 1.0)
    np.testing.assert_array_equal(rhs, R.get("Rhs"))
    R.close()


@pytest.mark.parametrize("name", list(CASES))
def test_pressure_gradient(name):
    case, R, st = _state(name)
    R.set_kflux(0.37, 1.9)
    ref.set_global("inlet_flux", 0.25)
    R.call("ref_pressure_gradient")
    dp = restatement.pressure_gradient(st, kforce=2, kdiff=0.37 - 0.25, karea=1.9)
    np.testing.assert_array_equal(dp, R.get("dP"))
    R.close()


@pytest.mark.parametrize("name", list(CASES))
def test_poisson_operator_rhs_projection(name):
    case, R, st = _state(name)
    R.call("ref_poisson_lhs")
    rp, col, val = R.poisson_csr()
    gid = R.gid()
    inner = np.zeros(R.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    own = (gid >= 0) & inner
    coef = restatement.poisson_lhs(st)
    # every reference matrix entry equals the restatement's coefficient for that column
    lin = np.flatnonzero(own.reshape(-1))
    row_of = gid.reshape(-1)[lin]
    cell_of_row = np.empty(len(rp) - 1, dtype=np.int64)
    cell_of_row[row_of] = lin
    off = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (1, -1, 0),
           (-1, 1, 0), (-1, -1, 0), (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1), (1, 0, 1), (1, 0, -1),
           (-1, 0, 1), (-1, 0, -1)]
    mz, my, mx = R.shape
    per = (case.i_periodic, case.j_periodic, case.k_periodic)

    def wrap(v, m, p):
        if p and v == 0:
            return m - 2
        if p and v == m - 1:
            return 1
        return v
    for r in range(len(rp) - 1):
        cell = cell_of_row[r]
        k, rem = divmod(cell, mx * my)
        j, i = divmod(rem, mx)
        mine = {}
        for s, (a, b, c) in enumerate(off):
            v = coef[s].reshape(-1)[cell]
            if v != 0.0 or s == 0:
                ii, jj, kk = wrap(i + a, mx, per[0]), wrap(j + b, my, per[1]), wrap(k + c, mz, per[2])
                mine[int(gid[kk, jj, ii])] = v
        theirs = {int(cc): vv for cc, vv in zip(col[rp[r]:rp[r + 1]], val[rp[r]:rp[r + 1]])}
        assert mine == theirs, (r, (i, j, k))
    b = R.poisson_rhs_hypre()
    want = np.zeros(R.shape)
    want[own] = b[gid[own]]
    got = restatement.poisson_rhs(st)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())
    # projection with the same Phi
    rng = np.random.Generator(np.random.Philox(3))
    phi2 = rng.standard_normal(len(rp) - 1) * 1e-2
    R.set("Phi2", phi2)
    R.call("ref_convert_phi2_phi")
    phi = R.get("Phi")
    R.call("ref_update_pressure")
    restatement.update_pressure(st, phi)
    np.testing.assert_array_equal(st.p, R.get("P"))
    R.call("ref_projection")
    restatement.projection(st, phi)
    np.testing.assert_array_equal(st.ucont, R.get("Ucont"))
    R.close()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("les,ti", [(2, 5), (2, 1), (1, 5)])
def test_dynamic_smagorinsky(name, les, ti):
    """Cs and nu_t of the dynamic model (and its fixed-value branches) bit for bit."""
    case, R, st = _state(name, les=True)
    st.g.les = les
    ref.set_global("les", les)
    ref.set_global("ti", ti)
    ref.set_global("tistart", 0)
    R.call("ref_contra2cart")
    restatement.contra2cart(st)
    R.call("ref_les", 1)
    cs = restatement.les(st, ti=ti)
    if les == 2 and ti >= 2:
        assert cs.max() > 0.0
    np.testing.assert_array_equal(cs, R.get("lCs"))
    np.testing.assert_array_equal(st.nut, R.get("lNu_t"))
    R.close()
