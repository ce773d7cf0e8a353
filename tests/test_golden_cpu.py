"""The C restatement oracle (oracle/vfs_oracle.c) against the committed golden fixtures
(tests/golden/*.npz, outputs of the reference's own functions; see
tests/golden/make_golden.py).  Needs no reference build: this pins the oracle wherever
the tests run."""
import os

import numpy as np
import pytest

from oracle import restatement
from conftest import ROOT
from golden_cases import FIXTURES, load

NAMES = list(FIXTURES)


def _state(name):
    case, d = load(name)
    if "metric_csi" in d:
        m = {k[len("metric_"):]: d[k] for k in d if k.startswith("metric_")}
    else:
        m = restatement.form_metrics(case)
    st = restatement.State(case, m, d["ucont"], d["ucat"], p=d["p"])
    return case, d, m, st


def test_fixture_metrics_match_the_restatement():
    case, d = load("wavy_channel_12x10x14")
    got = restatement.form_metrics(case)
    for k in got:
        np.testing.assert_array_equal(got[k], d["metric_" + k], err_msg=k)


@pytest.mark.parametrize("name", NAMES)
def test_contra2cart_formfunction2(name):
    case, d, m, st = _state(name)
    restatement.contra2cart(st)
    np.testing.assert_array_equal(st.ucat, d["ucat_c2c"])
    rhs = restatement.formfunction2(st, 0.75, rhs=d["rhs0"])
    np.testing.assert_array_equal(rhs, d["rhs_ff2"])


@pytest.mark.parametrize("name", NAMES)
def test_pressure_gradient(name):
    case, d, m, st = _state(name)
    dp = restatement.pressure_gradient(st, kforce=2, kdiff=0.37 - 0.25, karea=1.9)
    np.testing.assert_array_equal(dp, d["dp"])


@pytest.mark.parametrize("name", NAMES)
def test_poisson_operator_rhs(name):
    case, d, m, st = _state(name)
    coef = restatement.poisson_lhs(st)
    ax = restatement.poisson_apply(st, coef, d["x"])
    scale = np.abs(d["ax"]).max()
    assert np.abs(ax - d["ax"]).max() <= 1e-14 * scale
    b = restatement.poisson_rhs(st)
    assert np.abs(b - d["b"]).max() <= 1e-12 * np.abs(d["b"]).max()


@pytest.mark.parametrize("name", NAMES)
def test_update_pressure_projection(name):
    case, d, m, st = _state(name)
    st.p = np.array(d["p_before_up"])
    st.ucont = np.array(d["ucont_before_proj"])
    phi = restatement.update_pressure(st, d["phi"])
    np.testing.assert_array_equal(st.p, d["p_up"])
    restatement.projection(st, phi)
    # interior and non-periodic ghosts: the local Ucont of the reference
    np.testing.assert_array_equal(st.ucont[1:-1, 1:-1, 1:-1], d["ucont_proj"][1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("name", NAMES)
def test_restatement_les_matches_fixture(name):
    """The C restatement of the dynamic Smagorinsky model reproduces the fixture's Cs and
    nu_t bit for bit (les = 2, ti = 5, on the Contra2Cart velocity)."""
    from oracle import restatement
    case, d = load(name)
    case.les = 2
    m = restatement.form_metrics(case)
    st = restatement.State(case, m, d["ucont"], d["ucat"], nut=d["nut0"])
    restatement.contra2cart(st)
    cs = restatement.les(st, ti=5)
    np.testing.assert_array_equal(cs, d["cs_les"])
    np.testing.assert_array_equal(st.nut, d["nut_les"])


def test_ibm_fixture_is_the_reference_classification():
    """The committed nvert fixture is what the reference's ray test gives (when oracle/_ref
    is built here), and holds solid and IB-node cells."""
    d = np.load(os.path.join(ROOT, "tests", "golden", "ibm_sphere_wavy_24x20x28.npz"))
    assert (d["nvert"] == 3).sum() > 0 and (d["nvert"] == 1).sum() > 0
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from vfs_b200 import cases
    case = cases.channel(24, 20, 28, wavy=0.1)
    case.immersed = 1
    R = ref.Reference(case)
    got = R.ibm_classify(d["sx"], d["sy"], d["sz"], d["tri"])
    R.close()
    np.testing.assert_array_equal(got, d["nvert"])
