"""The oracle library runs every reference call sequence the GPU parity tests use, in one
process and in the same order (several reference set-ups in a row), on the CPU.  This
keeps the oracle itself sound before any GPU run: a fault in the shim-compiled reference
shows up here, on the CPU."""
import numpy as np
import pytest

from oracle import ref
from vfs_b200 import cases
import helpers

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _ref_state(case, les_nut=False, seed=0):
    R = ref.Reference(case)
    m, u, uc = helpers.seeded_state(case, R, seed)
    for n in ("Ucont", "lUcont", "Ucont_o", "lUcont_o"):
        R.set(n, uc)
    for n in ("Ucat", "lUcat", "lUcat_old"):
        R.set(n, u)
    rng = np.random.Generator(np.random.Philox(seed + 17))
    p = rng.standard_normal(R.shape) * 0.1
    R.set("P", p)
    R.set("lP", p)
    if les_nut:
        R.set("lNu_t", rng.random(R.shape) * 1e-3)
    return R


def test_step_sequences():
    import test_step_gpu as S
    for name in S.STEP_CASES:
        case = S.STEP_CASES[name]()
        case.inlet_flux = 5.0
        R = _ref_state(case)
        ref.set_global("inlet_flux", 5.0)
        S.reference_step(R)
        assert np.isfinite(R.get("P")).all()
        R.close()
    for name in ("wavy", "cylinders"):
        case = S.STEP_CASES[name]()
        case.les = 2
        case.inlet_flux = 5.0
        R = _ref_state(case, les_nut=True)
        ref.set_global("inlet_flux", 5.0)
        S.reference_les_step(R, 2)
        assert R.get("lCs").max() > 0
        R.close()


def test_inlet_outlet_sequences():
    import test_inlet_outlet_gpu as T
    from test_step_gpu import reference_step
    for rep in range(2):
        for name in T.NAMES + ["cylinders1"]:
            case = T._case(name)
            R = _ref_state(case)
            ref.set_global("inlet_flux", 0.8 * R.inlet_area())
            if case.inletprofile == 100:
                R.set_inflow_plane(cases.inflow_plane(case))
            R.call("ref_inflow_flux")
            R.call("ref_form_bcs_scaled", 1)
            if rep == 1:
                reference_step(R)
            R.close()


def test_les_and_ibm_sequences():
    for name in ("channel", "wavy", "cylinders"):
        case = {"channel": lambda: helpers.small_channel(), "wavy": lambda: helpers.small_channel(wavy=0.15),
                "cylinders": lambda: helpers.small_cylinders()}[name]()
        case.les = 2
        R = ref.Reference(case, extra_globals={"ti": 5, "tistart": 0})
        m, u, uc = helpers.seeded_state(case, R, 0)
        for n in ("Ucont", "lUcont"):
            R.set(n, uc)
        for n in ("Ucat", "lUcat", "lUcat_old"):
            R.set(n, u)
        R.call("ref_contra2cart")
        R.call("ref_les", 1)
        R.close()
    ref.set_global("ti", 0)
    for size, level in (((24, 20, 28), 3), ((40, 32, 48), 3)):
        case = cases.channel(*size, wavy=0.1)
        R = ref.Reference(case)
        nv = R.ibm_classify(*cases.icosphere((np.pi / 2, 1.0, np.pi), 0.4, level=level))
        assert (nv == 3).sum() > 0
        R.close()


def test_immersed_sequences():
    """The IB-node list, interpolation, immersed VolumeFlux and a whole immersed step, as
    test_ibm_gpu.py and test_step_gpu.py run them."""
    import test_step_gpu as S
    for size, level, radius in (((24, 20, 28), 3, 0.4), ((48, 40, 56), 4, 0.35)):
        case = cases.channel(*size, wavy=0.1)
        case.immersed = 1
        R = _ref_state(case)
        R.ibm_classify(*cases.icosphere((np.pi / 2, 1.0, np.pi), radius, level=level), build_list=True)
        ints, dbls = R.ibm_list()
        assert len(ints) > 50 and (ints[:, 4] >= 0).all()
        R.call("ref_ibm_interpolation", 1)
        flux, area = R.volume_flux_ibm()
        assert area > 0 and np.isfinite(flux)
        R.close()
    case = helpers.small_channel(16, 14, 20, wavy=0.1)
    case.immersed = 1
    case.inlet_flux = 5.0
    R = _ref_state(case)
    R.ibm_classify(*cases.icosphere((np.pi / 2, 1.0, np.pi), 0.45, level=3), build_list=True)
    ref.set_global("inlet_flux", 5.0)
    S.reference_immersed_step(R)
    assert np.isfinite(R.get("P")).all()
    R.close()
