"""Shared set-up for the parity tests: one synthetic case, the reference state built by
the oracle library, and the same inputs uploaded to the B200 library."""
import numpy as np

from oracle import ref
from vfs_b200 import cases
import vfs_b200 as vfs

DA_METRIC_NAMES = ("csi", "eta", "zet", "aj", "icsi", "ieta", "izet", "iaj", "jcsi", "jeta",
                   "jzet", "jaj", "kcsi", "keta", "kzet", "kaj", "cent")


def small_channel(nx=12, ny=10, nz=14, wavy=0.0):
    return cases.channel(nx, ny, nz, wavy=wavy)


def small_cylinders(nx=16, ny=12, nz=24):
    c = cases.open_channel_cylinders(nx, ny, nz, D=0.6, Lx=3.2, Lz=8.0, Ly=1.0)
    return c


def seeded_state(case, R, seed=0):
    """Velocity fields on both sides: Ucat from the seeded profile, Ucont from Ucat."""
    m = R.metrics()
    u = cases.initial_ucat(case, seed=seed)
    uc = cases.ucont_from_ucat(case, u, m)
    return m, u, uc


def build_pair(case, seed=0, les_nut=False, extra_globals=None):
    R = ref.Reference(case, extra_globals=extra_globals)
    m, u, uc = seeded_state(case, R, seed)
    for n in ("Ucont", "lUcont", "Ucont_o", "lUcont_o"):
        R.set(n, uc)
    for n in ("Ucat", "lUcat", "lUcat_old"):
        R.set(n, u)
    rng = np.random.Generator(np.random.Philox(seed + 17))
    p = rng.standard_normal(R.shape) * 0.1
    R.set("P", p)
    R.set("lP", p)
    nut = None
    if les_nut:
        nut = rng.random(R.shape) * 1e-3
        R.set("lNu_t", nut)
    ctx = vfs.Context(case.config())
    ctx.set_metrics(m)
    ctx.set_field(vfs.NVERT, case.nvert)
    ctx.set_field(vfs.UCONT, uc)
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    ctx.set_field(vfs.P, p)
    if nut is not None:
        ctx.set_field(vfs.NU_T, nut)
    return R, ctx


# Achieved errors of the parity tests, keyed "test id / quantity" (written out by
# conftest.py when VFS_PARITY_REPORT names a file).
REPORT = {}


def report(what, value):
    """Record an achieved error under the running test's id, and print it."""
    import os
    test = os.environ.get("PYTEST_CURRENT_TEST", "").split(" ")[0]
    REPORT["%s / %s" % (test, what)] = float(value)
    print("%s / %s: %.3e" % (test, what, value))


def assert_close(a, b, rtol=1e-12, atol_frac=1e-13, what=""):
    """max |a - b| <= (rtol + atol_frac) * max |b|; records the achieved max |a - b| / max |b|."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max()
    report(what + " max|diff|/max|ref|", err / scale)
    assert err <= atol_frac * scale + rtol * scale, "%s: max |diff| %.3e (scale %.3e)" % (what, err, scale)
    return err / scale
