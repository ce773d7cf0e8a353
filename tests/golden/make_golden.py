"""Writes the golden fixtures of the projection path: inputs and the reference's own
outputs for two small cases, produced by the reference sources compiled under the
single-rank PETSc shim (oracle/_ref, built by oracle/build_ref.py from the reference
tree).  Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (compressed .npz, float64):
  wavy_channel_12x10x14.npz  wavy-bottom channel, periodic i and k, walls in j
  cylinders_16x12x24.npz     open channel with blocked cylinders (nvert 0/1/3)

Each holds the grid nodes (X, Y, Z), nvert, the seeded inputs (ucat, ucont, p, rhs0,
phi) and the reference outputs:
  ucat_c2c     Contra2Cart (rhs.c:27)
  rhs_ff2      Formfunction_2(user, Rhs, 0.75) (momentum.c:456) added to rhs0
  cs_les, nut_les  Compute_Smagorinsky_Constant_1 + Compute_eddy_viscosity_LES (les.c:67,
               les.c:1135) with les = 2 at ti = 5 on ucat_c2c, lNu_t starting from nut0
  dp, p_pg     Pressure_Gradient (momentum.c:197) with mean k flux 0.37, area 1.9
  b            PoissonRHS2_hypre + Remove_Nullspace_Scale on the grid layout
  ax           the PoissonLHSNew operator applied to a seeded x (x also stored)
  p_up, ucont_proj, ucat_proj   UpdatePressure and Projection for the stored phi
and, for the wavy channel, the metrics of FormMetrics (metrics.c:4).

ibm_sphere_wavy_24x20x28.npz holds a triangulated sphere and the nvert flags that the
reference's ray test (point_cell_advanced, ibm.c:1068) gives it in the wavy channel.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vfs-geophysics-3.1_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import ref  # noqa: E402
from vfs_b200 import cases  # noqa: E402
from golden_cases import FIXTURES  # noqa: E402


def fixture_path(name):
    return os.path.join(HERE, name + ".npz")


def _csr_apply(R, x_grid):
    rp, col, val = R.poisson_csr()
    gid = R.gid()
    n = len(rp) - 1
    inner = np.zeros(R.shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    m = (gid >= 0) & inner
    xc = np.zeros(n)
    xc[gid[m]] = x_grid[m]
    y = np.zeros(n)
    for r in range(n):
        y[r] = np.dot(val[rp[r]:rp[r + 1]], xc[col[rp[r]:rp[r + 1]]])
    out = np.zeros(R.shape)
    out[m] = y[gid[m]]
    return out, m


def make(name):
    case = FIXTURES[name]()
    R = ref.Reference(case)
    d = {"X": case.X, "Y": case.Y, "Z": case.Z, "nvert": np.asarray(case.nvert, dtype=np.float64)}
    m = R.metrics()
    u = cases.initial_ucat(case, seed=0)
    uc = cases.ucont_from_ucat(case, u, m)
    rng = np.random.Generator(np.random.Philox(17))
    p = rng.standard_normal(R.shape) * 0.1
    for n in ("Ucont", "lUcont", "Ucont_o", "lUcont_o"):
        R.set(n, uc)
    for n in ("Ucat", "lUcat", "lUcat_old"):
        R.set(n, u)
    R.set("P", p)
    R.set("lP", p)
    d.update(ucat=u, ucont=uc, p=p)
    if name.startswith("wavy"):
        for k, v in m.items():
            d["metric_" + k] = v
    # Contra2Cart, then Formfunction_2 on its Ucat
    R.call("ref_contra2cart")
    d["ucat_c2c"] = R.get("Ucat")
    rhs0 = np.random.Generator(np.random.Philox(5)).standard_normal(R.shape + (3,))
    d["rhs0"] = rhs0
    R.set("Rhs", rhs0)
    R.call("ref_formfunction2", 0.75)
    d["rhs_ff2"] = R.get("Rhs")
    # dynamic Smagorinsky model on the Contra2Cart velocity (les = 2, ti = 5)
    nut0 = np.random.Generator(np.random.Philox(23)).random(R.shape) * 1e-3
    R.set("lNu_t", nut0)
    ref.set_global("les", 2)
    ref.set_global("ti", 5)
    ref.set_global("tistart", 0)
    R.call("ref_les", 1)
    d["nut0"] = nut0
    d["cs_les"] = R.get("lCs")
    d["nut_les"] = R.get("lNu_t")
    ref.set_global("les", case.les)
    ref.set_global("ti", 0)
    # Pressure_Gradient
    R.set_kflux(0.37, 1.9)
    ref.set_global("inlet_flux", 0.25)
    R.call("ref_pressure_gradient")
    d["dp"] = R.get("dP")
    d["p_pg"] = R.get("P")
    # Poisson operator and right-hand side
    R.call("ref_poisson_lhs")
    x = np.random.Generator(np.random.Philox(11)).standard_normal(R.shape)
    ax, mask = _csr_apply(R, x)
    x[~mask] = 0.0
    d["x"] = x
    d["ax"] = ax
    bc = R.poisson_rhs_hypre()
    gid = R.gid()
    b = np.zeros(R.shape)
    b[mask] = bc[gid[mask]]
    d["b"] = b
    # UpdatePressure and Projection for a seeded Phi
    phi2 = np.random.Generator(np.random.Philox(3)).standard_normal(len(bc)) * 1e-2
    R.set("Phi2", phi2)
    R.call("ref_convert_phi2_phi")
    d["phi"] = R.get("Phi")
    d["p_before_up"] = R.get("P")
    d["ucont_before_proj"] = R.get("lUcont")
    d["ucat_before_proj"] = R.get("Ucat")
    R.call("ref_update_pressure")
    d["p_up"] = R.get("P")
    R.call("ref_projection")
    d["ucont_proj"] = R.get("lUcont")
    d["ucat_proj"] = R.get("Ucat")
    R.close()
    np.savez_compressed(fixture_path(name), **d)
    return fixture_path(name)


def make_ibm(name="ibm_sphere_wavy_24x20x28"):
    """nvert of an icosphere (1280 triangles, centre (pi/2, 1, pi), radius 0.4) in the wavy
    channel, classified by the reference's own ray test (ref_ibm_classify)."""
    case = cases.channel(24, 20, 28, wavy=0.1)
    case.immersed = 1
    R = ref.Reference(case)
    x, y, z, tri = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.4, level=3)
    nv = R.ibm_classify(x, y, z, tri)
    R.close()
    np.savez_compressed(fixture_path(name), X=case.X, Y=case.Y, Z=case.Z, sx=x, sy=y, sz=z, tri=tri, nvert=nv)
    return fixture_path(name)


if __name__ == "__main__":
    if not ref.available():
        sys.exit("oracle/_ref is not built (python oracle/build_ref.py)")
    for n in FIXTURES:
        print(make(n), os.path.getsize(fixture_path(n)))
    print(make_ibm(), os.path.getsize(fixture_path("ibm_sphere_wavy_24x20x28")))
