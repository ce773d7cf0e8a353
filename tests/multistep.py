"""Several physical time steps of the reference (oracle/_ref) and of the B200 library
from the same inputs: the time loop of main.c:3534-3602 around Flow_Solver
(solvers.c:562-1390, implicit = 0).

The reference's steps are oracle.steps.ReferenceStepper's: the reference's own functions,
with its HYPRE solve replaced by oracle.poisson_mg (FGMRES + multigrid on the reference's
own CSR system, rtol 1e-13 or its rounding floor), started, like the reference's
persistent Phi2, from the previous solution.  Both sides start from the
seeded initial fields of vfs_b200.cases (P = 0, nu_t = 0, a fresh run: ti = tistart = 0).

Used by tests/test_multistep_gpu.py (64^3 channel, run live) and
tests/golden/make_multistep.py (the 128x96x128 wavy-wall sphere LES case, whose 20
reference steps take minutes on one core, committed as a fixture).
"""
import numpy as np

from oracle import ref, steps
from vfs_b200 import cases
import vfs_b200 as vfs


def channel_64():
    """The 64^3 periodic channel (streamwise k), tanh stretch beta = 2 in y,
    2pi x 2 x pi (x/z labels swapped so that k is streamwise), Re_b = 5600 (ren = 2800),
    laminar parabola + uniform noise 0.1 U_b (seed 0), dt = 1e-3, no immersed body, no LES."""
    c = cases.channel(64, 64, 64)
    c.inlet_flux = -1.0
    return c


def wavy_sphere_les(nx=128, ny=96, nz=128, level=5):
    """The 128 x 96 x 128 channel mapping with the sinusoidal bottom wall
    y_w = 0.1 sin(2 pi x/Lx) cos(2 pi z/Lz), an immersed sphere of diameter 0.4 at the
    domain centre (icosphere of 20 * 4**level triangles; level 5 = 20480), dynamic
    Smagorinsky LES (les = 2), Re = 1e4, FP64, dt = 1e-3."""
    c = cases.channel(nx, ny, nz, wavy=0.1)
    c.immersed = 1
    c.les = 2
    c.ren = 1e4
    body = cases.icosphere((np.pi / 2, 1.0, np.pi), 0.2, level=level)
    return c, body


class ReferenceRun:
    """The reference's functions driven through N time steps (oracle.steps)."""

    def __init__(self, case, body=None, rtol=1e-13):
        self.case = case
        R = ref.Reference(case, extra_globals={"dynamic_freq": 1})
        self.R = R
        if body is not None:
            R.ibm_classify(*body, build_list=True)
            R.call("ref_calc_inlet_area")          # main.c:3488, after the IB search
        self.m = R.metrics()
        u = cases.initial_ucat(case)
        uc = cases.ucont_from_ucat(case, u, self.m)
        self.u0, self.uc0 = u, uc
        for n in ("Ucont", "lUcont", "Ucont_o", "lUcont_o"):
            R.set(n, uc)
        for n in ("Ucat", "lUcat", "lUcat_old"):
            R.set(n, u)
        self.stepper = steps.ReferenceStepper(R, rtol=rtol)
        self.history = self.stepper.history

    def step(self):
        self.stepper.step()

    def fields(self):
        return self.stepper.fields()

    def close(self):
        self.R.close()


def device_run(case, m, u0, uc0, nsteps, precision=1, body=None, rtol=1e-13):
    """The same steps on the B200 library; returns (context, per-step stats)."""
    ctx = vfs.Context(case.config())
    ctx.set_metrics(m)
    ctx.set_field(vfs.NVERT, case.nvert)
    if body is not None:
        ctx.ibm_search(*body)
    ctx.set_field(vfs.UCONT, uc0)
    ctx.set_field(vfs.UCAT, u0)
    ctx.set_field(vfs.UCAT_O, u0)
    stats = [ctx.step(precision=precision, rtol=rtol) for _ in range(nsteps)]
    return ctx, stats


def sample_points(shape, n, seed=1234):
    """n seeded DA points (flat indices) for the fixture's point samples."""
    rng = np.random.Generator(np.random.Philox(seed))
    return np.sort(rng.choice(int(np.prod(shape)), size=n, replace=False))
