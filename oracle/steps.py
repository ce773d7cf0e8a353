"""Physical time steps of the reference (oracle/_ref), phase by phase.

TEST INFRASTRUCTURE ONLY: used by tests/ (multi-step parity) and bench.py's CPU baseline
and reference arm.  Never part of the product path.

One step follows the reference's time loop (main.c:3534-3602) around Flow_Solver for
implicit = 0 (solvers.c:562-1390): on the first step the IB-node interpolation and IB_BC
(solvers.c:603-611); Calc_k_Flux, the eddy viscosity when les is on (solvers.c:648-654),
Pressure_Gradient, RungeKutta; VolumeFlux, PoissonRHS2_hypre, the Poisson solve,
Remove_Nullspace, Convert_Phi2_Phi (poisson_hypre.c:498-620); UpdatePressure, Projection,
the IB-node interpolation, IB_BC, Contra2Cart; then the old-value copies of the time
loop.  Every call is the reference's own function, except the Poisson solve: HYPRE is not
in this image, so oracle.poisson_mg solves the reference's own CSR system (set up once,
as HYPRE's set-up runs at PoissonLHSNew time, poisson_hypre.c:527), starting from the
previous solution like the reference's persistent Phi2.
"""
import time

from oracle import ref, poisson_mg


class ReferenceStepper:
    """Drives a Reference (oracle.ref) through time steps; `step` returns the wall time
    of its three phases: momentum (Calc_k_Flux .. RungeKutta), poisson (VolumeFlux ..
    Convert_Phi2_Phi) and correction (UpdatePressure .. the end-of-step copies)."""

    def __init__(self, R, rtol=1e-13):
        self.R = R
        self.case = R.case
        self.rtol = rtol
        self.ti = 0
        self.phi2 = None
        self.history = []
        self._lhs()

    def _lhs(self):
        """PoissonLHSNew and the solver's set-up: once, or every step with moving bodies
        (poisson_hypre.c:540-553).  Run as at ti == tistart, when setup_lidx2 numbers the
        unknowns into fresh vectors (poisson.c:207-282)."""
        R, c = self.R, self.case
        ref.set_global("ti", 0)
        R.call("ref_poisson_lhs")
        ref.set_global("ti", self.ti)
        rp, col, val = R.poisson_csr()
        self.solver = poisson_mg.MGSolver(rp, col, val, R.gid(), (c.i_periodic, c.j_periodic, c.k_periodic))

    def _ibm_interpolation(self):
        """ibm_interpolation_advanced (its wall model applies from ti > 0, ibm.c:3456)."""
        self.R.call("ref_ibm_interpolation", 1)

    def step(self):
        """One time step with the reference's ti set to the step index (les.c:69 and the
        wall model of ibm.c:3456 read it)."""
        R, case = self.R, self.case
        ref.set_global("ti", self.ti)
        t0 = time.perf_counter()
        if self.ti > 0 and getattr(case, "moving", 0):
            self._lhs()
            self.phi2 = None          # the unknowns are numbered anew (setup_lidx2)
        if self.ti == 0:
            if case.immersed:
                self._ibm_interpolation()             # solvers.c:607
            R.call("ref_ib_bc")                       # solvers.c:609
            R.set("Ucont", R.get("lUcont"))
        R.call("ref_calc_k_flux")                     # solvers.c:644
        if case.les:                                  # solvers.c:648-654
            R.call("ref_contra2cart")
            R.call("ref_les", 1)                      # dynamic_freq = 1: every step
        R.call("ref_pressure_gradient")               # solvers.c:786
        R.call("ref_runge_kutta")                     # solvers.c:1294
        t1 = time.perf_counter()
        if case.immersed:
            R.volume_flux_ibm()                       # poisson_hypre.c:564
        else:
            R.volume_flux()                           # poisson_hypre.c:566
        b = R.poisson_rhs_hypre()                     # poisson_hypre.c:568
        x, it, rr = self.solver.solve(b, x0=self.phi2, rtol=self.rtol)
        self.phi2 = x.copy()
        x = R.remove_nullspace(x)                     # poisson_hypre.c:602
        R.set("Phi2", x)
        R.call("ref_convert_phi2_phi")                # poisson_hypre.c:610
        t2 = time.perf_counter()
        R.call("ref_update_pressure")                 # solvers.c:1341
        R.call("ref_projection")                      # solvers.c:1342
        if case.immersed:
            self._ibm_interpolation()                 # solvers.c:1368
        R.call("ref_ib_bc")                           # solvers.c:1381
        R.set("Ucont", R.get("lUcont"))
        R.call("ref_contra2cart")                     # solvers.c:1385
        R.call("ref_end_of_step")                     # main.c:3571-3602
        t3 = time.perf_counter()
        self.history.append({"poisson_iterations": it, "poisson_relres": rr})
        self.ti += 1
        ref.set_global("ti", 0)
        return {"momentum": t1 - t0, "poisson": t2 - t1, "correction": t3 - t2}

    def fields(self):
        R = self.R
        return {"P": R.get("P"), "Ucont": R.get("lUcont"), "Ucat": R.get("Ucat")}
