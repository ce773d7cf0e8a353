"""Benchmark of the B200 projection step (one JSON line on stdout, rank 0).

Workload: the 256 x 192 x 256-cell open channel with a staggered 3 x 2 array of vertical
cylinders (D = 0.2, spacing 4D) encoded in nvert as blocked cells (immersed = 0), no-slip
bottom, free-slip top, spanwise periodic, an inlet on the k = 0 face (bctype 5, inflow
plane of inletprofile 100 rescaled to bulk velocity 1) and an outlet on the k+ face
(bctype 4, outflow rescaled to the inflow); seeded turbulent-like field (log-law mean plus
random Fourier modes with a k^-5/3 spectrum, 5 % intensity), whose first plane is the
inflow plane.  One step = Flow_Solver for implicit = 0: Calc_k_Flux, Pressure_Gradient,
4-stage RungeKutta (InflowFlux, FormBCS, stages, FormBCS with outlet rescaling),
VolumeFlux, Poisson RHS, Poisson solve to rtol 1e-10, UpdatePressure, Projection,
Divergence, IB_BC, Contra2Cart.

`value` is the mixed-precision (FP32 V-cycle in FP64 FGMRES) step time in ms with every
field resident in HBM; the all-FP64 form, and the form whose FGMRES basis is FP32 as well
(`vfs_solve_opts.precision` 2), are timed on the same state.
`e2e` runs the same step through the C ABI with the flow state (Ucont, Ucat, P) copied
from pinned host memory before and back after every step.

Multi-GPU: the projection path runs on one GPU (no sharding), so N GPUs run N
independent replicas (weak scaling); the step time is the maximum over ranks.

`--impl reference` times the reference's own CPU code (oracle/_ref: its momentum.c,
rhs.c, poisson.c ... under the single-rank shim; the Poisson solve, HYPRE in the
reference, is FGMRES with a geometric multigrid preconditioner on the reference's own
matrix, set up outside the step) on a 64x48x64 sample of the workload, and extrapolates
each phase (momentum, Poisson, correction) to the full grid with an exponent fitted over
three sample sizes; the line says "extrapolated" and carries the fit.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "vfs-geophysics-3.1_b200"))

METRIC = "ms/step @256x192x256: mixed vs FP64 GPU at max|div u|<=1e-8; adjoint/forward ratio"
# The mixed form of the metric: precision 0 (the V-cycle in FP32 inside FP64 FGMRES).  The
# other mixed form, precision 2 (the FGMRES basis, preconditioned vectors and V-cycle in
# FP32, every restart cycle an FP64 iterative-refinement sweep), is timed beside it; on this
# workload it takes about one FGMRES iteration more per step and is slower.
MIXED = 0
ALT = 2
NX, NY, NZ = 256, 192, 256
WORKLOAD = ("open channel 256x192x256 cells, 3x2 staggered cylinders D=0.2 spacing 4D as nvert "
            "blocked cells (immersed=0), no-slip bottom, free-slip top, periodic i, inlet k=0 "
            "(inletprofile 100: log-law + k^-5/3 Fourier-mode plane, bulk velocity 1), outlet k+ "
            "with flux rescaling; Poisson rtol 1e-10")
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null while the reference's C code runs (it prints
    progress lines with printf, e.g. poisson.c:262), so stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.libc.fflush(None)
        self.saved = os.dup(1)
        dn = os.open(os.devnull, os.O_WRONLY)
        os.dup2(dn, 1)
        os.close(dn)
        return self

    def __exit__(self, *a):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


# ------------------------------------------------------------------ workload
def make_case(nx=NX, ny=NY, nz=NZ):
    from vfs_b200 import cases
    c = cases.inflow_outflow(cases.open_channel_cylinders(nx, ny, nz), 100)
    c.immersed = 0
    return c


def turbulent_like(case, seed=0, intensity=0.05, ub=1.0):
    """Log-law mean streamwise velocity plus divergence-agnostic random Fourier modes with
    an E(k) ~ k^-5/3 spectrum in the periodic (x, z) plane, rms `intensity`*ub."""
    KM, JM, IM = case.X.shape
    nz, ny, nx = KM - 1, JM - 1, IM - 1
    Y = case.Y
    yc = 0.125 * sum(Y[a:KM - 1 + a, b:JM - 1 + b, c:IM - 1 + c] for a in (0, 1) for b in (0, 1) for c in (0, 1))
    H = getattr(case, "Ly", 1.0)
    yp = np.clip(yc / H, 1e-3, 1.0)
    mean = 1.0 + np.log(yp / 0.2) / 0.41 * 0.0566   # log law, u_tau = 0.0566 ub
    mean /= mean.mean()
    rng = np.random.Generator(np.random.Philox(seed))
    kx = np.fft.fftfreq(nx)[None, None, :]
    kz = np.fft.fftfreq(nz)[:, None, None]
    kk = np.sqrt(kx ** 2 + kz ** 2)
    amp = np.zeros_like(kk)
    amp[kk > 0] = kk[kk > 0] ** (-5.0 / 6.0 - 0.5)   # |u_k| ~ sqrt(E(k)/k) in 2-D
    u = np.zeros(case.da_shape + (3,))
    for comp in range(3):
        ph = rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))
        f = np.real(np.fft.ifft2(np.fft.fft2(ph, axes=(0, 2)) * amp, axes=(0, 2)))
        f *= intensity * ub / max(f.std(), 1e-30)
        u[1:-1, 1:-1, 1:-1, comp] = f
    u[1:-1, 1:-1, 1:-1, 2] += mean * ub
    u[case.nvert > 0.1] = 0.0
    return u


def setup_context(case):
    import vfs_b200 as vfs
    from vfs_b200 import cases
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    m = {"icsi": ctx.get_field(vfs.ICSI), "jeta": ctx.get_field(vfs.JETA), "kzet": ctx.get_field(vfs.KZET)}
    u = turbulent_like(case)
    uc = cases.ucont_from_ucat(case, u, m)
    ctx.set_field(vfs.UCONT, uc)
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    ctx.set_inflow_plane(u[1])
    _, inlet_area = ctx.calc_inlet_area()
    ctx.set_scalar(vfs.S_INLET_FLUX, 1.0 * inlet_area)   # bulk velocity 1
    ctx.contra2cart()
    del m, uc
    return ctx, u


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for q, n in enumerate(names):
            if any(len(r) > 5 + q and r[5 + q].lower().startswith("active") for r in self.rows):
                reasons.append(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------------ timing helpers
def timed(ctx, fn, reps, torch):
    """Device time of `reps` calls of fn, with events recorded on the context's stream."""
    s = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    e0.record(s)
    out = [fn() for _ in range(reps)]
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1), out


# Algorithmic bytes per interior cell of the profiled kernels (compulsory traffic: each
# input read once, each output written once, at the stored precision, nvert as 1 byte).
# DRAM bytes (read + write) per launch of the profiled kernels from one ncu capture at
# 128x96x128 cells, scaled by the cell ratio (x8) to 256x192x256 (profiles/
# formfunction2_128x96x128.md): Formfunction_2 as the step runs it (k_face_flux, k_fp,
# k_rhs) moved 1285.6 MB per launch there.
KERNEL_TRAFFIC = {"formfunction2": 1285.6e6 * 8}

KERNEL_BYTES = {
    # Formfunction_2 accumulating into Rhs (Formfunction_2(user, Rhs, scale) adds), les = 0
    # as in the workload (nu_t is not read): Ucont 24 + Ucat 24 + nvert 1 + face metrics 240
    # + centre metrics 72 + Rhs read 24 + Rhs write 24
    "formfunction2": 409.0,
    # FP64 Poisson apply with the 7 stored stencil slots (no cross terms on this grid):
    # coefficients 56 + phi 8 + mask 1 + y 8
    "poisson_apply_fp64": 73.0,
    # one zebra line-Gauss-Seidel sweep (both colours) of the finest multigrid level, FP32:
    # couplings +i/+j/+k 12 + Thomas factors 8 + b 4 + x read 4 + x write 4
    "smoother_fp32": 32.0,
    # the same sweep in FP64
    "smoother_fp64": 64.0,
    # Pressure_Gradient: P 8 + the nine face-metric products 72 + iaj, jaj, kaj 24 + nvert 1 + dP 24
    "pressure_gradient": 129.0,
    # UpdatePressure + Projection: Phi 8 + products 72 + face Jacobians 24 + nvert 1 + Ucont 24 + 24
    # + P 8 + 8
    "projection_update": 169.0,
    # Contra2Cart interior + Divergence maxima: Ucont 24 + centre metrics 72 + aj 8 + nvert 1 + Ucat 24
    "contra2cart_div": 129.0,
}


def mg_levels(nx, ny, nz):
    """Number of multigrid levels the solver builds for an nx x ny x nz-cell grid."""
    n = 1
    while nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0 and min(nx, ny, nz) >= 4:
        nx, ny, nz, n = nx // 2, ny // 2, nz // 2, n + 1
    return n


def roofline_probe(ctx, torch, reps=20):
    """Time the profiled operators on the context's stream; returns per-launch ms."""
    res = {}
    for name, ids in (("formfunction2", (8,)), ("poisson_apply_fp64", (3,)), ("smoother_fp32", (4,)),
                      ("smoother_fp64", (5,)), ("pressure_gradient", (12,)), ("projection_update", (13,)),
                      ("contra2cart_div", (14,)), ("vcycle_fp32", (9,)), ("vcycle_fp64", (10,))):
        for w in range(3):
            for i in ids:
                ctx.run_kernel(i, 1)
        def body():
            for i in ids:
                ctx.run_kernel(i, 1)
        ms, _ = timed(ctx, body, reps, torch)
        res[name] = ms / reps
    return res


# ------------------------------------------------------------------ reference arm
# The reference's own CPU code (oracle/_ref) cannot run the 256x192x256 workload within a
# bench run (a step there takes a few minutes on one core), so it runs on samples of the
# workload, grids of the same domain and bodies with fewer cells, and the step time is
# extrapolated phase by phase: each phase's cost is fitted as t = c * cells^a over three
# sample sizes, and the sample's phase times are scaled by (cells ratio)^a.
REF_SIZES = ((32, 24, 32), (64, 48, 64), (128, 96, 128))
REF_STEP_SIZE = (64, 48, 64)
PHASES = ("momentum", "poisson", "correction")


class ReferenceSample:
    """The reference's step (oracle/_ref via oracle.steps) on an nx x ny x nz sample of the
    workload; the Poisson set-up (PoissonLHSNew and the solver's set-up) is done here,
    outside the timed steps, as HYPRE's set-up runs at PoissonLHSNew time
    (poisson_hypre.c:527)."""

    def __init__(self, nx, ny, nz, seed=0, rtol=1e-10):
        from oracle import ref, steps
        from vfs_b200 import cases
        case = make_case(nx, ny, nz)
        R = ref.Reference(case)
        m = R.metrics()
        u = turbulent_like(case, seed=seed)
        uc = cases.ucont_from_ucat(case, u, m)
        for n in ("Ucont", "lUcont", "Ucont_o", "lUcont_o"):
            R.set(n, uc)
        for n in ("Ucat", "lUcat", "lUcat_old"):
            R.set(n, u)
        R.set_inflow_plane(u[1])
        ref.set_global("inlet_flux", R.inlet_area())
        self.R = R
        self.cells = nx * ny * nz
        # the workload's Poisson tolerance unless asked otherwise
        self.stepper = steps.ReferenceStepper(R, rtol=rtol)

    def step(self):
        return self.stepper.step()

    def close(self):
        self.R.close()


def host_max_div(uc, aj, nv):
    """Divergence of main.c:1083-1090 on the host: max |(dU + dV + dW) aj| over interior
    cells with no solid in the 7-point neighbourhood."""
    d = ((uc[1:-1, 1:-1, 1:-1, 0] - uc[1:-1, 1:-1, :-2, 0]) + (uc[1:-1, 1:-1, 1:-1, 1] - uc[1:-1, :-2, 1:-1, 1]) +
         (uc[1:-1, 1:-1, 1:-1, 2] - uc[:-2, 1:-1, 1:-1, 2])) * aj[1:-1, 1:-1, 1:-1]
    s = (nv[1:-1, 1:-1, 1:-1] + nv[2:, 1:-1, 1:-1] + nv[:-2, 1:-1, 1:-1] + nv[1:-1, 2:, 1:-1] + nv[1:-1, :-2, 1:-1] +
         nv[1:-1, 1:-1, 2:] + nv[1:-1, 1:-1, :-2])
    return float(np.abs(np.where(s > 0, 0.0, d)).max())


def vs_reference_step(nx=64, ny=48, nz=64, nsteps=3):
    """The mixed and the FP64 forms against the reference's own FP64 steps (oracle/_ref)
    from the same state, on the nx x ny x nz sample of the workload: L2 and Linf of P and
    Ucat after nsteps steps, and each side's max |div u|; once with every Poisson solve to
    the workload's rtol 1e-10, once to 1e-13."""
    import vfs_b200 as vfs
    from threadpoolctl import threadpool_limits

    def rel(a, b):
        return {"l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                "linf": float(np.abs(a - b).max() / np.abs(b).max())}
    out = {"workload": "the metric workload on a %dx%dx%d grid, %d steps from the same state" % (nx, ny, nz, nsteps),
           "note": "a residual tolerance of 1e-10 bounds the Poisson solution only up to the operator's "
                   "conditioning, so two solvers stopping at rtol 1e-10 leave P about 1e-7 apart; with both "
                   "at 1e-13 the difference is the one left by the solves"}
    for rtol in (1e-10, 1e-13):
        with threadpool_limits(limits=1), quiet_stdout():
            S = ReferenceSample(nx, ny, nz, rtol=rtol)
            R = S.R
            m, u, uc, nv = R.metrics(), R.get("Ucat"), R.get("lUcont"), R.get("lNvert")
            plane = u[1].copy()
            for _ in range(nsteps):
                S.step()
            ref_p, ref_u, ref_uc = R.get("P"), R.get("Ucat"), R.get("lUcont")
            S.close()
        res = {"reference_max_div": host_max_div(ref_uc, m["aj"], nv)}
        for prec, name in ((MIXED, "mixed"), (ALT, "mixed_fp32_krylov"), (1, "fp64")):
            case = make_case(nx, ny, nz)
            ctx = vfs.Context(case.config())
            ctx.set_metrics(m)
            ctx.set_field(vfs.NVERT, nv)
            ctx.set_field(vfs.UCONT, uc)
            ctx.set_field(vfs.UCAT, u)
            ctx.set_field(vfs.UCAT_O, u)
            ctx.set_inflow_plane(plane)
            ctx.set_scalar(vfs.S_INLET_FLUX, 0.0)
            _, area = ctx.calc_inlet_area()
            ctx.set_scalar(vfs.S_INLET_FLUX, area)
            st = [ctx.step(precision=prec, rtol=rtol) for _ in range(nsteps)]
            res[name] = {"p": rel(ctx.get_field(vfs.P), ref_p), "u": rel(ctx.get_field(vfs.UCAT), ref_u),
                         "max_div": st[-1].max_div}
            ctx.close()
        out["rtol_%g" % rtol] = res
    return out


def reference_fit(steps_per_size=1):
    """Phase times of one reference step at each of REF_SIZES (after one untimed step)
    and the fitted exponent a of t = c * cells^a for every phase."""
    from threadpoolctl import threadpool_limits
    rows = []
    with threadpool_limits(limits=1), quiet_stdout():
        for (nx, ny, nz) in REF_SIZES:
            S = ReferenceSample(nx, ny, nz)
            S.step()
            t = [S.step() for _ in range(steps_per_size)]
            rows.append((S.cells, {p: float(np.median([x[p] for x in t])) for p in PHASES}))
            S.close()
    cells = np.log([r[0] for r in rows])
    expo = {}
    for p in PHASES:
        tp = np.log([max(r[1][p], 1e-9) for r in rows])
        expo[p] = float(np.polyfit(cells, tp, 1)[0])
    return rows, expo


def extrapolate(phase_s, cells, expo, full=NX * NY * NZ):
    """ms of a full-size step from a sample's phase times and the fitted exponents."""
    return 1e3 * sum(phase_s[p] * (full / cells) ** expo[p] for p in PHASES)


def fit_note(rows, expo):
    return ("extrapolated to 256x192x256 phase by phase: t = c * cells^a fitted over one reference step at "
            "each of %s (a: %s); Poisson (HYPRE in the reference) by FGMRES with a geometric multigrid "
            "preconditioner on the reference's own matrix, rtol 1e-10, its set-up outside the step; one host "
            "thread (the oracle is single-rank)" % (
                ", ".join("%dx%dx%d" % s for s in REF_SIZES),
                ", ".join("%s %.2f" % (p, expo[p]) for p in PHASES)))


def max_over_ranks(values, dist, torch, device):
    """The largest of each value over the ranks of the process group (the replicas' step
    times: the job is as slow as its slowest replica)."""
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def arm_config(world, nx=NX, ny=NY, nz=NZ, size=None):
    """The `config` object of the JSON line, the same for both arms."""
    npts = (nx + 2) * (ny + 2) * (nz + 2)
    return {"workload": WORKLOAD if not size else "size override %s" % size,
            "cells": nx * ny * nz, "parallelism": "replicas" if world > 1 else "single-gpu",
            "precision": "mixed: FP32 multigrid V-cycle (%d levels, zebra y-line Gauss-Seidel 3+3 "
                         "sweeps, trilinear prolongation) in FP64 FGMRES(30)" % mg_levels(nx, ny, nz),
            "l2": "inputs larger than L2 (every field is a %d MB array)" % (npts * 8 // 2 ** 20)}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvfsref.so was not built"}))
        return
    from threadpoolctl import threadpool_limits
    rows, expo = reference_fit()
    samples = []
    with threadpool_limits(limits=1), quiet_stdout():
        S = ReferenceSample(*REF_STEP_SIZE)
        for s in range(args.warmup + args.steps):
            t = S.step()
            if s >= args.warmup:
                samples.append(extrapolate(t, S.cells, expo))
        S.close()
    v = float(np.mean(samples))
    sample = ("each step: one reference step (oracle/_ref, the reference's own momentum.c, rhs.c, poisson.c, "
              "bcs.c ... under the single-rank shim) on a %dx%dx%d sample of the workload, %s"
              % (REF_STEP_SIZE + (fit_note(rows, expo),)))
    out = {"metric": METRIC, "value": round(v, 3), "unit": "ms/step", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference", "extrapolated": True,
           "config": arm_config(world),
           "cpu_baseline": {"value": round(v, 3), "unit": "ms/step", "cores": 1, "kind": "reference",
                            "sample": sample, "extrapolated": True,
                            "fit": {"sizes": ["%dx%dx%d" % s for s in REF_SIZES],
                                    "phase_seconds": [r[1] for r in rows], "exponent": expo}},
           "e2e": {"value": round(v, 3), "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ------------------------------------------------------------------ our arm
ADJ_WORKLOAD = ("wavy-wall channel %dx%dx%d cells (bottom y_w = 0.1 sin(2 pi x/Lx) cos(2 pi z/Lz)), "
                "immersed sphere D=0.4 at the centre (icosphere, 20480 triangles, IB nodes), inlet k=0 "
                "(inletprofile 100) and outlet k+, FP64 Poisson rtol 1e-10; objective: streamwise "
                "drag on the body (pressure force plus viscous traction on its cell faces) after %d steps; control: the inflow plane; checkpoint "
                "every %d steps")


def adjoint_context(nx, ny, nz):
    """The adjoint window's context: the curvilinear channel with the immersed sphere, an
    inlet (inletprofile 100) and an outlet, a seeded initial field."""
    import vfs_b200 as vfs
    from vfs_b200 import cases
    case = cases.channel(nx, ny, nz, wavy=0.1)
    case.immersed = 1
    cases.inflow_outflow(case, 100)
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    ctx.ibm_search(*cases.icosphere((np.pi / 2, 1.0, np.pi), 0.2, level=5))
    m = {n: ctx.get_field(f) for n, f in vfs.METRIC_FIELDS.items()}
    case.nvert = ctx.get_field(vfs.NVERT)
    u = cases.initial_ucat(case, seed=0)
    ctx.set_field(vfs.UCONT, cases.ucont_from_ucat(case, u, m))
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    ctx.set_scalar(vfs.S_INLET_FLUX, 0.0)
    _, area = ctx.calc_inlet_area()
    ctx.set_scalar(vfs.S_INLET_FLUX, area)
    ctx.set_inflow_plane(cases.inflow_plane(case))
    return ctx, case



def adjoint_window(nx, ny, nz, steps, every, torch):
    """The discrete adjoint of a window of FP64 steps on the curvilinear grid with the
    sphere: gradient of the body's drag after `steps` steps with respect to the inflow
    plane.  Returns the reverse sweep (segment recomputation + adjoint steps) and the
    forward sweep timed on the device, and the one-off operator set-up time."""
    import vfs_b200 as vfs
    from vfs_b200 import cases
    ctx, case = adjoint_context(nx, ny, nz)
    t0 = time.perf_counter()
    ctx.adjoint_setup()
    setup_s = time.perf_counter() - t0
    kw = dict(objective=vfs.OBJ_DRAG, control=vfs.CTRL_INFLOW_PLANE, precision=1, rtol=1e-10)
    for _ in range(2):  # warm-up: tapes, checkpoints, Krylov space, clocks
        ctx.adjoint_gradient(steps, checkpoint_every=every, **kw)
    torch.cuda.synchronize()
    # the launched steps of both sweeps read the solver's loop flags and the adjoint's global
    # sums back on the host, so a busy host stretches their event times: five windows, the
    # median ratio, the smallest beside it
    sampler = ClockSampler(torch.cuda.current_device())
    with sampler:
        runs = [ctx.adjoint_gradient(steps, checkpoint_every=every, **kw) for _ in range(5)]
    sm = [float(r[1]) for r in sampler.rows if r[1].replace(".", "").isdigit()]
    ratios = [r[1].ms_adjoint / r[1].ms_forward for r in runs]
    g, st = runs[int(np.argsort(ratios)[2])]
    # central difference of J along one combined direction: 32 seeded interior inlet entries
    # of the streamwise component, random signs, scaled by the plane's RMS streamwise velocity
    plane = cases.inflow_plane(case)
    rng = np.random.Generator(np.random.Philox(7))
    d = np.zeros_like(plane)
    jj = rng.integers(1, plane.shape[0] - 1, 32)
    ii = rng.integers(1, plane.shape[1] - 1, 32)
    d[jj, ii, 2] = rng.choice([-1.0, 1.0], 32) * float(np.sqrt((plane[..., 2] ** 2).mean()))
    # The check runs every Poisson solve for 30 FGMRES iterations (one restart cycle, past
    # the FP64 floor of about 15): J is then free of the jumps that a tolerance-based stopping
    # point puts into it.  What remains is J's own rounding floor (a few 1e-13 of J: the drag
    # sums pressures far larger than their net), which bounds the central difference at a
    # step eps to about floor / (eps |dJ/deps| / J): hence the range of steps and the
    # Richardson combination of the two largest.
    kw_fd = dict(kw, rtol=1e-300, max_iter=30)
    ad = float((g * d).sum())
    g30, _ = ctx.adjoint_gradient(steps, checkpoint_every=every, **kw_fd)
    ad30 = float((g30 * d).sum())
    _, dj_tan = ctx.tangent(d, steps, objective=vfs.OBJ_DRAG, control=vfs.CTRL_INFLOW_PLANE, precision=1,
                            rtol=1e-300, max_iter=30)
    fd_check = {"direction": "32 seeded interior inlet entries of w, random signs, x RMS(w) of the plane",
                "adjoint": ad, "adjoint_30_iterations": ad30, "tangent_30_iterations": dj_tan,
                "adjoint_vs_tangent_rel": abs(ad30 - dj_tan) / abs(dj_tan),
                "adjoint_rtol_1e-10_vs_30_iterations_rel": abs(ad - ad30) / abs(ad30),
                "poisson": "30 FGMRES iterations per solve in every window of the check",
                "central_difference": {}, "rel_err": {}}
    fds = {}
    for eps in (2e-3, 1e-3, 1e-4, 1e-5, 1e-6):
        jpm = []
        for sgn in (1.0, -1.0):
            ctx.set_inflow_plane(plane + sgn * eps * d)
            jpm.append(ctx.objective(steps, **kw_fd))
        fds[eps] = (jpm[0] - jpm[1]) / (2 * eps)
        fd_check["central_difference"]["%g" % eps] = fds[eps]
        fd_check["rel_err"]["%g" % eps] = abs(fds[eps] - ad30) / abs(ad30)
    rich = (4 * fds[1e-3] - fds[2e-3]) / 3
    fd_check["richardson_1e-3_2e-3"] = rich
    fd_check["rel_err_richardson"] = abs(rich - ad30) / abs(ad30)
    fd_check["implied_J_noise_rel"] = abs(fds[1e-6] - ad30) * 2e-6 / abs(st.J)
    ctx.set_inflow_plane(plane)
    ctx.close()
    return {"workload": ADJ_WORKLOAD % (nx, ny, nz, steps, every), "steps": steps, "checkpoint_every": every,
            "forward_ms": round(st.ms_forward, 2), "adjoint_ms": round(st.ms_adjoint, 2),
            "ratio": round(st.ms_adjoint / st.ms_forward, 3), "ratio_min": round(min(ratios), 3),
            "ratios_of_5_windows": [round(v, 3) for v in ratios],
            "windows_ms": [[round(r[1].ms_forward, 2), round(r[1].ms_adjoint, 2)] for r in runs],
            "clocks": dict(sampler.summary(), sm_mhz_min=min(sm) if sm else None),
            "recomputed_steps": st.recomputed_steps,
            "tape_bytes": st.tape_bytes, "operator_setup_s": round(setup_s, 1),
            "J": st.J, "gradient_norm": float(np.sqrt((g * g).sum())), "fd_check": fd_check,
            "poisson_iterations": {"forward": st.poisson_iterations_forward,
                                   "adjoint": st.poisson_iterations_adjoint},
            "note": "ratio = reverse sweep (recomputation of every checkpoint segment plus the adjoint "
                    "steps) / forward sweep of the same window; the window with the median of five ratios"}


# Algorithmic bytes per cell of the step's parts (each input read once, each output written
# once at its stored precision), for the large-window HBM figure.
STEP_BYTES = {
    "formfunction2": 4 * 433.0,           # four RK stages (pUcont and dP read, Ucont written)
    "contra2cart": 10 * 121.0,            # two per RK stage, two in the correction
    "pressure_gradient": 129.0,
    "calc_k_flux_and_rhs": 25.0 + 33.0,   # Ucont.z + nvert; Ucont + nvert -> b
    "projection_update": 169.0,
    "divergence": 8.0,                    # aj, in Projection's Contra2Cart
    "end_of_step_copies": 96.0,           # Ucont -> Ucont_o, Ucat -> Ucat_o
    # per FGMRES iteration: the FP64 apply 73, one FP32 V-cycle (3+3 zebra sweeps at 32 B,
    # restriction and prolongation about 40, the zebra layout conversions 24, coarser
    # levels x 8/7: about 293), the basis passes (three over j+1 vectors, 8 B each, about
    # 24 (j+1)) and the Z and V writes 16
    "per_iteration_fixed": 73.0 + 293.0 + 16.0,
}


def step_bytes_per_cell(iterations):
    it = int(round(iterations))
    fixed = sum(v for k, v in STEP_BYTES.items() if k != "per_iteration_fixed")
    krylov = sum(STEP_BYTES["per_iteration_fixed"] + 24.0 * (j + 1) for j in range(it))
    return fixed + krylov


def large_window(torch, nx=384, ny=256, nz=384, steps=50, every=7):
    """A 50-step window on the 384 x 256 x 384 wavy-bottom open channel with the cylinder
    array, mixed precision, the step as one CUDA graph: steps/s, algorithmic HBM GB/s
    (STEP_BYTES), device memory held.  Then, on the same context, the gradient of the total
    kinetic energy after 50 steps with respect to the inflow plane: checkpoints every 7
    steps (about sqrt(50)), each segment recomputed with its tapes before its adjoint steps;
    the forward and reverse sweeps timed on the device and the peak device memory."""
    import vfs_b200 as vfs
    from vfs_b200 import cases
    free0, total = torch.cuda.mem_get_info()
    case = cases.inflow_outflow(cases.open_channel_cylinders(nx, ny, nz, wavy=0.05), 100)
    case.immersed = 0
    ctx, _ = setup_context(case)
    ctx.step(precision=MIXED, rtol=1e-10)
    for _ in range(3):
        ctx.step(precision=MIXED, rtol=1e-10, graph=1)
    ms, stats = timed(ctx, lambda: ctx.step(precision=MIXED, rtol=1e-10, graph=1), steps, torch)
    free1, _ = torch.cuda.mem_get_info()
    its = float(np.mean([s.poisson.iterations for s in stats]))
    ms_step = ms / steps
    cells = nx * ny * nz
    bpc = step_bytes_per_cell(its)
    out = {"workload": "wavy-bottom open channel %dx%dx%d cells (y_w = 0.05 sin(2 pi x/Lx) cos(2 pi z/Lz)), "
                       "the 3x2 cylinder array as blocked cells, inlet k=0 (inletprofile 100), outlet k+, "
                       "mixed precision, Poisson rtol 1e-10" % (nx, ny, nz),
           "steps": steps, "ms_per_step": round(ms_step, 3), "steps_per_s": round(1000.0 / ms_step, 3),
           "poisson_iterations": its, "max_div": max(s.max_div for s in stats),
           "hbm_gbs": round(bpc * cells / (ms_step * 1e-3) / 1e9, 1), "bytes_per_cell_per_step": round(bpc, 1),
           "device_memory_gb": round((free0 - free1) / 1e9, 2),
           "note": "hbm_gbs = algorithmic bytes of the step (each input read once, each output written "
                   "once; STEP_BYTES) / step time"}
    # the adjoint of the window, from the state the forward window left
    kw = dict(objective=vfs.OBJ_KINETIC_ENERGY, control=vfs.CTRL_INFLOW_PLANE, precision=MIXED, rtol=1e-10)
    t0 = time.perf_counter()
    ctx.adjoint_setup()
    setup_s = time.perf_counter() - t0
    ctx.adjoint_gradient(every, checkpoint_every=every, **kw)  # warm-up: tapes, one segment
    g, st = ctx.adjoint_gradient(steps, checkpoint_every=every, **kw)
    free2, _ = torch.cuda.mem_get_info()
    out["adjoint"] = {
        "objective": "total kinetic energy 0.5 sum |u|^2 / aj over the fluid cells after the window",
        "control": "the inflow plane (3 x %d x %d)" % (nx, ny), "steps": steps, "checkpoint_every": every,
        "forward_ms": round(st.ms_forward, 1), "adjoint_ms": round(st.ms_adjoint, 1),
        "ratio": round(st.ms_adjoint / st.ms_forward, 3),
        "forward_sweep_ms_per_step": round(st.ms_forward / steps, 2),
        "poisson_iterations": {"forward": st.poisson_iterations_forward, "adjoint": st.poisson_iterations_adjoint},
        "J": st.J, "gradient_norm": float(np.sqrt((g * g).sum())), "tape_gb": round(st.tape_bytes / 1e9, 2),
        "device_memory_gb": round((free0 - free2) / 1e9, 2), "device_total_gb": round(total / 1e9, 2),
        "setup_s": round(setup_s, 2),
        "note": "ratio = reverse sweep (recomputation of each 7-step segment with its tapes, then its "
                "adjoint steps) / forward sweep that stores the checkpoints; every operator transposed by "
                "hand-written kernels (no measured matrix on this grid)"}
    ctx.close()
    return out


# FP64 instructions per cell of one dynamic-Smagorinsky evaluation (Compute_Smagorinsky_
# Constant_1 + Compute_eddy_viscosity_LES) on the 128 x 96 x 128 wavy channel, counted by
# ncu (2 x DFMA + DMUL + DADD, executed thread instructions, every kernel of the call; the
# division and square-root sequences count by their instructions):
# profiles/les_dynamic_smagorinsky_128x96x128.md.
LES_FLOPS_PER_CELL = 5373
FP64_PEAK_TFLOPS = 37.0   # nominal B200 FP64 (vector), no measured figure in MEASURED_PEAKS.json


def les_context(nx=128, ny=96, nz=128):
    """Config 2's grid (128 x 96 x 128 channel, wavy bottom y_w = 0.1 sin cos) with the
    dynamic Smagorinsky model (les = 2) and a seeded turbulent-like field."""
    import vfs_b200 as vfs
    from vfs_b200 import cases
    case = cases.channel(nx, ny, nz, wavy=0.1)
    case.les = 2
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    m = {n: ctx.get_field(f) for n, f in vfs.METRIC_FIELDS.items()}
    u = cases.initial_ucat(case, seed=0)
    ctx.set_field(vfs.UCONT, cases.ucont_from_ucat(case, u, m))
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    ctx.contra2cart()
    ctx.set_scalar(vfs.S_TI, 5)   # Cs is 0 in the first two steps of a fresh run (les.c:69-72)
    return ctx, nx * ny * nz


def les_probe(torch, reps=20):
    """Time of one dynamic-Smagorinsky evaluation (the Cs field with its averaging and
    clipping, then nu_t) on config 2's grid, and its FP64 rate against the nominal peak."""
    ctx, cells = les_context()
    for _ in range(3):
        ctx.smagorinsky_constant()
        ctx.eddy_viscosity()

    def body():
        ctx.smagorinsky_constant()
        ctx.eddy_viscosity()
    ms, _ = timed(ctx, body, reps, torch)
    ctx.close()
    ms /= reps
    out = {"workload": "dynamic Smagorinsky (les = 2: Compute_Smagorinsky_Constant_1 + "
                       "Compute_eddy_viscosity_LES) on the 128x96x128 wavy channel of config 2",
           "ms_per_call": round(ms, 4), "cells": cells}
    if LES_FLOPS_PER_CELL:
        tf = LES_FLOPS_PER_CELL * cells / (ms * 1e-3) / 1e12
        out.update({"fp64_flops_per_cell": LES_FLOPS_PER_CELL, "achieved_tflops": round(tf, 3),
                    "peak_tflops": FP64_PEAK_TFLOPS, "peak_source": "nominal",
                    "frac": round(tf / FP64_PEAK_TFLOPS, 4)})
    return out


def immersed_variant(nx, ny, nz, torch, steps=10):
    """The metric workload with the six cylinders as immersed bodies (immersed = 1): closed
    triangulated cylinder surfaces, classified by the IB search, with the IB-node
    reconstruction in every step (ibm_interpolation_advanced, noslip) and the immersed
    VolumeFlux.  Mixed-precision step time in the graph form."""
    import vfs_b200 as vfs
    from vfs_b200 import cases
    case = make_case(nx, ny, nz)
    case.immersed = 1
    case.nvert = np.zeros(case.da_shape)
    ctx = vfs.Context(case.config())
    ctx.form_metrics(case.X, case.Y, case.Z)
    ctx.set_field(vfs.NVERT, case.nvert)
    ctx.set_scalar(vfs.S_NBODIES, len(case.centers))
    for ibi, (cx, cz) in enumerate(case.centers):
        ctx.ibm_search(*cases.cylinder_surface((cx, cz), 0.5 * case.D, -0.1, case.Ly + 0.1, 96, 24), ibi=ibi)
    nv = ctx.get_field(vfs.NVERT)
    case.nvert = nv
    m = {"icsi": ctx.get_field(vfs.ICSI), "jeta": ctx.get_field(vfs.JETA), "kzet": ctx.get_field(vfs.KZET)}
    u = turbulent_like(case)
    ctx.set_field(vfs.UCONT, cases.ucont_from_ucat(case, u, m))
    ctx.set_field(vfs.UCAT, u)
    ctx.set_field(vfs.UCAT_O, u)
    ctx.set_inflow_plane(u[1])
    _, inlet_area = ctx.calc_inlet_area()
    ctx.set_scalar(vfs.S_INLET_FLUX, 1.0 * inlet_area)
    ctx.contra2cart()
    ctx.step(precision=MIXED, rtol=1e-10)
    for _ in range(3):
        ctx.step(precision=MIXED, rtol=1e-10, graph=1)
    ms, st = timed(ctx, lambda: ctx.step(precision=MIXED, rtol=1e-10, graph=1), steps, torch)
    nib = int(ctx.ibm_list()[0].shape[0])
    ctx.close()
    return {"workload": "the metric workload with the 6 cylinders as immersed bodies (immersed=1): closed "
                        "triangulated surfaces (96 x 24 facets each), IB search, IB-node reconstruction "
                        "(noslip) and immersed VolumeFlux every step",
            "ib_nodes": nib, "ms_per_step": round(ms / steps, 3),
            "poisson_iterations": float(np.mean([s.poisson.iterations for s in st])),
            "max_div": max(s.max_div for s in st)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", default=None, help="nx,ny,nz override (not for reported numbers)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement")
    ap.add_argument("--no-immersed", action="store_true", help="skip the immersed-cylinder variant")
    ap.add_argument("--no-large", action="store_true", help="skip the 384x256x384 50-step window")
    ap.add_argument("--adjoint-size", default="128,128,128")
    ap.add_argument("--adjoint-steps", type=int, default=20)
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="run one 2-step adjoint gradient of the adjoint window (checkpoint every "
                         "step) inside cudaProfilerStart/Stop and exit (for ncu --profile-from-start off)")
    ap.add_argument("--profile-les", action="store_true",
                    help="run one dynamic-Smagorinsky evaluation on config 2's grid inside "
                         "cudaProfilerStart/Stop and exit (for ncu --profile-from-start off)")
    ap.add_argument("--profile-step", action="store_true",
                    help="after the warm-up, run one mixed step inside cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off); prints no JSON")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    import vfs_b200 as vfs
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.profile_adjoint:
        ax, ay, az = (int(v) for v in args.adjoint_size.split(","))
        actx, _ = adjoint_context(ax, ay, az)
        kw = dict(objective=vfs.OBJ_DRAG, control=vfs.CTRL_INFLOW_PLANE, precision=1, rtol=1e-10)
        actx.adjoint_gradient(2, checkpoint_every=1, **kw)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        actx.adjoint_gradient(2, checkpoint_every=1, **kw)
        actx.synchronize()
        torch.cuda.profiler.stop()
        actx.close()
        return

    if args.profile_les:
        lctx, _ = les_context()
        for _ in range(3):
            lctx.smagorinsky_constant()
            lctx.eddy_viscosity()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        lctx.smagorinsky_constant()
        lctx.eddy_viscosity()
        lctx.synchronize()
        torch.cuda.profiler.stop()
        lctx.close()
        return

    nx, ny, nz = (NX, NY, NZ) if not args.size else tuple(int(v) for v in args.size.split(","))
    case = make_case(nx, ny, nz)
    ctx, u0 = setup_context(case)
    ncell = nx * ny * nz

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (also the first-step set-up: inlet area, Poisson operator, IB_BC)
    for _ in range(max(3, args.warmup)):
        ctx.step(precision=0, rtol=1e-10)
    if args.profile_step:
        ctx.step(precision=MIXED, rtol=1e-10)   # the mixed form's workspace
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ctx.step(precision=MIXED, rtol=1e-10)
        ctx.synchronize()
        torch.cuda.profiler.stop()
        ctx.close()
        return

    # the flow state after the warm-up; the FP64 steps are timed from the same state as the
    # mixed ones (the Poisson solve starts from the previous Phi, so its iteration count
    # depends on how far the flow has developed)
    state_fields = (vfs.UCONT, vfs.UCAT, vfs.P, vfs.UCAT_O, vfs.UCONT_O, vfs.PHI)
    keep = {f: ctx.get_field(f) for f in state_fields}
    ti = ctx.get_scalar(vfs.S_TI)

    def restore():
        for f, v in keep.items():
            ctx.set_field(f, v)
        ctx.set_scalar(vfs.S_TI, ti)

    for _ in range(2):  # FP64 multigrid set-up and the step graphs, outside the timed steps
        ctx.step(precision=1, rtol=1e-10, graph=1)
    for prec in (MIXED, ALT):
        restore()
        ctx.step(precision=prec, rtol=1e-10)            # the form's workspace
        restore()
        ctx.step(precision=prec, rtol=1e-10, graph=1)   # its graph
    restore()
    sampler = ClockSampler(local)
    with sampler:
        barrier()
        ms_mixed, stats = timed(ctx, lambda: ctx.step(precision=MIXED, rtol=1e-10, graph=1), args.steps, torch)
        barrier()
        restore()
        barrier()
        ms_fp64, stats64 = timed(ctx, lambda: ctx.step(precision=1, rtol=1e-10, graph=1), args.steps, torch)
        barrier()
        restore()
        barrier()
        ms_alt, stats_alt = timed(ctx, lambda: ctx.step(precision=ALT, rtol=1e-10, graph=1), args.steps, torch)
        barrier()
        restore()
        barrier()
        ms_launched, _ = timed(ctx, lambda: ctx.step(precision=MIXED, rtol=1e-10), args.steps, torch)
        barrier()
    ms_mixed /= args.steps
    ms_fp64 /= args.steps
    ms_alt /= args.steps
    ms_launched /= args.steps
    maxdiv = max(s.max_div for s in stats)
    maxdiv64 = max(s.max_div for s in stats64)
    maxdiv_alt = max(s.max_div for s in stats_alt)
    its = float(np.mean([s.poisson.iterations for s in stats]))
    its64 = float(np.mean([s.poisson.iterations for s in stats64]))
    its_alt = float(np.mean([s.poisson.iterations for s in stats_alt]))

    # mixed against FP64 from one state: L2 and Linf of P and Ucat (both solves to rtol 1e-10,
    # both from the same Phi)
    outs = {}
    for prec in (MIXED, ALT, 1):
        restore()
        st = ctx.step(precision=prec, rtol=1e-10)
        outs[prec] = (ctx.get_field(vfs.P), ctx.get_field(vfs.UCAT), st.max_div)

    def rel(a, b):
        return {"l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                "linf": float(np.abs(a - b).max() / np.abs(b).max())}
    mixed_err = {"p": rel(outs[MIXED][0], outs[1][0]), "u": rel(outs[MIXED][1], outs[1][1]),
                 "max_div": {"mixed": outs[MIXED][2], "fp64": outs[1][2]},
                 "fp32_krylov_form": {"p": rel(outs[ALT][0], outs[1][0]), "u": rel(outs[ALT][1], outs[1][1]),
                                      "max_div": outs[ALT][2]},
                 "note": "one step from the same state, the mixed forms against the all-FP64 form"}

    # e2e: flow state from pinned host memory each step, result back to the host
    shp3 = ctx.shape + (3,)
    h_uc = torch.empty(shp3, dtype=torch.float64, pin_memory=True).numpy()
    h_u = torch.empty(shp3, dtype=torch.float64, pin_memory=True).numpy()
    h_p = torch.empty(ctx.shape, dtype=torch.float64, pin_memory=True).numpy()
    h_uc[...] = ctx.get_field(vfs.UCONT)
    h_u[...] = ctx.get_field(vfs.UCAT)
    h_p[...] = ctx.get_field(vfs.P)

    def e2e_step():
        ctx.set_field(vfs.UCONT, h_uc)
        ctx.set_field(vfs.UCAT, h_u)
        ctx.set_field(vfs.P, h_p)
        st = ctx.step(precision=MIXED, rtol=1e-10, graph=1)
        ctx.get_field(vfs.UCONT, out=h_uc)
        ctx.get_field(vfs.UCAT, out=h_u)
        ctx.get_field(vfs.P, out=h_p)
        return st
    e2e_step()
    barrier()
    t0 = time.perf_counter()
    e2e_ms, _ = timed(ctx, e2e_step, max(2, args.steps // 2), torch)
    barrier()
    e2e_ms /= max(2, args.steps // 2)
    npts = int(np.prod(ctx.shape))
    io_bytes = npts * 8 * 7

    # roofline of the dominant operator
    launch = roofline_probe(ctx, torch)
    peak, peak_kind = hbm_peak()
    dom = "formfunction2"
    achieved = KERNEL_BYTES[dom] * ncell / (launch[dom] * 1e-3) / 1e9
    kernel_frac = {k: round(KERNEL_BYTES[k] * ncell / (launch[k] * 1e-3) / 1e9 / peak, 3)
                   for k in KERNEL_BYTES if k in launch}
    # Amdahl: one V-cycle per FGMRES iteration; everything else in the mixed step is the same
    # FP64 work as in the FP64 form
    v32, v64 = launch["vcycle_fp32"], launch["vcycle_fp64"]
    common = ms_mixed - its * v32
    amdahl = {"vcycle_fp32_ms": round(v32, 4), "vcycle_fp64_ms": round(v64, 4),
              "vcycle_speedup": round(v64 / v32, 3), "vcycles_per_step": {"mixed": its, "fp64": its64},
              "rest_of_step_ms": round(common, 3),
              "fp64_predicted_ms": round(common + its64 * v64, 3),
              "formfunction2_ms_per_step": round(4 * launch["formfunction2"], 3),
              "speedup_bound_vcycle_free": round(ms_fp64 / common, 3),
              "speedup_bound_vcycle_2x": round(ms_fp64 / (common + its64 * v64 / 2), 3),
              "note": "rest_of_step = mixed step - iterations x FP32 V-cycle (every other kernel is the "
                      "same FP64 work in both forms); bounds: FP64 step / mixed step if the V-cycle cost "
                      "nothing, or ran at twice the FP64 speed"}
    launches_per_step = None

    if dist is not None:
        ms_mixed, ms_fp64, e2e_ms = max_over_ranks([ms_mixed, ms_fp64, e2e_ms], dist, torch, "cuda")

    n0 = ctx.launch_count()
    ctx.step(precision=MIXED, rtol=1e-10, graph=1)
    launches_per_step = ctx.launch_count() - n0
    ctx.close()
    del keep

    imm = None
    if not args.no_immersed and not args.size:
        try:
            imm = immersed_variant(nx, ny, nz, torch)
        except Exception as e:  # reported, never fatal for the forward numbers
            imm = {"failed": str(e)}

    les = None
    if not args.size:
        try:
            les = les_probe(torch)
        except Exception as e:  # reported, never fatal for the forward numbers
            les = {"failed": str(e)}

    large = None
    if not args.no_large and not args.size:
        try:
            large = large_window(torch)
        except Exception as e:  # reported, never fatal for the forward numbers
            large = {"failed": str(e)}

    adj = None
    if not args.no_adjoint and not args.size:
        ax, ay, az = (int(v) for v in args.adjoint_size.split(","))
        try:
            adj = adjoint_window(ax, ay, az, args.adjoint_steps, 5, torch)
        except Exception as e:  # reported, never fatal for the forward numbers
            adj = {"failed": str(e)}

    out = None
    if rank == 0:
        cpu = None
        vsref = None
        if world == 1 and not args.no_cpu_baseline and not args.size:
            try:
                from oracle import ref
                if ref.available():
                    rows, expo = reference_fit()
                    cells, big = rows[-1]
                    cpu = {"value": round(extrapolate(big, cells, expo), 1), "unit": "ms/step", "cores": 1,
                           "kind": "reference", "extrapolated": True,
                           "sample": "one reference step (oracle/_ref) on the 128x96x128 sample of this "
                                     "workload, " + fit_note(rows, expo),
                           "fit": {"sizes": ["%dx%dx%d" % s for s in REF_SIZES],
                                   "phase_seconds": [r[1] for r in rows], "exponent": expo}}
            except Exception as e:  # the baseline is reported, never required
                cpu = {"value": None, "unit": "ms/step", "cores": 1, "kind": "reference",
                       "sample": "failed: %s" % e}
            try:
                from oracle import ref
                if ref.available():
                    vsref = vs_reference_step()
            except Exception as e:  # reported, never fatal
                vsref = {"failed": str(e)}
        out = {
            "metric": METRIC, "value": round(ms_mixed * world / world, 3), "unit": "ms/step",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": arm_config(world, nx, ny, nz, args.size),
            "fp64_ms_per_step": round(ms_fp64, 3),
            "launched_ms_per_step": round(ms_launched, 3),
            "step_form": "one CUDA graph per step (captured once, replayed; the Poisson solve's loops as "
                         "conditional nodes); launched_ms_per_step: the same kernels launched one by one",
            "mixed_speedup_vs_fp64": round(ms_fp64 / ms_mixed, 3),
            "fp32_krylov_form": {"ms_per_step": round(ms_alt, 3), "speedup_vs_fp64": round(ms_fp64 / ms_alt, 3),
                                 "poisson_iterations": its_alt, "max_div": maxdiv_alt,
                                 "note": "precision 2: the FGMRES basis, preconditioned vectors and V-cycle in "
                                         "FP32, every restart cycle an iterative-refinement sweep from the FP64 "
                                         "residual"},
            "max_div": {"mixed": maxdiv, "fp64": maxdiv64},
            "poisson_iterations": {"mixed": its, "fp64": its64},
            "mixed_vs_fp64": mixed_err,
            "vs_reference_step": vsref,
            "amdahl": amdahl,
            "adjoint_forward_ratio": adj.get("ratio") if adj else None,
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms/step", "h2d_bytes_per_step": io_bytes,
                    "d2h_bytes_per_step": io_bytes},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": KERNEL_TRAFFIC.get(dom), "traffic_unit": "bytes per launch", "kernel": dom,
                         "peak_source": peak_kind, "bytes_per_cell": KERNEL_BYTES[dom],
                         "ms_per_launch": round(launch[dom], 4),
                         "other_ms_per_launch": {k: round(v, 4) for k, v in launch.items()},
                         "frac_of_peak": kernel_frac},
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": sampler.summary(),
        }
        if adj is not None:
            out["adjoint"] = adj
        if imm is not None:
            out["immersed_variant"] = imm
        if large is not None:
            out["large_window"] = large
        if les is not None:
            out["les"] = les
        if cpu is not None:
            out["cpu_baseline"] = cpu
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
