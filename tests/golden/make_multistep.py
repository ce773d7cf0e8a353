"""Generates tests/golden/multistep_wavy_sphere_les_128x96x128.npz: the reference's own
20 time steps (oracle/_ref, tests/multistep.py) of the 128x96x128 wavy-wall channel with
the immersed 20480-triangle sphere and dynamic Smagorinsky LES (Re = 1e4, dt = 1e-3).

The whole fields are 90 MB, so the fixture keeps P, Ucont (the reference's lUcont) and
Ucat at 20000 seeded DA points, their sums over each k plane, their largest magnitudes,
nvert at the same points, and the per-step Poisson iteration counts.  Runs on the CPU in
this container (about ten minutes on one core); needs oracle/_ref.

    python tests/golden/make_multistep.py
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "vfs-geophysics-3.1_b200"), os.path.dirname(HERE)):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import multistep  # noqa: E402

NSTEPS = 20
NPTS = 20000


def main(out=os.path.join(HERE, "multistep_wavy_sphere_les_128x96x128.npz")):
    case, body = multistep.wavy_sphere_les()
    t0 = time.time()
    run = multistep.ReferenceRun(case, body=body)
    nv = run.R.get("lNvert")
    for s in range(NSTEPS):
        run.step()
        print("step %d: %.1f s, Poisson %s" % (s, time.time() - t0, run.history[-1]), flush=True)
    f = run.fields()
    idx = multistep.sample_points(nv.shape, NPTS)
    res = {"nsteps": NSTEPS, "idx": idx, "nvert": nv.ravel()[idx],
           "poisson_iterations": np.array([h["poisson_iterations"] for h in run.history])}
    for name, a in f.items():
        flat = a.reshape(-1) if a.ndim == 3 else a.reshape(-1, 3)
        res[name + "_pts"] = flat[idx]
        res[name + "_planes"] = a.sum(axis=(1, 2))
        res[name + "_max"] = np.abs(a).max()
    np.savez_compressed(out, **res)
    run.close()
    print("wrote", out)


if __name__ == "__main__":
    main()
