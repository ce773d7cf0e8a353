"""Loading of the golden fixtures (tests/golden/*.npz) together with the synthetic case
that produced them; the case's grid and flags must equal the stored ones."""
import os

import numpy as np

from vfs_b200 import cases

HERE = os.path.dirname(os.path.abspath(__file__))

FIXTURES = {
    "wavy_channel_12x10x14": lambda: cases.channel(12, 10, 14, wavy=0.15),
    "cylinders_16x12x24": lambda: cases.open_channel_cylinders(16, 12, 24, D=0.6, Lx=3.2, Lz=8.0, Ly=1.0),
}


def load(name):
    d = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    case = FIXTURES[name]()
    for k in ("X", "Y", "Z"):
        np.testing.assert_array_equal(getattr(case, k), d[k], err_msg="fixture grid " + k)
    np.testing.assert_array_equal(np.asarray(case.nvert, dtype=np.float64), d["nvert"])
    return case, d
