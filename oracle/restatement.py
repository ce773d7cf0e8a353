"""ctypes wrapper of oracle/liboracle.so, the C restatement of the reference's projection
path (oracle/vfs_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline to compare against, never by the product.  Arrays use the reference's DA layout
(numpy shape (mz, my, mx[, 3])).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


class OgGrid(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int),
                ("iper", ctypes.c_int), ("jper", ctypes.c_int), ("kper", ctypes.c_int),
                ("immersed", ctypes.c_int), ("les", ctypes.c_int), ("bc", ctypes.c_int * 6),
                ("ren", ctypes.c_double), ("dt", ctypes.c_double), ("st", ctypes.c_double)]


class OgMetrics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("icsi", "ieta", "izet", "iaj", "jcsi", "jeta", "jzet", "jaj",
                                               "kcsi", "keta", "kzet", "kaj", "csi", "eta", "zet")]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build_oracle
            build_oracle.build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.og_divergence.restype = ctypes.c_double
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


METRIC_NAMES = ("cent", "csi", "eta", "zet", "aj", "icsi", "ieta", "izet", "iaj", "jcsi", "jeta", "jzet",
                "jaj", "kcsi", "keta", "kzet", "kaj")


def grid_of(case):
    g = OgGrid()
    g.mz, g.my, g.mx = case.da_shape
    g.iper, g.jper, g.kper = case.i_periodic, case.j_periodic, case.k_periodic
    g.immersed, g.les = case.immersed, case.les
    for q in range(6):
        g.bc[q] = case.bctype[q]
    g.ren, g.dt, g.st = case.ren, case.dt, case.st
    return g


def form_metrics(case):
    """FormMetrics (metrics.c:4, NEWMETRIC) from the case's grid.dat nodes."""
    g = grid_of(case)
    sh = case.da_shape
    out = {}
    for n in METRIC_NAMES:
        out[n] = np.zeros(sh if n.endswith("aj") else sh + (3,))
    X, Y, Z = (np.ascontiguousarray(a, dtype=np.float64) for a in (case.X, case.Y, case.Z))
    lib().og_form_metrics(ctypes.byref(g), _p(X), _p(Y), _p(Z), *[_p(out[n]) for n in METRIC_NAMES])
    return out


class State:
    """Flow state of one case on the reference layout."""

    def __init__(self, case, m, ucont, ucat, p=None, nut=None):
        self.case = case
        self.g = grid_of(case)
        self.m = {k: np.ascontiguousarray(v) for k, v in m.items()}
        self.ucont = np.array(ucont, dtype=np.float64)
        self.ucat = np.array(ucat, dtype=np.float64)
        self.ucat_old = np.array(ucat, dtype=np.float64)
        self.nvert = np.ascontiguousarray(case.nvert, dtype=np.float64)
        self.p = np.zeros(case.da_shape) if p is None else np.array(p, dtype=np.float64)
        self.nut = np.zeros(case.da_shape) if nut is None else np.array(nut, dtype=np.float64)
        self.om = OgMetrics(**{n: _p(self.m[n]) for n, _ in OgMetrics._fields_})


def contra2cart(st):
    lib().og_contra2cart(ctypes.byref(st.g), _p(st.ucont), _p(st.m["csi"]), _p(st.m["eta"]), _p(st.m["zet"]),
                         _p(st.nvert), _p(st.ucat_old), _p(st.ucat))


def formfunction2(st, scale, rhs=None):
    out = np.zeros(st.case.da_shape + (3,)) if rhs is None else np.array(rhs, dtype=np.float64)
    lib().og_formfunction2(ctypes.byref(st.g), ctypes.byref(st.om), _p(st.ucont), _p(st.ucat), _p(st.nvert),
                           _p(st.nut), ctypes.c_double(scale), _p(out))
    return out


def pressure_gradient(st, kforce=0, mpg=0.0, kdiff=0.0, karea=1.0):
    dp = np.zeros(st.case.da_shape + (3,))
    lib().og_pressure_gradient(ctypes.byref(st.g), ctypes.byref(st.om), _p(st.nvert), _p(st.p), ctypes.c_int(kforce),
                               ctypes.c_double(mpg), ctypes.c_double(kdiff), ctypes.c_double(karea), _p(dp))
    return dp


def poisson_lhs(st):
    coef = np.zeros((19,) + st.case.da_shape)
    lib().og_poisson_lhs(ctypes.byref(st.g), ctypes.byref(st.om), _p(st.nvert), _p(coef))
    return coef


def poisson_apply(st, coef, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(st.case.da_shape)
    lib().og_poisson_apply(ctypes.byref(st.g), _p(coef), _p(st.nvert), _p(x), _p(y))
    return y


def poisson_rhs(st):
    b = np.zeros(st.case.da_shape)
    lib().og_poisson_rhs(ctypes.byref(st.g), _p(st.ucont), _p(st.nvert), _p(st.m["aj"]), _p(b))
    return b


def update_pressure(st, phi):
    phi = np.array(phi, dtype=np.float64)
    lib().og_update_pressure(ctypes.byref(st.g), _p(st.nvert), _p(phi), _p(st.p))
    return phi


def projection(st, phi):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    lib().og_projection(ctypes.byref(st.g), ctypes.byref(st.om), _p(st.nvert), _p(phi), _p(st.ucont))


def divergence(st):
    return lib().og_divergence(ctypes.byref(st.g), _p(st.ucont), _p(st.m["aj"]), _p(st.nvert))


def les(st, ti=5, tistart=0, rstart=0, max_cs=0.5, cs=None):
    """Compute_Smagorinsky_Constant_1 + Compute_eddy_viscosity_LES (les.c:67-1252) on the
    state's Ucat; returns Cs and updates st.nut in place."""
    cs = np.zeros(st.case.da_shape) if cs is None else np.array(cs, dtype=np.float64)
    lib().og_les(ctypes.byref(st.g), _p(st.ucat), _p(st.m["csi"]), _p(st.m["eta"]), _p(st.m["zet"]),
                 _p(st.m["aj"]), _p(st.nvert), ctypes.c_int(ti), ctypes.c_int(tistart), ctypes.c_int(rstart),
                 ctypes.c_double(max_cs), _p(cs), _p(st.nut))
    return cs
