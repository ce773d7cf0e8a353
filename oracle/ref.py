"""ctypes wrapper of oracle/_ref/libvfsref.so — the reference's own hot-path sources
compiled against the single-rank PETSc shim (see oracle/build_ref.py).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, to compare against.  Never part of the product path.

The reference keeps its run options in C globals (main.c:1-393); they are plain symbols
of the library and are set here by name before each set-up.  One Reference instance
drives the library's single UserCtx at a time.
"""
import ctypes
import os
import shutil
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libvfsref.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libvfsref.so is not built (oracle/build_ref.py)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.ref_setup.argtypes = [ctypes.c_char_p]
        L.ref_field_size.argtypes = [ctypes.c_char_p]
        L.ref_field_size.restype = ctypes.c_long
        L.ref_get_field.argtypes = [ctypes.c_char_p, vp]
        L.ref_set_field.argtypes = [ctypes.c_char_p, vp]
        L.ref_set_params.argtypes = [ctypes.c_double] * 3
        L.ref_get_params.argtypes = [ctypes.POINTER(ctypes.c_double)] * 3
        L.ref_set_bctype.argtypes = [vp]
        L.ref_get_bctype.argtypes = [vp]
        L.ref_get_kflux.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
        L.ref_set_kflux.argtypes = [ctypes.c_double] * 2
        L.ref_formfunction2.argtypes = [ctypes.c_double]
        L.ref_poisson_csr.argtypes = [vp, vp, vp, ctypes.POINTER(ctypes.c_int)]
        L.ref_poisson_csr.restype = ctypes.c_long
        L.ref_poisson_rhs2_hypre.argtypes = [vp]
        L.ref_remove_nullspace.argtypes = [vp, ctypes.c_int]
        L.ref_les.argtypes = [ctypes.c_int]
        L.ref_inlet_area.restype = ctypes.c_double
        L.ref_volume_flux.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
        L.ref_volume_flux_ibm.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
        L.ref_form_bcs_scaled.argtypes = [ctypes.c_int]
        L.ref_flux_in.restype = ctypes.c_double
        L.ref_set_inflow_plane.argtypes = [vp]
        L.ref_ibm_classify.argtypes = [ctypes.c_int] * 2 + [vp] * 3 + [ctypes.c_int] + [vp] * 3 + [ctypes.c_int]
        L.ref_ibm_list.argtypes = [ctypes.c_int, vp, vp, ctypes.c_int]
        L.ref_ibm_interpolation.argtypes = [ctypes.c_int]
        L.ref_ibm_set_velocity.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.ref_restart_output.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.ref_restart_input.argtypes = [ctypes.c_char_p, ctypes.c_int]
        _lib = L
    return _lib


INT_GLOBALS = ("i_periodic", "j_periodic", "k_periodic", "ii_periodic", "jj_periodic",
               "kk_periodic", "periodic", "les", "rans", "levelset", "immersed", "inletprofile",
               "poisson", "implicit", "ti", "tistart", "weno", "second_order", "central",
               "inviscid", "skew", "clark", "laplacian", "dpdz_set", "movefsi", "rotatefsi",
               "wallfunction", "pseudo_periodic", "conv_diff", "density_current", "sediment",
               "wave_momentum_source", "wave_sponge_layer", "surface_tension",
               "air_flow_levelset_periodic", "dynamic_freq", "testfilter_ik", "testfilter_1d",
               "i_homo_filter", "j_homo_filter", "k_homo_filter", "NumberOfBodies")
DBL_GLOBALS = ("inlet_flux", "mean_pressure_gradient", "max_cs", "roughness_size")


def set_global(name, value):
    L = lib()
    if name in DBL_GLOBALS:
        ctypes.c_double.in_dll(L, name).value = float(value)
    else:
        ctypes.c_int.in_dll(L, name).value = int(value)


def get_global(name):
    L = lib()
    if name in DBL_GLOBALS:
        return ctypes.c_double.in_dll(L, name).value
    return ctypes.c_int.in_dll(L, name).value


# Reference names of the metric vectors (variables.h:555-559), keyed like the product's.
METRIC_VECS = {"csi": "lCsi", "eta": "lEta", "zet": "lZet", "aj": "lAj",
               "icsi": "lICsi", "ieta": "lIEta", "izet": "lIZet", "iaj": "lIAj",
               "jcsi": "lJCsi", "jeta": "lJEta", "jzet": "lJZet", "jaj": "lJAj",
               "kcsi": "lKCsi", "keta": "lKEta", "kzet": "lKZet", "kaj": "lKAj",
               "cent": "lCent"}


class Reference:
    """The reference solver state for one synthetic case (grid.dat / bcs.dat written to a
    scratch directory and read by MG_Initial)."""

    def __init__(self, case, extra_globals=None, grid_writer=None):
        self.case = case
        L = lib()
        g = {"i_periodic": case.i_periodic, "j_periodic": case.j_periodic,
             "k_periodic": case.k_periodic, "ii_periodic": 0, "jj_periodic": 0, "kk_periodic": 0,
             "periodic": case.i_periodic + case.j_periodic + case.k_periodic,
             "les": case.les, "rans": 0, "levelset": 0, "immersed": case.immersed,
             "inletprofile": case.inletprofile, "poisson": 1, "implicit": 0, "ti": 0,
             "tistart": 0, "weno": 0, "second_order": 0, "central": 0, "inviscid": 0,
             "skew": 0, "clark": 0, "laplacian": 0, "dpdz_set": 0, "movefsi": 0,
             "rotatefsi": 0, "inlet_flux": case.inlet_flux, "NumberOfBodies": 1,
             "wallfunction": getattr(case, "wallfunction", 0),
             "rough_set": int(getattr(case, "roughness", 0.0) > 0),
             "roughness_size": getattr(case, "roughness", 0.0)}
        if getattr(case, "moving", 0):
            g["movefsi"] = 1
        if extra_globals:
            g.update(extra_globals)
        for k, v in g.items():
            set_global(k, v)
        self.dir = tempfile.mkdtemp(prefix="vfsref_")
        if grid_writer is None:
            case.write_grid_dat(os.path.join(self.dir, "grid.dat"))
        else:  # the caller writes grid.dat (or xyz.dat) into the directory
            grid_writer(self.dir)
        case.write_bcs_dat(os.path.join(self.dir, "bcs.dat"))
        if L.ref_setup(self.dir.encode()):
            raise RuntimeError("reference MG_Initial failed")
        mx, my, mz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.ref_dims(ctypes.byref(mx), ctypes.byref(my), ctypes.byref(mz))
        self.shape = (mz.value, my.value, mx.value)
        L.ref_set_params(case.ren, case.dt, case.st)
        self.set("lNvert", case.nvert)
        self.set("Nvert", case.nvert)
        # first-step set-up of main.c:3488 (mean k-face area, inlet area)
        L.ref_calc_inlet_area()

    def close(self):
        shutil.rmtree(self.dir, ignore_errors=True)

    def get(self, name):
        L = lib()
        n = L.ref_field_size(name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n)
        L.ref_get_field(name.encode(), out.ctypes.data)
        npts = int(np.prod(self.shape))
        if n == npts:
            return out.reshape(self.shape)
        if n == 3 * npts:
            return out.reshape(self.shape + (3,))
        return out

    def set(self, name, arr):
        L = lib()
        a = np.ascontiguousarray(arr, dtype=np.float64)
        n = L.ref_field_size(name.encode())
        if n != a.size:
            raise ValueError("%s: expected %d values, got %d" % (name, n, a.size))
        L.ref_set_field(name.encode(), a.ctypes.data)

    def metrics(self):
        return {k: self.get(v) for k, v in METRIC_VECS.items()}

    def call(self, fname, *args):
        rc = getattr(lib(), fname)(*args)
        if rc:
            raise RuntimeError("%s returned %d" % (fname, rc))

    def kflux(self):
        f, a = ctypes.c_double(), ctypes.c_double()
        lib().ref_get_kflux(ctypes.byref(f), ctypes.byref(a))
        return f.value, a.value

    def volume_flux(self):
        """VolumeFlux(user, Ucont, ...) (poisson.c:3306); returns (ibm_Flux, ibm_Area)."""
        f, a = ctypes.c_double(), ctypes.c_double()
        lib().ref_volume_flux(ctypes.byref(f), ctypes.byref(a))
        return f.value, a.value

    def volume_flux_ibm(self):
        """VolumeFlux(user, &ibm_Flux, &ibm_Area, 0) (poisson.c:3570), the immersed = 1 form;
        returns (ibm_Flux, ibm_Area)."""
        f, a = ctypes.c_double(), ctypes.c_double()
        lib().ref_volume_flux_ibm(ctypes.byref(f), ctypes.byref(a))
        return f.value, a.value

    def inlet_area(self):
        return lib().ref_inlet_area()

    def ibm_classify(self, x, y, z, tri, ibi=0, build_list=False):
        """The nvert flags of ibm_search_advanced (ibm.c:85) for body ibi, classified by the
        reference's own point_cell_advanced (see ref_driver.cpp), and with build_list its
        IB-node list from the reference's nearestcell1/InterceptionPoint; returns lNvert."""
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        t = np.ascontiguousarray(tri, dtype=np.int32)
        cols = [np.ascontiguousarray(t[:, q]) for q in range(3)]
        self.call("ref_ibm_classify", ibi, len(xs[0]), xs[0].ctypes.data, xs[1].ctypes.data, xs[2].ctypes.data,
                  len(t), cols[0].ctypes.data, cols[1].ctypes.data, cols[2].ctypes.data, int(build_list))
        return self.get("lNvert")

    def ibm_set_velocity(self, u, v, w, ibi=0):
        """ibm->u of body ibi (the surface velocity of its vertices)."""
        a = [np.ascontiguousarray(t, dtype=np.float64) for t in (u, v, w)]
        self.call("ref_ibm_set_velocity", ibi, len(a[0]), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data)

    def ibm_list(self, ibi=0):
        """The IB-node list (ints (n, 14): i j k cell imode i1 j1 k1 i2 j2 k2 i3 j3 k3; doubles
        (n, 8): cr1..3 cs1..3 d_s d_i), in list order."""
        L = lib()
        n = L.ref_ibm_list(ibi, None, None, 0)
        ints = np.zeros((n, 14), dtype=np.int32)
        dbls = np.zeros((n, 8))
        L.ref_ibm_list(ibi, ints.ctypes.data, dbls.ctypes.data, n)
        return ints, dbls

    def flux_in(self):
        """FluxInSum after the last InflowFlux (bcs.c:778)."""
        return lib().ref_flux_in()

    def set_inflow_plane(self, plane):
        a = np.ascontiguousarray(plane, dtype=np.float64)
        lib().ref_set_inflow_plane(a.ctypes.data)

    def set_kflux(self, flux, area):
        lib().ref_set_kflux(flux, area)

    def restart_output(self, directory, ti):
        """Ucont_P_Binary_Output (main.c:765): the restart files of step ti in directory."""
        self.call("ref_restart_output", os.fsencode(directory), ti)

    def restart_input(self, directory, ti):
        """Ucont_P_Binary_Input (main.c:394): loads the restart files of step ti."""
        self.call("ref_restart_input", os.fsencode(directory), ti)

    def poisson_csr(self):
        L = lib()
        m = ctypes.c_int()
        nnz = L.ref_poisson_csr(None, None, None, ctypes.byref(m))
        rp = np.zeros(m.value + 1, dtype=np.int32)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        L.ref_poisson_csr(rp.ctypes.data, col.ctypes.data, val.ctypes.data, ctypes.byref(m))
        return rp, col, val

    def poisson_rhs_hypre(self):
        L = lib()
        n = L.ref_phi2_size()
        out = np.zeros(n)
        L.ref_poisson_rhs2_hypre(out.ctypes.data)
        return out

    def remove_nullspace(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        lib().ref_remove_nullspace(x.ctypes.data, x.size)
        return x

    def gid(self):
        """Compressed unknown index per DA point (-1 if none), as setup_lidx2 leaves it."""
        return self.get("Gid").astype(np.int64)
