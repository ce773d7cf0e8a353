"""Host-side binding of the B200 projection-path library (libvfs_b200.so).

The library is the product: hand-written sm_100a kernels behind the C ABI declared in
include/vfs_b200.h.  This module only loads it with ctypes and wraps the entry points in
a small class whose method names follow the reference functions they replace
(Formfunction_2, Contra2Cart, PoissonLHSNew, ...).  There is no CPU fallback: if the
shared library is missing or no B200 is present, construction raises.

Host arrays use the reference's layout: the DA of (IM+1) x (JM+1) x (KM+1) points,
[k][j][i] with i fastest, vector fields as interleaved {x,y,z} (numpy shape
(mz, my, mx, 3)).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libvfs_b200.so")

# field identifiers (include/vfs_b200.h)
UCONT, UCAT, P, PHI, NVERT, NU_T, RHS, DP, UCONT_O, UCAT_O, B, CENT = range(12)
CSI, ETA, ZET, AJ = 12, 13, 14, 15
ICSI, IETA, IZET, IAJ = 16, 17, 18, 19
JCSI, JETA, JZET, JAJ = 20, 21, 22, 23
KCSI, KETA, KZET, KAJ = 24, 25, 26, 27
CS = 28
USTAR = 29
RHS_O = 30
NFIELDS = 31
FIELD_DOF = [3, 3, 1, 1, 1, 1, 3, 3, 3, 3, 1, 3, 3, 3, 3, 1, 3, 3, 3, 1, 3, 3, 3, 1, 3, 3, 3, 1, 1, 1, 3]
METRIC_FIELDS = {
    "csi": CSI, "eta": ETA, "zet": ZET, "aj": AJ,
    "icsi": ICSI, "ieta": IETA, "izet": IZET, "iaj": IAJ,
    "jcsi": JCSI, "jeta": JETA, "jzet": JZET, "jaj": JAJ,
    "kcsi": KCSI, "keta": KETA, "kzet": KZET, "kaj": KAJ,
    "cent": CENT,
}

# scalars
(S_MEAN_K_FLUX, S_MEAN_K_AREA, S_INLET_FLUX, S_INLET_AREA, S_DT, S_REN, S_ST, S_TI, S_FLUX_IN, S_FLUX_OUT,
 S_IB_UNRESOLVED, S_NBODIES) = range(12)

OK, ERR_INVALID, ERR_CUDA, ERR_NOT_CONVERGED, ERR_NO_DEVICE, ERR_STATE = range(6)


class VfsConfig(ctypes.Structure):
    _fields_ = [
        ("IM", ctypes.c_int), ("JM", ctypes.c_int), ("KM", ctypes.c_int),
        ("bctype", ctypes.c_int * 6),
        ("i_periodic", ctypes.c_int), ("j_periodic", ctypes.c_int), ("k_periodic", ctypes.c_int),
        ("immersed", ctypes.c_int), ("les", ctypes.c_int), ("inletprofile", ctypes.c_int),
        ("dynamic_freq", ctypes.c_int), ("tistart", ctypes.c_int), ("rstart", ctypes.c_int),
        ("wallfunction", ctypes.c_int), ("moving", ctypes.c_int), ("implicit", ctypes.c_int),
        ("reserved_i", ctypes.c_int * 2),
        ("ren", ctypes.c_double), ("dt", ctypes.c_double), ("st", ctypes.c_double),
        ("inlet_flux", ctypes.c_double), ("mean_pressure_gradient", ctypes.c_double),
        ("dpdz_set", ctypes.c_int), ("reserved_j", ctypes.c_int * 7),
        ("max_cs", ctypes.c_double), ("imp_tol", ctypes.c_double), ("roughness", ctypes.c_double),
        ("reserved_d", ctypes.c_double * 5),
    ]


class SolveOpts(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int), ("restart", ctypes.c_int), ("max_iter", ctypes.c_int),
        ("levels", ctypes.c_int), ("pre_smooth", ctypes.c_int), ("post_smooth", ctypes.c_int),
        ("coarse_iters", ctypes.c_int), ("zero_guess", ctypes.c_int), ("graph", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
        ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("reserved_d", ctypes.c_double * 4),
    ]


class SolveStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
        ("r0", ctypes.c_double), ("rfinal", ctypes.c_double), ("ms", ctypes.c_double),
        ("reserved", ctypes.c_double * 4),
    ]


class StepStats(ctypes.Structure):
    _fields_ = [
        ("max_div", ctypes.c_double), ("mean_k_flux", ctypes.c_double),
        ("poisson", SolveStats), ("ms", ctypes.c_double), ("reserved", ctypes.c_double * 4),
    ]


class NewtonStats(ctypes.Structure):
    _fields_ = [
        ("newton_iterations", ctypes.c_int), ("krylov_iterations", ctypes.c_int), ("converged", ctypes.c_int),
        ("reserved_i", ctypes.c_int), ("f0", ctypes.c_double), ("ffinal", ctypes.c_double),
        ("reserved", ctypes.c_double * 4),
    ]


class AdjointOpts(ctypes.Structure):
    _fields_ = [
        ("nsteps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("objective", ctypes.c_int),
        ("control", ctypes.c_int), ("reserved", ctypes.c_int * 4), ("solve", SolveOpts),
    ]


class AdjointStats(ctypes.Structure):
    _fields_ = [
        ("J", ctypes.c_double), ("ms_forward", ctypes.c_double), ("ms_adjoint", ctypes.c_double),
        ("recomputed_steps", ctypes.c_int), ("checkpoints", ctypes.c_int), ("tape_bytes", ctypes.c_longlong),
        ("poisson_iterations_forward", ctypes.c_double), ("poisson_iterations_adjoint", ctypes.c_double),
        ("reserved", ctypes.c_double * 2),
    ]


OBJ_KINETIC_ENERGY, OBJ_PRESSURE_DRAG, OBJ_DRAG = 0, 1, 2
CTRL_INITIAL_UCONT, CTRL_INFLOW_PLANE = 0, 1
OP_NAMES = ["contra2cart", "form_bcs_tail", "pressure_gradient", "volume_flux", "poisson_rhs",
            "update_pressure", "projection", "ib_bc", "ibm_interpolation"]
# operators whose adjoint is a hand-written kernel (VolumeFlux and IB_BC only without IB
# nodes); IB_BC and the IB-node interpolation with IB nodes are applied by measured matrices
OP_HANDWRITTEN = ["contra2cart", "form_bcs_tail", "pressure_gradient", "volume_flux", "poisson_rhs",
                  "update_pressure", "projection", "ib_bc"]

EXPORTS = [
    "vfs_create", "vfs_destroy", "vfs_last_error", "vfs_dims", "vfs_synchronize",
    "vfs_launch_count", "vfs_set_field", "vfs_get_field", "vfs_set_scalar", "vfs_get_scalar",
    "vfs_field_device_ptr", "vfs_contra2cart", "vfs_formfunction2", "vfs_pressure_gradient",
    "vfs_calc_k_flux", "vfs_runge_kutta", "vfs_poisson_lhs", "vfs_poisson_rhs",
    "vfs_poisson_solve", "vfs_poisson_apply", "vfs_update_pressure", "vfs_projection",
    "vfs_divergence", "vfs_step", "vfs_calc_inlet_area", "vfs_form_bcs", "vfs_ib_bc",
    "vfs_form_metrics", "vfs_volume_flux", "vfs_get_stream", "vfs_run_kernel",
    "vfs_smagorinsky_constant", "vfs_eddy_viscosity", "vfs_inflow_flux", "vfs_set_inflow_plane",
    "vfs_ibm_search", "vfs_ibm_list", "vfs_ibm_interpolation",
    "vfs_adjoint_setup", "vfs_objective", "vfs_tangent", "vfs_adjoint_gradient",
    "vfs_adjoint_op_info", "vfs_adjoint_op_check", "vfs_adjoint_op_measured",
    "vfs_petsc_vec_write", "vfs_petsc_vec_read", "vfs_restart_write", "vfs_restart_read",
    "vfs_ibm_set_velocity", "vfs_grid_read", "vfs_grid_write", "vfs_implicit_residual",
    "vfs_implicit_momentum",
]

GRID_ASCII, GRID_BINARY, GRID_XYZ = 0, 1, 2

_lib = None


def petsc_vec_write(path, values):
    """One vector in PETSc's binary Vec format (the reference's restart files)."""
    a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    lib = load_library()
    if lib.vfs_petsc_vec_write(os.fsencode(path), a.ctypes.data, a.size):
        raise VfsError(1, lib.vfs_last_error(None).decode())


def petsc_vec_read(path, n):
    """The n doubles of a PETSc binary Vec file."""
    out = np.empty(n)
    lib = load_library()
    if lib.vfs_petsc_vec_read(os.fsencode(path), out.ctypes.data, n):
        raise VfsError(1, lib.vfs_last_error(None).decode())
    return out


def grid_read(path, fmt=GRID_ASCII, block=0, cl=1.0, L_dim=1.0):
    """Node coordinates (x, y, z), each (KM, JM, IM), of one block of a grid.dat / xyz.dat
    file, as the reference's MG_Initial reads them (init.c:313-440)."""
    lib = load_library()
    d = [ctypes.c_int() for _ in range(3)]
    if lib.vfs_grid_read(os.fsencode(path), fmt, block, cl, L_dim, *[ctypes.byref(v) for v in d], None, None, None):
        raise VfsError(1, lib.vfs_last_error(None).decode())
    IM, JM, KM = (v.value for v in d)
    x, y, z = (np.empty((KM, JM, IM)) for _ in range(3))
    if lib.vfs_grid_read(os.fsencode(path), fmt, block, cl, L_dim, *[ctypes.byref(v) for v in d],
                         x.ctypes.data, y.ctypes.data, z.ctypes.data):
        raise VfsError(1, lib.vfs_last_error(None).decode())
    return x, y, z


def grid_write(path, x, y, z, fmt=GRID_ASCII):
    """One block of node coordinates (each (KM, JM, IM)) as grid.dat / xyz.dat."""
    lib = load_library()
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z)]
    KM, JM, IM = a[0].shape
    if lib.vfs_grid_write(os.fsencode(path), fmt, IM, JM, KM, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data):
        raise VfsError(1, lib.vfs_last_error(None).decode())


def load_library(path=None):
    """Load libvfs_b200.so (built in-tree by build.py), or the library at `path`, which the
    contexts created afterwards then use.  Raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libvfs_b200.so not built (%s); run __graft_entry__.build()" % p)
    lib = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.vfs_create.argtypes = [ctypes.POINTER(VfsConfig), ctypes.c_int, ctypes.POINTER(vp)]
    lib.vfs_destroy.argtypes = [vp]
    lib.vfs_last_error.argtypes = [vp]
    lib.vfs_last_error.restype = ctypes.c_char_p
    lib.vfs_dims.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                             ctypes.POINTER(ctypes.c_int)]
    lib.vfs_synchronize.argtypes = [vp]
    lib.vfs_launch_count.argtypes = [vp]
    lib.vfs_launch_count.restype = ctypes.c_longlong
    lib.vfs_set_field.argtypes = [vp, ctypes.c_int, vp]
    lib.vfs_get_field.argtypes = [vp, ctypes.c_int, vp]
    lib.vfs_set_scalar.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    lib.vfs_get_scalar.argtypes = [vp, ctypes.c_int, dp]
    lib.vfs_field_device_ptr.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    for n in ("vfs_contra2cart", "vfs_pressure_gradient", "vfs_runge_kutta", "vfs_poisson_lhs",
              "vfs_poisson_rhs", "vfs_update_pressure", "vfs_projection", "vfs_calc_inlet_area",
              "vfs_ib_bc", "vfs_volume_flux", "vfs_smagorinsky_constant",
              "vfs_eddy_viscosity", "vfs_inflow_flux", "vfs_ibm_interpolation"):
        getattr(lib, n).argtypes = [vp]
    lib.vfs_formfunction2.argtypes = [vp, ctypes.c_double]
    lib.vfs_form_bcs.argtypes = [vp, ctypes.c_int]
    lib.vfs_set_inflow_plane.argtypes = [vp, vp]
    lib.vfs_ibm_search.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, vp]
    lib.vfs_ibm_list.argtypes = [vp, vp, vp, ctypes.c_int]
    lib.vfs_ibm_set_velocity.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    lib.vfs_calc_k_flux.argtypes = [vp, dp]
    lib.vfs_divergence.argtypes = [vp, dp]
    lib.vfs_poisson_solve.argtypes = [vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveStats)]
    lib.vfs_poisson_apply.argtypes = [vp, vp, vp]
    lib.vfs_step.argtypes = [vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(StepStats)]
    lib.vfs_form_metrics.argtypes = [vp, vp, vp, vp]
    lib.vfs_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.vfs_run_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.vfs_adjoint_setup.argtypes = [vp]
    lib.vfs_objective.argtypes = [vp, ctypes.POINTER(AdjointOpts), dp]
    lib.vfs_tangent.argtypes = [vp, ctypes.POINTER(AdjointOpts), vp, dp, dp]
    lib.vfs_adjoint_gradient.argtypes = [vp, ctypes.POINTER(AdjointOpts), vp, ctypes.POINTER(AdjointStats)]
    lib.vfs_adjoint_op_info.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), vp,
                                        ctypes.POINTER(ctypes.c_longlong)]
    lib.vfs_adjoint_op_check.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp]
    lib.vfs_adjoint_op_measured.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.vfs_petsc_vec_write.argtypes = [ctypes.c_char_p, vp, ctypes.c_longlong]
    lib.vfs_petsc_vec_read.argtypes = [ctypes.c_char_p, vp, ctypes.c_longlong]
    lib.vfs_restart_write.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    lib.vfs_restart_read.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    lib.vfs_implicit_residual.argtypes = [vp]
    lib.vfs_implicit_momentum.argtypes = [vp, ctypes.POINTER(NewtonStats)]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.vfs_grid_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ip, ip, ip, vp, vp, vp]
    lib.vfs_grid_write.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    _lib = lib
    return lib


class VfsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("vfs error %d: %s" % (code, msg))
        self.code = code


class Context:
    """One structured block on one GPU (vfs_ctx)."""

    def __init__(self, cfg: VfsConfig, device=0):
        self.lib = load_library()
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = self.lib.vfs_create(ctypes.byref(cfg), device, ctypes.byref(h))
        if rc:
            raise VfsError(rc, self.lib.vfs_last_error(None).decode())
        self.h = h
        mx, my, mz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.vfs_dims(h, ctypes.byref(mx), ctypes.byref(my), ctypes.byref(mz))
        self.shape = (mz.value, my.value, mx.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.vfs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, allow=()):
        if rc and rc not in allow:
            raise VfsError(rc, self.lib.vfs_last_error(self.h).decode())
        return rc

    # ---- fields
    def set_field(self, field, arr):
        dof = FIELD_DOF[field]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        want = int(np.prod(self.shape)) * dof
        if a.size != want:
            raise ValueError("field %d: expected %d values, got %d" % (field, want, a.size))
        self._check(self.lib.vfs_set_field(self.h, field, a.ctypes.data))

    def get_field(self, field, out=None):
        """Field in the reference layout; written into `out` (C-contiguous float64 of the
        field's shape, e.g. pinned memory) when given."""
        dof = FIELD_DOF[field]
        shape = self.shape + ((3,) if dof == 3 else ())
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        elif out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("get_field: out must be C-contiguous float64 of shape %s" % (shape,))
        self._check(self.lib.vfs_get_field(self.h, field, out.ctypes.data))
        return out

    def set_metrics(self, m):
        """m: dict name -> array (names of METRIC_FIELDS)."""
        for name, fid in METRIC_FIELDS.items():
            if name in m:
                self.set_field(fid, m[name])

    def form_metrics(self, X, Y, Z):
        """FormMetrics on the device from grid.dat node arrays of shape (KM, JM, IM)."""
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (X, Y, Z)]
        self._check(self.lib.vfs_form_metrics(self.h, xs[0].ctypes.data, xs[1].ctypes.data,
                                              xs[2].ctypes.data))

    def set_scalar(self, which, v):
        self._check(self.lib.vfs_set_scalar(self.h, which, float(v)))

    def get_scalar(self, which):
        v = ctypes.c_double()
        self._check(self.lib.vfs_get_scalar(self.h, which, ctypes.byref(v)))
        return v.value

    def stream(self):
        """Address of the context's cudaStream_t."""
        s = ctypes.c_void_p()
        self._check(self.lib.vfs_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def run_kernel(self, which, reps=1):
        self._check(self.lib.vfs_run_kernel(self.h, which, reps))

    def launch_count(self):
        return self.lib.vfs_launch_count(self.h)

    def synchronize(self):
        self._check(self.lib.vfs_synchronize(self.h))

    def ibm_search(self, x, y, z, tri, ibi=0):  # ibm_search_advanced, ibm.c:85
        """nvert flags of a closed triangulated surface (vertices x, y, z; (n, 3) 0-based
        triangles); returns the new nvert field."""
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        t = np.ascontiguousarray(tri, dtype=np.int32)
        cols = [np.ascontiguousarray(t[:, q]) for q in range(3)]
        self._check(self.lib.vfs_ibm_search(self.h, ibi, len(xs[0]), xs[0].ctypes.data, xs[1].ctypes.data,
                                            xs[2].ctypes.data, len(t), cols[0].ctypes.data, cols[1].ctypes.data,
                                            cols[2].ctypes.data))
        return self.get_field(NVERT)

    def ibm_set_velocity(self, u, v, w, ibi=0):  # ibm->u (surface velocity of the vertices)
        a = [np.ascontiguousarray(t, dtype=np.float64) for t in (u, v, w)]
        self._check(self.lib.vfs_ibm_set_velocity(self.h, ibi, len(a[0]), a[0].ctypes.data, a[1].ctypes.data,
                                                  a[2].ctypes.data))

    def ibm_list(self):
        """The IB-node list: ints (n, 14) i j k cell imode i1 j1 k1 i2 j2 k2 i3 j3 k3 and
        doubles (n, 8) cr1..3 cs1..3 d_s d_i."""
        n = self.lib.vfs_ibm_list(self.h, None, None, 0)
        if n < 0:
            self._check(-n)
        ints = np.zeros((n, 14), dtype=np.int32)
        dbls = np.zeros((n, 8))
        self.lib.vfs_ibm_list(self.h, ints.ctypes.data, dbls.ctypes.data, n)
        return ints, dbls

    def ibm_interpolation(self):      # ibm_interpolation_advanced, ibm.c:3294
        self._check(self.lib.vfs_ibm_interpolation(self.h))

    # ---- operators (reference names in comments)
    def contra2cart(self):            # Contra2Cart, rhs.c:27
        self._check(self.lib.vfs_contra2cart(self.h))

    def formfunction2(self, scale=1.0):  # Formfunction_2, momentum.c:456
        self._check(self.lib.vfs_formfunction2(self.h, scale))

    def pressure_gradient(self):      # Pressure_Gradient, momentum.c:197
        self._check(self.lib.vfs_pressure_gradient(self.h))

    def calc_k_flux(self):            # Calc_k_Flux, rhs2.c:1562
        v = ctypes.c_double()
        self._check(self.lib.vfs_calc_k_flux(self.h, ctypes.byref(v)))
        return v.value

    def calc_inlet_area(self):        # Calc_Inlet_Area, bcs.c:216
        self._check(self.lib.vfs_calc_inlet_area(self.h))
        return self.get_scalar(S_MEAN_K_AREA), self.get_scalar(S_INLET_AREA)

    def form_bcs(self, outflow_scale=1):  # FormBCS, bcs.c:1841
        self._check(self.lib.vfs_form_bcs(self.h, int(outflow_scale)))

    def inflow_flux(self):            # InflowFlux, bcs.c:329
        self._check(self.lib.vfs_inflow_flux(self.h))
        return self.get_scalar(S_FLUX_IN)

    def set_inflow_plane(self, plane):  # ucont_plane (read_inflow_section, rhs2.c:701)
        a = np.ascontiguousarray(plane, dtype=np.float64)
        if a.size != self.shape[1] * self.shape[2] * 3:
            raise ValueError("inflow plane: expected my*mx*3 values")
        self._check(self.lib.vfs_set_inflow_plane(self.h, a.ctypes.data))

    def volume_flux(self):            # VolumeFlux, poisson.c:3306 (immersed = 0) / 3570 (immersed = 1)
        self._check(self.lib.vfs_volume_flux(self.h))

    def ib_bc(self):                  # IB_BC, momentum.c:1982
        self._check(self.lib.vfs_ib_bc(self.h))

    def smagorinsky_constant(self):   # Compute_Smagorinsky_Constant_1, les.c:67
        self._check(self.lib.vfs_smagorinsky_constant(self.h))

    def eddy_viscosity(self):         # Compute_eddy_viscosity_LES, les.c:1135
        self._check(self.lib.vfs_eddy_viscosity(self.h))

    def runge_kutta(self):            # RungeKutta, rhs.c:1578
        self._check(self.lib.vfs_runge_kutta(self.h))

    def poisson_lhs(self):            # PoissonLHSNew, poisson.c:971
        self._check(self.lib.vfs_poisson_lhs(self.h))

    def poisson_rhs(self):            # PoissonRHS2 (+ Remove_Nullspace_Scale)
        self._check(self.lib.vfs_poisson_rhs(self.h))

    def poisson_apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.shape)
        y = np.empty_like(x)
        self._check(self.lib.vfs_poisson_apply(self.h, x.ctypes.data, y.ctypes.data))
        return y

    def poisson_solve(self, precision=0, rtol=1e-10, restart=30, max_iter=200, levels=0,
                      pre_smooth=3, post_smooth=3, coarse_iters=4, allow_unconverged=False, zero_guess=0):
        o = SolveOpts(precision=precision, restart=restart, max_iter=max_iter, levels=levels,
                      pre_smooth=pre_smooth, post_smooth=post_smooth, coarse_iters=coarse_iters,
                      rtol=rtol, zero_guess=zero_guess)
        st = SolveStats()
        allow = (ERR_NOT_CONVERGED,) if allow_unconverged else ()
        self._check(self.lib.vfs_poisson_solve(self.h, ctypes.byref(o), ctypes.byref(st)), allow)
        return st

    def update_pressure(self):        # UpdatePressure, poisson.c:3144
        self._check(self.lib.vfs_update_pressure(self.h))

    def projection(self):             # Projection, poisson.c:2707
        self._check(self.lib.vfs_projection(self.h))

    def divergence(self):             # Divergence, main.c:1047
        v = ctypes.c_double()
        self._check(self.lib.vfs_divergence(self.h, ctypes.byref(v)))
        return v.value

    def restart_write(self, directory, ti, block=0):  # Ucont_P_Binary_Output, main.c:765
        self._check(self.lib.vfs_restart_write(self.h, os.fsencode(directory), ti, block))

    def restart_read(self, directory, ti, block=0):   # Ucont_P_Binary_Input, main.c:394
        self._check(self.lib.vfs_restart_read(self.h, os.fsencode(directory), ti, block))

    def step(self, precision=0, rtol=1e-10, **kw):  # Flow_Solver, solvers.c:562 (implicit=0)
        o = _solve_opts(precision, rtol, **kw)
        st = StepStats()
        self._check(self.lib.vfs_step(self.h, ctypes.byref(o), ctypes.byref(st)))
        return st

    def implicit_residual(self):  # FormFunction_SNES, momentum.c:2197
        self._check(self.lib.vfs_implicit_residual(self.h))

    def implicit_momentum(self):  # Implicit_MatrixFree, implicitsolver.c:4196
        st = NewtonStats()
        self._check(self.lib.vfs_implicit_momentum(self.h, ctypes.byref(st)))
        return st

    # ---- tangent-linear and adjoint of a window of steps (no reference counterpart)
    def _adj_opts(self, nsteps, objective, control, checkpoint_every, precision, rtol, kw):
        return AdjointOpts(nsteps=nsteps, checkpoint_every=checkpoint_every, objective=objective,
                           control=control, solve=_solve_opts(precision, rtol, **kw))

    def control_shape(self, control):
        if control == CTRL_INFLOW_PLANE:
            return (self.shape[1], self.shape[2], 3)
        return self.shape + (3,)

    def adjoint_setup(self):
        self._check(self.lib.vfs_adjoint_setup(self.h))

    def objective(self, nsteps, objective=OBJ_KINETIC_ENERGY, control=CTRL_INITIAL_UCONT, checkpoint_every=0,
                  precision=1, rtol=1e-12, **kw):
        """J after nsteps steps from the current state (the state is kept)."""
        o = self._adj_opts(nsteps, objective, control, checkpoint_every, precision, rtol, kw)
        J = ctypes.c_double()
        self._check(self.lib.vfs_objective(self.h, ctypes.byref(o), ctypes.byref(J)))
        return J.value

    def tangent(self, direction, nsteps, objective=OBJ_KINETIC_ENERGY, control=CTRL_INITIAL_UCONT,
                precision=1, rtol=1e-12, **kw):
        """(J, dJ) with dJ the derivative of J along direction (the control's shape)."""
        o = self._adj_opts(nsteps, objective, control, 0, precision, rtol, kw)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        if d.shape != self.control_shape(control):
            raise ValueError("direction must have shape %s" % (self.control_shape(control),))
        J, dJ = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.vfs_tangent(self.h, ctypes.byref(o), d.ctypes.data, ctypes.byref(J), ctypes.byref(dJ)))
        return J.value, dJ.value

    def adjoint_gradient(self, nsteps, objective=OBJ_KINETIC_ENERGY, control=CTRL_INITIAL_UCONT,
                         checkpoint_every=0, precision=1, rtol=1e-12, **kw):
        """(gradient of J with respect to the control, AdjointStats)."""
        o = self._adj_opts(nsteps, objective, control, checkpoint_every, precision, rtol, kw)
        g = np.zeros(self.control_shape(control))
        st = AdjointStats()
        self._check(self.lib.vfs_adjoint_gradient(self.h, ctypes.byref(o), g.ctypes.data, ctypes.byref(st)))
        return g, st

    def adjoint_op_info(self, op):
        n = ctypes.c_int()
        fields = (ctypes.c_int * 20)()
        nnz = ctypes.c_longlong()
        self._check(self.lib.vfs_adjoint_op_info(self.h, op, ctypes.byref(n), fields, ctypes.byref(nnz)))
        return [(fields[2 * s], fields[2 * s + 1]) for s in range(n.value)], nnz.value

    def adjoint_op_check(self, op, x, y):
        """(L x by the operator's kernels, L^T y by the transpose the adjoint sweep applies:
        hand-written for OP_HANDWRITTEN, else the measured matrix); x, y: slots x N."""
        slots, _ = self.adjoint_op_info(op)
        N = int(np.prod(self.shape))
        a = np.ascontiguousarray(x, dtype=np.float64).reshape(len(slots), N)
        b = np.ascontiguousarray(y, dtype=np.float64).reshape(len(slots), N)
        lx = np.zeros_like(a)
        lty = np.zeros_like(b)
        self._check(self.lib.vfs_adjoint_op_check(self.h, op, a.ctypes.data, b.ctypes.data, lx.ctypes.data,
                                                  lty.ctypes.data))
        return lx, lty

    def adjoint_op_measured(self, op, y):
        """L^T y by the operator's measured matrix (y: slots x N)."""
        slots, _ = self.adjoint_op_info(op)
        N = int(np.prod(self.shape))
        b = np.ascontiguousarray(y, dtype=np.float64).reshape(len(slots), N)
        lty = np.zeros_like(b)
        self._check(self.lib.vfs_adjoint_op_measured(self.h, op, b.ctypes.data, lty.ctypes.data))
        return lty


def _solve_opts(precision=0, rtol=1e-10, **kw):
    return SolveOpts(precision=precision, rtol=rtol, restart=kw.get("restart", 30),
                     max_iter=kw.get("max_iter", 200), levels=kw.get("levels", 0),
                     pre_smooth=kw.get("pre_smooth", 3), post_smooth=kw.get("post_smooth", 3),
                     coarse_iters=kw.get("coarse_iters", 4), zero_guess=kw.get("zero_guess", 0),
                     graph=kw.get("graph", 0))


def make_config(IM, JM, KM, bctype, i_periodic=0, j_periodic=0, k_periodic=0, immersed=0, les=0,
                inletprofile=13, ren=3000.0, dt=0.04, st=1.0, inlet_flux=-1.0,
                mean_pressure_gradient=0.0, dpdz_set=0, dynamic_freq=1, tistart=0, rstart=0,
                max_cs=0.5, wallfunction=0, moving=0, implicit=0, imp_tol=1e-4, roughness=0.0):
    c = VfsConfig()
    c.IM, c.JM, c.KM = IM, JM, KM
    for q in range(6):
        c.bctype[q] = bctype[q]
    c.i_periodic, c.j_periodic, c.k_periodic = i_periodic, j_periodic, k_periodic
    c.immersed, c.les, c.inletprofile = immersed, les, inletprofile
    c.ren, c.dt, c.st = ren, dt, st
    c.inlet_flux, c.mean_pressure_gradient, c.dpdz_set = inlet_flux, mean_pressure_gradient, dpdz_set
    c.dynamic_freq, c.tistart, c.rstart, c.max_cs = dynamic_freq, tistart, rstart, max_cs
    c.wallfunction, c.moving = wallfunction, moving
    c.implicit, c.imp_tol, c.roughness = implicit, imp_tol, roughness
    return c
