"""Synthetic inputs for the projection path, in the reference's input formats.

The reference ships no example grids, so every case is generated here with a fixed seed:
node coordinates as grid.dat stores them (IM x JM x KM nodes, x-, then y-, then z-block,
init.c:384-437), the six bcs.dat codes, periodic flags, the IB flag field nvert on the
DA (0 fluid, 1 IB node, 3 solid, as ibm_search_advanced leaves it: ibm.c:511-512), and
initial velocity fields.

Cases (streamwise direction k, as the reference forces periodic flow only along k,
momentum.c:382):
  * channel   - periodic in i and k, no-slip walls in j, tanh-stretched in y.
  * open_channel_cylinders - spanwise periodic, no-slip bottom, free-slip top, with a
    staggered array of vertical cylinders encoded in nvert.
"""
import numpy as np


class Case:
    def __init__(self, name, X, Y, Z, bctype, i_periodic=0, j_periodic=0, k_periodic=0,
                 immersed=0, les=0, ren=3000.0, dt=1e-3, st=1.0, inletprofile=13,
                 inlet_flux=-1.0):
        self.name = name
        self.X, self.Y, self.Z = X, Y, Z           # (KM, JM, IM) node arrays
        self.KM, self.JM, self.IM = X.shape
        self.bctype = list(bctype)
        self.i_periodic, self.j_periodic, self.k_periodic = i_periodic, j_periodic, k_periodic
        self.immersed, self.les = immersed, les
        self.ren, self.dt, self.st = ren, dt, st
        self.inletprofile, self.inlet_flux = inletprofile, inlet_flux
        self.wallfunction, self.moving = 0, 0
        self.implicit, self.imp_tol = 0, 1e-4
        self.roughness = 0.0
        self.nvert = np.zeros(self.da_shape)
        self.ucat0 = None

    @property
    def da_shape(self):
        return (self.KM + 1, self.JM + 1, self.IM + 1)

    def write_grid_dat(self, path):
        """grid.dat in the reference's ASCII form (init.c:336-437)."""
        with open(path, "w") as f:
            f.write("1\n%d %d %d\n" % (self.IM, self.JM, self.KM))
            for arr in (self.X, self.Y, self.Z):
                np.savetxt(f, arr.reshape(-1), fmt="%.17e")

    def write_bcs_dat(self, path):
        with open(path, "w") as f:
            f.write(" ".join(str(b) for b in self.bctype) + "\n")

    def config(self):
        from . import make_config
        return make_config(self.IM, self.JM, self.KM, self.bctype, self.i_periodic,
                           self.j_periodic, self.k_periodic, self.immersed, self.les,
                           self.inletprofile, self.ren, self.dt, self.st, self.inlet_flux,
                           wallfunction=self.wallfunction, moving=self.moving,
                           implicit=self.implicit, imp_tol=self.imp_tol, roughness=self.roughness)


def tanh_stretch(n, beta, lo, hi):
    """n+1 nodes on [lo, hi] clustered at both ends (tanh mapping with parameter beta)."""
    eta = np.linspace(-1.0, 1.0, n + 1)
    y = np.tanh(beta * eta) / np.tanh(beta)
    return lo + (hi - lo) * 0.5 * (y + 1.0)


def channel(nx=64, ny=64, nz=64, beta=2.0, Lx=np.pi, Ly=2.0, Lz=2 * np.pi, re_b=5600.0,
            dt=1e-3, wavy=0.0):
    """Periodic channel: nx*ny*nz cells, walls at y=0 and y=Ly (bctype 1), periodic i and k.

    With wavy > 0 the bottom wall is y_w = wavy*sin(2 pi x/Lx)*cos(2 pi z/Lz) and the
    nodes follow y = y_w + eta*(Ly - y_w) (curvilinear case)."""
    x = np.linspace(0.0, Lx, nx + 1)
    yh = tanh_stretch(ny, beta, 0.0, Ly)
    z = np.linspace(0.0, Lz, nz + 1)
    Z, Y, X = np.meshgrid(z, yh, x, indexing="ij")
    if wavy:
        yw = wavy * np.sin(2 * np.pi * X / Lx) * np.cos(2 * np.pi * Z / Lz)
        Y = yw + (Y / Ly) * (Ly - yw)
    # bctype 7: periodic face (no boundary treatment of its own)
    c = Case("channel%dx%dx%d" % (nx, ny, nz), X, Y, Z, [7, 7, 1, 1, 7, 7], i_periodic=1,
             k_periodic=1, ren=re_b / 2.0, dt=dt, inletprofile=13)
    c.Ly = Ly
    return c


def cylinders_nvert(case, centers, radius):
    """nvert of vertical (y-aligned) cylinders: 3 inside, 1 on cells whose 3x3x3
    neighbourhood touches an inside cell (the near-boundary marking of ibm.c:322-345
    followed by the 2->1, 4->3 remap of ibm.c:511-512), 0 elsewhere.  Cell centres are
    the 8-node averages (metrics.c:82-101)."""
    X, Y, Z = case.X, case.Y, case.Z
    KM, JM, IM = X.shape
    xc = 0.125 * sum(X[a:KM - 1 + a, b:JM - 1 + b, c:IM - 1 + c] for a in (0, 1) for b in (0, 1) for c in (0, 1))
    zc = 0.125 * sum(Z[a:KM - 1 + a, b:JM - 1 + b, c:IM - 1 + c] for a in (0, 1) for b in (0, 1) for c in (0, 1))
    inside = np.zeros(xc.shape, dtype=bool)
    for (cx, cz) in centers:
        inside |= (xc - cx) ** 2 + (zc - cz) ** 2 < radius ** 2
    nv = np.zeros(case.da_shape)
    core = nv[1:-1, 1:-1, 1:-1]
    near = np.zeros_like(inside)
    pad = np.pad(inside, 1)
    for a in range(3):
        for b in range(3):
            for c in range(3):
                near |= pad[a:a + inside.shape[0], b:b + inside.shape[1], c:c + inside.shape[2]]
    core[near] = 1.0
    core[inside] = 3.0
    return nv


def open_channel_cylinders(nx=256, ny=192, nz=256, Lx=3.2, Ly=1.0, Lz=8.0, D=0.2, dt=5e-4,
                           ren=1e4, beta=1.5, wavy=0.0):
    """Open channel with a staggered 3x2 array of vertical cylinders (D, spacing 4D):
    spanwise periodic (i), no-slip bottom (j-: 1), free-slip top (j+: 10), streamwise
    periodic k with the bulk flux held by the k-periodic forcing (momentum.c:382-399).
    With wavy > 0 the bottom is y_w = wavy*sin(2 pi x/Lx)*cos(2 pi z/Lz) and the nodes
    follow y = y_w + eta*(Ly - y_w) (curvilinear)."""
    x = np.linspace(0.0, Lx, nx + 1)
    eta = np.linspace(0.0, 1.0, ny + 1)
    y = Ly * (1.0 - np.tanh(beta * (1.0 - eta)) / np.tanh(beta))
    z = np.linspace(0.0, Lz, nz + 1)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    if wavy:
        yw = wavy * np.sin(2 * np.pi * X / Lx) * np.cos(2 * np.pi * Z / Lz)
        Y = yw + (Y / Ly) * (Ly - yw)
    c = Case("open_channel_cyl%dx%dx%d" % (nx, ny, nz), X, Y, Z, [7, 7, 1, 10, 7, 7],
             i_periodic=1, k_periodic=1, immersed=1, ren=ren, dt=dt, inletprofile=13)
    s = 4 * D
    z0 = 0.5 * Lz - s
    centers = []
    for row in range(3):          # 3 rows streamwise, 2 per row, staggered spanwise
        for col in range(2):
            xs = 0.5 * Lx + (col - 0.5) * s + (0.5 * s if row % 2 else 0.0) - 0.25 * s
            centers.append((xs, z0 + row * s))
    c.centers, c.D = centers, D
    c.nvert = cylinders_nvert(c, centers, 0.5 * D)
    c.Ly = Ly
    return c


def icosphere(center=(0.0, 0.0, 0.0), radius=0.5, level=3):
    """Closed triangulated sphere: an icosahedron subdivided `level` times (20*4**level
    triangles, outward-oriented), its vertices pushed onto the sphere.  Returns the vertex
    coordinates x, y, z and the (n_elmt, 3) array of 0-based vertex indices, the form the
    reference's surface reader leaves in IBMNodes (ibm_io.c:582-905)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    return v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), np.array(faces, dtype=np.int32)


def cylinder_surface(center, radius, y0, y1, n_theta=64, n_y=16):
    """Closed triangulated vertical cylinder (axis along y from y0 to y1, capped, outward
    oriented) around center = (x, z): vertex coordinates x, y, z and the (n_elmt, 3) array
    of 0-based vertex indices, like icosphere."""
    cx, cz = center
    th = 2 * np.pi * np.arange(n_theta) / n_theta
    ys = np.linspace(y0, y1, n_y + 1)
    xs, yy, zs = [], [], []
    for yv in ys:
        xs.extend(cx + radius * np.cos(th))
        yy.extend(np.full(n_theta, yv))
        zs.extend(cz + radius * np.sin(th))
    xs += [cx, cx]
    yy += [y0, y1]
    zs += [cz, cz]
    bot, top = len(xs) - 2, len(xs) - 1
    faces = []
    for r in range(n_y):
        for q in range(n_theta):
            a, b = r * n_theta + q, r * n_theta + (q + 1) % n_theta
            c, d = a + n_theta, b + n_theta
            # outward normal: (b - a) x (c - a) points away from the axis for this order
            faces.append((a, c, b))
            faces.append((b, c, d))
    for q in range(n_theta):
        a, b = q, (q + 1) % n_theta
        faces.append((bot, a, b))                      # bottom cap, normal -y
        c, d = n_y * n_theta + q, n_y * n_theta + (q + 1) % n_theta
        faces.append((top, d, c))                      # top cap, normal +y
    return (np.array(xs), np.array(yy), np.array(zs), np.array(faces, dtype=np.int32))


def write_ucd(path, x, y, z, tri):
    """The surface in the reference's ibmdata UCD form (ibm_io.c:609-905): three header
    lines, 'n_v n_elmt 0 0 0', the vertices, then 1-based triangles."""
    with open(path, "w") as f:
        f.write("# UCD surface\n#\n#\n%d %d 0 0 0\n" % (len(x), len(tri)))
        for q in range(len(x)):
            f.write("%d %.17e %.17e %.17e\n" % (q + 1, x[q], y[q], z[q]))
        for e, (a, b, c) in enumerate(tri):
            f.write("%d 0 tri %d %d %d\n" % (e + 1, a + 1, b + 1, c + 1))


def inflow_outflow(case, inletprofile=100):
    """The same grid and bodies with an inlet on the k = 0 face (bctype 5) and an outlet on
    the k+ face (bctype 4) instead of streamwise periodicity (bcs.c:329, bcs.c:2285)."""
    case.bctype[4], case.bctype[5] = 5, 4
    case.k_periodic = 0
    case.inletprofile = inletprofile
    case.name += "_inout%d" % inletprofile
    return case


def inflow_plane(case, seed=0, intensity=0.05, ub=1.0):
    """A Cartesian inflow velocity plane (my, mx, 3) for inletprofile 100: the mean profile
    of initial_ucat's first interior k plane plus uniform noise of the given intensity."""
    u0 = initial_ucat(case, seed=seed, noise=0.0, ub=ub)[1]
    rng = np.random.Generator(np.random.Philox(seed + 101))
    return u0 + intensity * ub * (2.0 * rng.random(u0.shape) - 1.0)


def initial_ucat(case, seed=0, noise=0.1, ub=1.0):
    """Cartesian velocity on the DA cell centres: laminar parabola w = 1.5*Ub*y(2-y)/... in
    the streamwise (z) direction plus uniform noise in +-noise*Ub on all components from a
    counter-based generator with the given seed (numpy Philox)."""
    KM, JM, IM = case.X.shape
    shape = case.da_shape
    X, Y = case.X, case.Y
    yc = np.zeros(shape)
    yc[1:-1, 1:-1, 1:-1] = 0.125 * sum(Y[a:KM - 1 + a, b:JM - 1 + b, c:IM - 1 + c]
                                       for a in (0, 1) for b in (0, 1) for c in (0, 1))
    H = getattr(case, "Ly", 2.0)
    eta = np.clip(yc / H, 0.0, 1.0)
    w = 6.0 * ub * eta * (1.0 - eta)   # bulk velocity ub across the full height
    rng = np.random.Generator(np.random.Philox(seed))
    u = np.zeros(shape + (3,))
    u[..., 2] = w
    u[1:-1, 1:-1, 1:-1, :] += noise * ub * (2.0 * rng.random((KM - 1, JM - 1, IM - 1, 3)) - 1.0)
    u[case.nvert > 0.1] = 0.0
    return u


def ucont_from_ucat(case, ucat, m):
    """Face fluxes from the centre velocity: the average of the two adjacent cells dotted
    with the face metric (icsi, jeta, kzet), zero on faces touching a non-fluid cell or a
    non-periodic domain wall."""
    nv = case.nvert
    uc = np.zeros(case.da_shape + (3,))
    for comp, (met, ax) in enumerate(((m["icsi"], 2), (m["jeta"], 1), (m["kzet"], 0))):
        up = np.roll(ucat, -1, axis=ax)
        f = 0.5 * (ucat + up)
        val = (f * met).sum(-1)
        nvp = np.roll(nv, -1, axis=ax)
        val[(nv + nvp) > 0.1] = 0.0
        uc[..., comp] = val
    # only interior faces (ghost-plane values are filled by the periodic copies / BCs)
    mask = np.zeros(case.da_shape, dtype=bool)
    mask[1:-1, 1:-1, 1:-1] = True
    for comp, ax, per, bc_lo in ((0, 2, case.i_periodic, case.bctype[0]),
                                 (1, 1, case.j_periodic, case.bctype[2]),
                                 (2, 0, case.k_periodic, case.bctype[4])):
        v = uc[..., comp]
        v[~mask] = 0.0
        n = case.da_shape[ax]
        sl = [slice(None)] * 3
        sl[ax] = n - 2
        if not per:
            v[tuple(sl)] = 0.0          # face on the upper wall
    return uc
