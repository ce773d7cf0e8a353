"""CPU solve of the reference's own pressure-Poisson system, standing in for HYPRE.

TEST INFRASTRUCTURE ONLY: used by tests/, the golden-fixture scripts and bench.py's
reference arm to solve the matrix that PoissonLHSNew recorded (poisson.c:971-1683, the
CSR of the shim's Mat) with the right-hand side of PoissonRHS2_hypre
(poisson_hypre.c:330-360).  The reference hands this system to HYPRE 2.11.2 (BoomerAMG-
preconditioned GMRES, poisson_hypre.c:26-88, 498-620), which is not in this image; what
matters for parity is the converged solution of the reference's system, up to the
null-space constant that Remove_Nullspace (poisson_hypre.c:194) removes afterwards.

Method: right-preconditioned flexible GMRES (Saad 1993) on the CSR matrix, to a relative
true residual `rtol`, with one geometric multigrid V-cycle as the preconditioner:

* levels are the interior cells of the DA grid, coarsened by 2 per direction while every
  interior dimension is even and at least 4;
* the operator on each level is 7-point: on the finest level the conductance between a
  cell and its +i/+j/+k neighbour is the mean of the two matrix entries that couple them
  (clipped at zero), a coarse face conducts half the sum of the four fine faces it covers,
  and the diagonal is minus the sum of a cell's conductances;
* smoother: zebra line Gauss-Seidel along j (all j-lines of one colour solved at once by
  vectorised Thomas elimination), `sweeps` colour pairs before and after the coarse
  correction;
* restriction sums the residuals of the eight children; prolongation is separable
  cell-centred linear interpolation (weights 3/4, 1/4), a coarse neighbour beyond a
  non-periodic edge giving its weight to the parent;
* the coarsest level is solved with a pseudo-inverse (the Neumann/periodic operator is
  singular).

Set-up (`MGSolver(...)`) is done once per matrix, as HYPRE's set-up runs at PoissonLHSNew
time (poisson_hypre.c:527); `solve` may start from the previous solution, like the
reference's persistent Phi2 (poisson_hypre.c:571, 604).
"""
import numpy as np
import scipy.sparse as sp


class _Level:
    pass


def _pad_take(a, axis, shift, periodic):
    """a shifted by `shift` (+1: value of the +1 neighbour) along `axis`; at a
    non-periodic edge the missing neighbour is replaced by the cell itself."""
    if periodic:
        return np.roll(a, -shift, axis=axis)
    out = np.roll(a, -shift, axis=axis)
    idx = [slice(None)] * a.ndim
    idx[axis] = -1 if shift > 0 else 0
    out[tuple(idx)] = a[tuple(idx)]
    return out


class MGSolver:
    """FGMRES + geometric multigrid for the reference's Poisson CSR system.

    gid: DA-shaped (mz, my, mx) array of unknown numbers (-1: no unknown), as setup_lidx2
    leaves it (poisson.c:182-330); only interior points own unknowns.
    """

    def __init__(self, rp, col, val, gid, periodic=(0, 0, 0), sweeps=2):
        n = len(rp) - 1
        self.A = sp.csr_matrix((val, col, rp), shape=(n, n))
        self.n = n
        self.sweeps = sweeps
        inner = gid[1:-1, 1:-1, 1:-1]
        self.own = inner >= 0            # (nz, ny, nx) cells with an unknown
        self.idx = inner[self.own]       # their unknown numbers
        self.ip, self.jp, self.kp = periodic
        self.levels = []
        self._build(inner)

    # ------------------------------------------------------------------ set-up
    def _fine_couplings(self, inner):
        A = self.A
        nz, ny, nx = inner.shape
        cs = []
        for axis, per in ((2, self.ip), (1, self.jp), (0, self.kp)):
            nb = np.roll(inner, -1, axis=axis)
            ok = (inner >= 0) & (nb >= 0)
            if not per:
                idx = [slice(None)] * 3
                idx[axis] = -1
                ok[tuple(idx)] = False
            r = inner[ok]
            c = nb[ok]
            a1 = np.asarray(A[r, c]).ravel()
            a2 = np.asarray(A[c, r]).ravel()
            cond = np.zeros(inner.shape)
            cond[ok] = np.maximum(0.0, 0.5 * (a1 + a2))
            cs.append(cond)
        return cs   # conductances to +i, +j, +k

    def _build(self, inner):
        ce, cn, ct = self._fine_couplings(inner)
        act = inner >= 0
        while True:
            L = _Level()
            L.ce, L.cn, L.ct, L.act = ce, cn, ct, act
            L.shape = ce.shape
            self._finish_level(L)
            self.levels.append(L)
            nz, ny, nx = L.shape
            if not all(d % 2 == 0 and d >= 4 for d in (nx, ny, nz)):
                break
            # coarse conductances: half the sum of the four fine faces across a coarse face
            ce = 0.5 * L.ce[:, :, 1::2].reshape(nz // 2, 2, ny // 2, 2, nx // 2).sum(axis=(1, 3))
            cn = 0.5 * L.cn[:, 1::2, :].reshape(nz // 2, 2, ny // 2, nx // 2, 2).sum(axis=(1, 4))
            ct = 0.5 * L.ct[1::2, :, :].reshape(nz // 2, ny // 2, 2, nx // 2, 2).sum(axis=(2, 4))
            act = act.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).any(axis=(1, 3, 5))
        Lc = self.levels[-1]
        Lc.dense_pinv = np.linalg.pinv(self._dense(Lc)) if Lc.ce.size <= 4096 else None

    def _finish_level(self, L):
        # conductances to the -1 neighbours and the diagonal
        L.cw = np.roll(L.ce, 1, axis=2)
        L.cs = np.roll(L.cn, 1, axis=1)
        L.cb = np.roll(L.ct, 1, axis=0)
        if not self.ip:
            L.cw[:, :, 0] = 0
        if not self.jp:
            L.cs[:, 0, :] = 0
        if not self.kp:
            L.cb[0, :, :] = 0
        L.dg = -(L.ce + L.cw + L.cn + L.cs + L.ct + L.cb)
        nz, ny, nx = L.shape
        kk, ii = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        L.colour = ((ii ^ kk) & 1)     # (nz, nx)
        # Thomas factors of every j-line (in-line couplings; a periodic j wrap is treated
        # by the right-hand side)
        cpr = np.zeros(L.shape)
        iden = np.zeros(L.shape)
        prev = np.zeros((nz, nx))
        lower = np.zeros((nz, nx))
        for j in range(ny):
            dg = L.dg[:, j, :]
            upper = L.cn[:, j, :] if j + 1 < ny else np.zeros((nz, nx))
            den = dg - lower * prev
            good = (dg != 0) & (np.abs(den) > 1e-12 * np.abs(dg))
            iden[:, j, :] = np.where(good, 1.0 / np.where(good, den, 1.0), 0.0)
            cpr[:, j, :] = upper * iden[:, j, :]
            prev = cpr[:, j, :]
            lower = upper
        L.cpr, L.iden = cpr, iden

    def _dense(self, L):
        nz, ny, nx = L.shape
        m = nz * ny * nx
        D = np.zeros((m, m))
        num = np.arange(m).reshape(L.shape)
        for c, axis, per in ((L.ce, 2, self.ip), (L.cn, 1, self.jp), (L.ct, 0, self.kp)):
            nb = np.roll(num, -1, axis=axis)
            ok = c != 0
            r, q, w = num[ok], nb[ok], c[ok]
            D[r, q] += w
            D[q, r] += w
        D[num.ravel(), num.ravel()] += L.dg.ravel()
        return D

    # ------------------------------------------------------------------ operators
    def _apply(self, L, x):
        y = L.dg * x
        y += L.ce * _pad_take(x, 2, 1, self.ip) + L.cw * _pad_take(x, 2, -1, self.ip)
        y += L.cn * _pad_take(x, 1, 1, self.jp) + L.cs * _pad_take(x, 1, -1, self.jp)
        y += L.ct * _pad_take(x, 0, 1, self.kp) + L.cb * _pad_take(x, 0, -1, self.kp)
        return y

    def _smooth(self, L, x, b):
        nz, ny, nx = L.shape
        for colour in (0, 1):
            sel = L.colour == colour                     # (nz, nx)
            r = b - L.ce * _pad_take(x, 2, 1, self.ip) - L.cw * _pad_take(x, 2, -1, self.ip) \
                - L.ct * _pad_take(x, 0, 1, self.kp) - L.cb * _pad_take(x, 0, -1, self.kp)
            if self.jp:
                r[:, 0, :] -= L.cs[:, 0, :] * x[:, -1, :]
                r[:, -1, :] -= L.cn[:, -1, :] * x[:, 0, :]
            # forward elimination and back substitution along j for this colour's lines
            rs = r.transpose(1, 0, 2)[:, sel]             # (ny, ncol)
            cpr = L.cpr.transpose(1, 0, 2)[:, sel]
            iden = L.iden.transpose(1, 0, 2)[:, sel]
            low = L.cs.transpose(1, 0, 2)[:, sel]
            d = np.empty_like(rs)
            prev = np.zeros(rs.shape[1])
            for j in range(ny):
                lo = low[j] if j > 0 else 0.0
                prev = (rs[j] - lo * prev) * iden[j]
                d[j] = prev
            for j in range(ny - 2, -1, -1):
                d[j] -= cpr[j] * d[j + 1]
            xt = x.transpose(1, 0, 2)
            xt[:, sel] = d
        return x

    def _restrict(self, L, r):
        nz, ny, nx = L.shape
        return r.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).sum(axis=(1, 3, 5))

    def _prolong(self, Lc, e):
        per = (self.kp, self.jp, self.ip)
        out = e
        for axis in (0, 1, 2):
            lo = _pad_take(out, axis, -1, per[axis])
            hi = _pad_take(out, axis, 1, per[axis])
            out = np.stack((0.75 * out + 0.25 * lo, 0.75 * out + 0.25 * hi), axis=axis + 1)
            shp = list(out.shape)
            shp[axis] *= 2
            del shp[axis + 1]
            out = out.reshape(shp)
        return out

    def _vcycle(self, l, b):
        L = self.levels[l]
        if l == len(self.levels) - 1:
            if L.dense_pinv is not None:
                return (L.dense_pinv @ b.ravel()).reshape(L.shape)
            x = np.zeros(L.shape)
            for _ in range(8):
                x = self._smooth(L, x, b)
            return x
        x = np.zeros(L.shape)
        for _ in range(self.sweeps):
            x = self._smooth(L, x, b)
        r = b - self._apply(L, x)
        ec = self._vcycle(l + 1, self._restrict(L, r))
        x += self._prolong(self.levels[l + 1], ec) * L.act
        for _ in range(self.sweeps):
            x = self._smooth(L, x, b)
        return x

    def precondition(self, v):
        """One V-cycle: unknown vector -> unknown vector."""
        b = np.zeros(self.own.shape)
        b[self.own] = v[self.idx]
        x = self._vcycle(0, b)
        z = np.zeros(self.n)
        z[self.idx] = x[self.own]
        # the operator's null space is the constant: keep the iterates free of it, so that
        # their size (and the rounding of b - A x) stays that of the solution
        return z - z.mean()

    # ------------------------------------------------------------------ FGMRES
    def solve(self, b, x0=None, rtol=1e-13, restart=30, maxiter=400):
        """FGMRES(restart) to ||b - A x|| <= rtol ||b||, or until a restart cycle no longer
        lowers the true residual (the rounding floor of b - A x in FP64, which for the
        larger grids lies a little above 1e-13 ||b||); returns (x, iterations, relres)."""
        A = self.A
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        bn = np.linalg.norm(b)
        if bn == 0:
            return x, 0, 0.0
        it = 0
        best = np.inf
        while True:
            x -= x.mean()
            r = b - A @ x
            beta = np.linalg.norm(r)
            if beta <= rtol * bn or it >= maxiter or beta > 0.5 * best:
                return x, it, beta / bn
            best = beta
            m = restart
            V = np.zeros((m + 1, self.n))
            Z = np.zeros((m, self.n))
            H = np.zeros((m + 1, m))
            cs = np.zeros(m)
            sn = np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            V[0] = r / beta
            k = 0
            for k in range(m):
                Z[k] = self.precondition(V[k])
                w = A @ Z[k]
                for q in range(2):               # classical Gram-Schmidt, re-orthogonalised
                    h = V[:k + 1] @ w
                    w -= h @ V[:k + 1]
                    H[:k + 1, k] += h
                H[k + 1, k] = np.linalg.norm(w)
                if H[k + 1, k] > 0:
                    V[k + 1] = w / H[k + 1, k]
                for q in range(k):
                    t = cs[q] * H[q, k] + sn[q] * H[q + 1, k]
                    H[q + 1, k] = -sn[q] * H[q, k] + cs[q] * H[q + 1, k]
                    H[q, k] = t
                d = np.hypot(H[k, k], H[k + 1, k])
                cs[k], sn[k] = (1.0, 0.0) if d == 0 else (H[k, k] / d, H[k + 1, k] / d)
                H[k, k] = d
                H[k + 1, k] = 0.0
                g[k + 1] = -sn[k] * g[k]
                g[k] = cs[k] * g[k]
                it += 1
                if abs(g[k + 1]) <= 0.5 * rtol * bn or it >= maxiter:
                    break
            kk = k + 1
            y = np.linalg.solve(np.triu(H[:kk, :kk]), g[:kk])
            x += y @ Z[:kk]
