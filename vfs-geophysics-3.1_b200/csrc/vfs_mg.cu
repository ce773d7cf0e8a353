// Geometric multigrid preconditioner of the pressure-Poisson solve (one V-cycle per
// FGMRES iteration), FP32 or FP64.
//
// The reference preconditions its Krylov solve with HYPRE BoomerAMG
// (poisson_hypre.c:26-88); this is a B200-first geometric replacement, not a port:
//
//   * Levels are cell-centred and coarsened by 2 in every direction while all interior
//     dimensions are even and at least 4 (256x192x256 -> ... -> 4x3x4: seven levels).
//   * Every level, the finest included, smooths with the 7-point conductance form of the
//     operator: the coupling of two unknowns across a face is the symmetrised, clipped
//     main-term coefficient of the reference's 19-point row (exactly the operator on
//     orthogonal grids, where the reference's filter drops every cross term).  A coarse
//     face conducts 0.5 x the sum of the four fine faces it covers; diagonals are minus
//     the sum of a cell's couplings, so every level is a consistent Neumann operator.
//   * Smoother: line Gauss-Seidel along j (the wall-normal, most strongly coupled
//     direction of the channel grids) in zebra order: the columns with (i+k) even are
//     solved first, then the odd ones, so each column's i/k neighbours are fixed while it
//     is solved and the update is in place and deterministic.  The tridiagonal factors
//     (Thomas forward coefficients and pivots) are precomputed once per operator.
//   * Restriction sums the residuals of the 8 children; prolongation is cell-centred
//     trilinear (weights 27/64, 9/64, 3/64, 1/64), a missing or inactive coarse
//     neighbour giving its weight to the parent.  With these transfers the FGMRES
//     iteration count stays flat as the grid is refined.
//
// Layout: every level stores its cells in "zebra" order, ((k*ny + j)*2 + colour)*hx + i/2
// with colour = (i xor k) & 1 and hx = ceil(nx/2), so the columns of one colour are
// contiguous half-rows and each colour pass reads and writes with unit stride.  The
// finest level is indexed by interior cell (DA index minus one); conversion to and from
// the solver's DA-layout FP64 vectors happens once per V-cycle.
//
// A level with an odd number of cells along a periodic i or k direction cannot be two-
// coloured; it is smoothed by damped (0.8) line Jacobi instead.
#include <algorithm>
#include <cmath>

#include "vfs_internal.cuh"

namespace vfs {

enum { OP_CE = 0, OP_CN, OP_CT, OP_DG, OP_CPR, OP_IDEN, NOP };

__host__ __device__ inline long long zidx(const ZL &L, int i, int j, int k) {
  return (((long long)k * L.ny + j) * 2 + ((i ^ k) & 1)) * L.hx + (i >> 1);
}

// ------------------------------------------------------------------ set-up (FP64)
// Fine-level couplings from the reference operator (19 slots on the DA layout).
__global__ void k_mg_fine_couplings(Grid g, ZL L, const double *__restrict__ coef, const uint8_t *__restrict__ fluid,
                                    double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  const long long N = g.N;
  const long long p = lidx(g, i + 1, j + 1, k + 1);
  const long long q = zidx(L, i, j, k);
  double ce = 0, cn = 0, ct = 0;
  if (fluid[p]) {
    if (i + 1 < L.nx || L.ip) {
      const long long e = lidx(g, wrapi(g, i + 2), j + 1, k + 1);
      if (fluid[e]) ce = fmax(0.0, 0.5 * (coef[EP * N + p] + coef[WP * N + e]));
    }
    if (j + 1 < L.ny || L.jp) {
      const long long e = lidx(g, i + 1, wrapj(g, j + 2), k + 1);
      if (fluid[e]) cn = fmax(0.0, 0.5 * (coef[NP * N + p] + coef[SP * N + e]));
    }
    if (k + 1 < L.nz || L.kp) {
      const long long e = lidx(g, i + 1, j + 1, wrapk(g, k + 2));
      if (fluid[e]) ct = fmax(0.0, 0.5 * (coef[TP * N + p] + coef[BP * N + e]));
    }
  }
  op[OP_CE * L.n + q] = ce;
  op[OP_CN * L.n + q] = cn;
  op[OP_CT * L.n + q] = ct;
}

// Coarse couplings: 0.5 x the sum of the four fine couplings across each coarse face.
__global__ void k_mg_coarse_couplings(ZL F, ZL C, const double *__restrict__ opF, double *__restrict__ opC) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)C.nx * C.ny * C.nz;
  if (t >= ncell) return;
  const int I = (int)(t % C.nx);
  const long long r = t / C.nx;
  const int J = (int)(r % C.ny), K = (int)(r / C.ny);
  double sx = 0, sy = 0, sz = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      sx += opF[OP_CE * F.n + zidx(F, 2 * I + 1, 2 * J + u, 2 * K + v)];
      sy += opF[OP_CN * F.n + zidx(F, 2 * I + u, 2 * J + 1, 2 * K + v)];
      sz += opF[OP_CT * F.n + zidx(F, 2 * I + u, 2 * J + v, 2 * K + 1)];
    }
  const long long q = zidx(C, I, J, K);
  opC[OP_CE * C.n + q] = 0.5 * sx;
  opC[OP_CN * C.n + q] = 0.5 * sy;
  opC[OP_CT * C.n + q] = 0.5 * sz;
}

// Neighbour cells of (i,j,k) with the level's periodic wrap; -1 where there is none.
struct ZNb {
  int ie, iw, jn, js, kt, kb;
};
__device__ __forceinline__ ZNb znb(const ZL &L, int i, int j, int k) {
  ZNb r;
  r.ie = i + 1 < L.nx ? i + 1 : (L.ip ? 0 : -1);
  r.iw = i > 0 ? i - 1 : (L.ip ? L.nx - 1 : -1);
  r.jn = j + 1 < L.ny ? j + 1 : (L.jp ? 0 : -1);
  r.js = j > 0 ? j - 1 : (L.jp ? L.ny - 1 : -1);
  r.kt = k + 1 < L.nz ? k + 1 : (L.kp ? 0 : -1);
  r.kb = k > 0 ? k - 1 : (L.kp ? L.nz - 1 : -1);
  return r;
}

__global__ void k_mg_diag(ZL L, double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  const long long q = zidx(L, i, j, k), n = L.n;
  const ZNb b = znb(L, i, j, k);
  double s = op[OP_CE * n + q] + op[OP_CN * n + q] + op[OP_CT * n + q];
  if (b.iw >= 0) s += op[OP_CE * n + zidx(L, b.iw, j, k)];
  if (b.js >= 0) s += op[OP_CN * n + zidx(L, i, b.js, k)];
  if (b.kb >= 0) s += op[OP_CT * n + zidx(L, i, j, b.kb)];
  op[OP_DG * n + q] = -s;
}

// Thomas factors of every j-line (the in-line couplings only; a periodic j wrap is left
// to the right-hand side): cpr_j = upper_j / den_j, iden_j = 1 / den_j,
// den_j = dg_j - lower_j * cpr_{j-1}.  Inactive or degenerate rows get zero factors, so
// the smoother leaves their unknown at zero.
__global__ void k_mg_thomas(ZL L, double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.nx * L.nz) return;
  const int i = (int)(t % L.nx), k = (int)(t / L.nx);
  const long long n = L.n;
  double cprev = 0, lower = 0;
  for (int j = 0; j < L.ny; j++) {
    const long long q = zidx(L, i, j, k);
    const double dg = op[OP_DG * n + q];
    const double upper = j + 1 < L.ny ? op[OP_CN * n + q] : 0.0;
    double cpr = 0, iden = 0;
    if (dg != 0) {
      const double den = dg - lower * cprev;
      if (fabs(den) > 1e-12 * fabs(dg)) {
        iden = 1.0 / den;
        cpr = upper * iden;
      }
    }
    op[OP_CPR * n + q] = cpr;
    op[OP_IDEN * n + q] = iden;
    cprev = cpr;
    lower = upper;
  }
}

__global__ void k_mg_cast(long long n, const double *__restrict__ a, float *__restrict__ b) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) b[p] = (float)a[p];
}

// ------------------------------------------------------------------ smoother
// One colour pass of zebra line Gauss-Seidel (colour 0/1; x read for the other colour,
// written for this one), or, with colour < 0, one damped line-Jacobi sweep over all
// columns (neighbours read from xr = the previous iterate, a separate array).
// x_zero: the neighbours read are known to be zero (first pass from a zero guess).
// The forward elimination stores d'_j in ds; the back substitution writes x.
template <typename T>
__global__ void __launch_bounds__(64) k_zline(ZL L, const T *__restrict__ op, const T *__restrict__ b,
                                              const T *__restrict__ xr, T *__restrict__ ds, T *__restrict__ xw,
                                              int colour, T omega, int x_zero) {
  const int hx = L.hx;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int c, h, k;
  if (colour >= 0) {
    if (t >= (long long)L.nz * hx) return;
    h = (int)(t % hx); k = (int)(t / hx); c = colour;
  } else {
    if (t >= 2LL * L.nz * hx) return;
    h = (int)(t % hx); c = (int)((t / hx) & 1); k = (int)(t / (2LL * hx));
  }
  const int i = 2 * h + (c ^ (k & 1));
  if (i >= L.nx) return;
  const long long n = L.n;
  const ZNb nb = znb(L, i, 0, k);
  const long long p0 = zidx(L, i, 0, k);
  // offsets of the neighbour columns (constant along j).  A missing neighbour (domain
  // edge) borrows the offset of the opposite one with a zero weight, so every x read
  // is of the other colour (every level has at least 2 cells along i and k).
  const T me = nb.ie >= 0 ? T(1) : T(0), mw = nb.iw >= 0 ? T(1) : T(0);
  const T mt = nb.kt >= 0 ? T(1) : T(0), mb = nb.kb >= 0 ? T(1) : T(0);
  const long long oe = zidx(L, nb.ie >= 0 ? nb.ie : nb.iw, 0, k) - p0;
  const long long ow = zidx(L, nb.iw >= 0 ? nb.iw : nb.ie, 0, k) - p0;
  const long long ot = zidx(L, i, 0, nb.kt >= 0 ? nb.kt : nb.kb) - p0;
  const long long ob = zidx(L, i, 0, nb.kb >= 0 ? nb.kb : nb.kt) - p0;
  const long long sj = 2LL * hx;
  const T *__restrict__ ce = op + OP_CE * n;
  const T *__restrict__ cn = op + OP_CN * n;
  const T *__restrict__ ct = op + OP_CT * n;
  const T *__restrict__ cpr = op + OP_CPR * n;
  const T *__restrict__ idn = op + OP_IDEN * n;
  const int ny = L.ny;
  T dprev = 0, lower = 0;
  if (x_zero) {
#pragma unroll 8
    for (int j = 0; j < ny; j++) {
      const long long q = p0 + j * sj;
      const T d = (b[q] - lower * dprev) * idn[q];
      lower = cn[q];
      ds[q] = d;
      dprev = d;
    }
  } else {
    const T *__restrict__ xs = colour >= 0 ? xw : xr;  // own column (periodic j only)
#pragma unroll 8
    for (int j = 0; j < ny; j++) {
      const long long q = p0 + j * sj;
      T r = b[q];
      r -= me * ce[q] * xr[q + oe];
      r -= mw * ce[q + ow] * xr[q + ow];
      r -= mt * ct[q] * xr[q + ot];
      r -= mb * ct[q + ob] * xr[q + ob];
      if (L.jp) {
        if (j == 0) r -= cn[p0 + (ny - 1) * sj] * xs[p0 + (ny - 1) * sj];
        if (j == ny - 1) r -= cn[q] * xs[p0];
      }
      const T d = (r - lower * dprev) * idn[q];
      lower = cn[q];
      ds[q] = d;
      dprev = d;
    }
  }
  T xnext = 0;
  if (colour >= 0) {
#pragma unroll 8
    for (int j = ny - 1; j >= 0; j--) {
      const long long q = p0 + j * sj;
      const T v = ds[q] - cpr[q] * xnext;
      xnext = v;
      xw[q] = v;
    }
  } else {
#pragma unroll 8
    for (int j = ny - 1; j >= 0; j--) {
      const long long q = p0 + j * sj;
      const T v = ds[q] - cpr[q] * xnext;
      xnext = v;
      xw[q] = x_zero ? omega * v : xr[q] + omega * (v - xr[q]);
    }
  }
}

// Residual b - A x at one cell of a level.
template <typename T>
__device__ __forceinline__ T zresid(const ZL &L, const T *__restrict__ op, const T *__restrict__ x,
                                    const T *__restrict__ b, int i, int j, int k, long long q) {
  const long long n = L.n;
  const ZNb nb = znb(L, i, j, k);
  T ax = op[OP_DG * n + q] * x[q];
  if (nb.ie >= 0) ax += op[OP_CE * n + q] * x[zidx(L, nb.ie, j, k)];
  if (nb.iw >= 0) { const long long w = zidx(L, nb.iw, j, k); ax += op[OP_CE * n + w] * x[w]; }
  if (nb.jn >= 0) ax += op[OP_CN * n + q] * x[zidx(L, i, nb.jn, k)];
  if (nb.js >= 0) { const long long s = zidx(L, i, nb.js, k); ax += op[OP_CN * n + s] * x[s]; }
  if (nb.kt >= 0) ax += op[OP_CT * n + q] * x[zidx(L, i, j, nb.kt)];
  if (nb.kb >= 0) { const long long s = zidx(L, i, j, nb.kb); ax += op[OP_CT * n + s] * x[s]; }
  return b[q] - ax;
}

// Coarse right-hand side: the sum of the residuals of the (active) children.
template <typename T>
__global__ void k_zrestrict(ZL F, ZL C, const T *__restrict__ opF, const T *__restrict__ x, const T *__restrict__ b,
                            T *__restrict__ bc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)C.nx * C.ny * C.nz;
  if (t >= ncell) return;
  const int I = (int)(t % C.nx);
  const long long r = t / C.nx;
  const int J = (int)(r % C.ny), K = (int)(r / C.ny);
  T s = 0;
  for (int c = 0; c < 2; c++)
    for (int bb = 0; bb < 2; bb++)
      for (int a = 0; a < 2; a++) {
        const int i = 2 * I + a, j = 2 * J + bb, k = 2 * K + c;
        const long long q = zidx(F, i, j, k);
        if (opF[OP_DG * F.n + q] == T(0)) continue;
        s += zresid<T>(F, opF, x, b, i, j, k, q);
      }
  bc[zidx(C, I, J, K)] = s;
}

// x_fine += P x_coarse (cell-centred trilinear).
template <typename T>
__global__ void k_zprolong(ZL F, ZL C, const T *__restrict__ opF, const T *__restrict__ opC, T *__restrict__ x,
                           const T *__restrict__ xc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)F.nx * F.ny * F.nz;
  if (t >= ncell) return;
  const int i = (int)(t % F.nx);
  const long long r = t / F.nx;
  const int j = (int)(r % F.ny), k = (int)(r / F.ny);
  const long long q = zidx(F, i, j, k);
  if (opF[OP_DG * F.n + q] == T(0)) return;
  const int I = i >> 1, J = j >> 1, K = k >> 1;
  // the other coarse cell nearest along each direction, or -1
  int In = I + ((i & 1) ? 1 : -1), Jn = J + ((j & 1) ? 1 : -1), Kn = K + ((k & 1) ? 1 : -1);
  if (In < 0 || In >= C.nx) In = C.ip ? (In + C.nx) % C.nx : -1;
  if (Jn < 0 || Jn >= C.ny) Jn = C.jp ? (Jn + C.ny) % C.ny : -1;
  if (Kn < 0 || Kn >= C.nz) Kn = C.kp ? (Kn + C.nz) % C.nz : -1;
  const long long own = zidx(C, I, J, K);
  const T *__restrict__ dgC = opC + OP_DG * C.n;
  T wown = T(27) / T(64);
  T s = 0;
  for (int c = 0; c < 2; c++)
    for (int bb = 0; bb < 2; bb++)
      for (int a = 0; a < 2; a++) {
        if (a + bb + c == 0) continue;
        const T w = (a ? T(1) : T(3)) * (bb ? T(1) : T(3)) * (c ? T(1) : T(3)) / T(64);
        const int ii = a ? In : I, jj = bb ? Jn : J, kk = c ? Kn : K;
        if (ii < 0 || jj < 0 || kk < 0) { wown += w; continue; }
        const long long qc = zidx(C, ii, jj, kk);
        if (dgC[qc] == T(0)) { wown += w; continue; }
        s += w * xc[qc];
      }
  x[q] += s + wown * xc[own];
}

// DA-layout FP64 vector -> finest-level right-hand side.
template <typename T>
__global__ void k_to_zebra(Grid g, ZL L, const double *__restrict__ v, T *__restrict__ b) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  b[zidx(L, i, j, k)] = (T)v[lidx(g, i + 1, j + 1, k + 1)];
}

// Finest-level solution -> DA-layout FP64 vector (zero off the unknowns).
template <typename T>
__global__ void k_from_zebra(Grid g, ZL L, const uint8_t *__restrict__ fluid, const T *__restrict__ x,
                             double *__restrict__ z) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int i = (int)(p % g.mx);
  const long long r = p / g.mx;
  const int j = (int)(r % g.my), k = (int)(r / g.my);
  double v = 0;
  if (fluid[p] && i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2)
    v = (double)x[zidx(L, i - 1, j - 1, k - 1)];
  z[p] = v;
}

// ------------------------------------------------------------------ host side
static ZL make_zl(int nx, int ny, int nz, const Grid &g) {
  ZL L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.hx = (nx + 1) / 2;
  L.ip = g.iper; L.jp = g.jper; L.kp = g.kper;
  L.n = (long long)nz * ny * 2 * L.hx;
  return L;
}

void mg_free(Poisson &P) {
  for (MGLevel &L : P.lv) {
    cudaFree(L.op64); cudaFree(L.op32); cudaFree(L.v64); cudaFree(L.v32);
  }
  P.lv.clear();
}

int mg_setup(Ctx *c) {
  Poisson &P = c->ps;
  const Grid &g = c->g;
  int rc;
  mg_free(P);
  int nx = g.mx - 2, ny = g.my - 2, nz = g.mz - 2;
  const int maxlev = 12;
  while ((int)P.lv.size() < maxlev) {
    MGLevel L;
    L.z = make_zl(nx, ny, nz, g);
    L.zebra = !((L.z.ip && (nx & 1)) || (L.z.kp && (nz & 1)));
    const long long n = L.z.n;
    bool ok = cudaMalloc(&L.op64, sizeof(double) * NOP * n) == cudaSuccess;
    ok &= cudaMalloc(&L.op32, sizeof(float) * NOP * n) == cudaSuccess;
    ok &= cudaMalloc(&L.v64, sizeof(double) * 4 * n) == cudaSuccess;
    ok &= cudaMalloc(&L.v32, sizeof(float) * 4 * n) == cudaSuccess;
    if (!ok) {
      P.lv.push_back(L);
      return set_err(c, VFS_ERR_CUDA, "poisson_lhs: multigrid allocation failed");
    }
    cudaMemsetAsync(L.op64, 0, sizeof(double) * NOP * n, c->stream);
    cudaMemsetAsync(L.v64, 0, sizeof(double) * 4 * n, c->stream);
    cudaMemsetAsync(L.v32, 0, sizeof(float) * 4 * n, c->stream);
    const long long ncell = (long long)nx * ny * nz;
    if (P.lv.empty()) {
      k_mg_fine_couplings<<<nblocks(ncell, 128), 128, 0, c->stream>>>(g, L.z, P.coef, P.fluid, L.op64);
    } else {
      const MGLevel &F = P.lv.back();
      k_mg_coarse_couplings<<<nblocks(ncell, 128), 128, 0, c->stream>>>(F.z, L.z, F.op64, L.op64);
    }
    if ((rc = check_launch(c, "k_mg_couplings"))) { P.lv.push_back(L); return rc; }
    k_mg_diag<<<nblocks(ncell, 128), 128, 0, c->stream>>>(L.z, L.op64);
    k_mg_thomas<<<nblocks((long long)nx * nz, 64), 64, 0, c->stream>>>(L.z, L.op64);
    k_mg_cast<<<nblocks(NOP * n, 256), 256, 0, c->stream>>>(NOP * n, L.op64, L.op32);
    P.lv.push_back(L);
    if ((rc = check_launch(c, "k_mg_setup"))) return rc;
    if ((nx & 1) || (ny & 1) || (nz & 1) || nx < 4 || ny < 4 || nz < 4) break;
    nx /= 2; ny /= 2; nz /= 2;
  }
  return VFS_OK;
}

template <typename T> struct MGp;
template <> struct MGp<float> {
  static const float *op(const MGLevel &L) { return L.op32; }
  static float *v(const MGLevel &L) { return L.v32; }
};
template <> struct MGp<double> {
  static const double *op(const MGLevel &L) { return L.op64; }
  static double *v(const MGLevel &L) { return L.v64; }
};

static const double kJacobiOmega = 0.8;

// `sweeps` smoothing sweeps on level l; x_zero: x is taken as zero on entry.
template <typename T>
static int mg_smooth(Ctx *c, int l, int sweeps, bool x_zero) {
  const MGLevel &L = c->ps.lv[l];
  const long long n = L.z.n;
  const T *op = MGp<T>::op(L);
  T *x = MGp<T>::v(L), *b = x + n, *xo = x + 2 * n, *ds = x + 3 * n;
  const long long half = (long long)L.z.nz * L.z.hx;
  for (int s = 0; s < sweeps; s++) {
    const bool z = x_zero && s == 0;
    if (L.zebra) {
      for (int col = 0; col < 2; col++)
        k_zline<T><<<nblocks(half, 64), 64, 0, c->stream>>>(L.z, op, b, x, ds, x, col, T(1), (z && col == 0) ? 1 : 0);
    } else {
      if (!z) cudaMemcpyAsync(xo, x, sizeof(T) * n, cudaMemcpyDeviceToDevice, c->stream);
      k_zline<T><<<nblocks(2 * half, 64), 64, 0, c->stream>>>(L.z, op, b, xo, ds, x, -1, T(kJacobiOmega), z ? 1 : 0);
    }
  }
  return check_launch(c, "k_zline");
}

template <typename T>
static int mg_vcycle(Ctx *c, int l, int nl, const vfs_solve_opts &o) {
  int rc;
  if (l == nl - 1) return mg_smooth<T>(c, l, o.coarse_iters, true);
  if ((rc = mg_smooth<T>(c, l, o.pre_smooth, true))) return rc;
  const MGLevel &F = c->ps.lv[l], &C = c->ps.lv[l + 1];
  const long long nc = (long long)C.z.nx * C.z.ny * C.z.nz, nf = (long long)F.z.nx * F.z.ny * F.z.nz;
  T *xf = MGp<T>::v(F), *xc = MGp<T>::v(C);
  k_zrestrict<T><<<nblocks(nc, 128), 128, 0, c->stream>>>(F.z, C.z, MGp<T>::op(F), xf, xf + F.z.n, xc + C.z.n);
  if ((rc = check_launch(c, "k_zrestrict"))) return rc;
  if ((rc = mg_vcycle<T>(c, l + 1, nl, o))) return rc;
  k_zprolong<T><<<nblocks(nf, 256), 256, 0, c->stream>>>(F.z, C.z, MGp<T>::op(F), MGp<T>::op(C), xf, xc);
  if ((rc = check_launch(c, "k_zprolong"))) return rc;
  return mg_smooth<T>(c, l, o.post_smooth, false);
}

template <typename T>
static int mg_apply(Ctx *c, const double *v, double *z, const vfs_solve_opts &o) {
  Poisson &P = c->ps;
  const MGLevel &L0 = P.lv[0];
  const long long ncell = (long long)L0.z.nx * L0.z.ny * L0.z.nz;
  T *x0 = MGp<T>::v(L0);
  int rc;
  k_to_zebra<T><<<nblocks(ncell, 256), 256, 0, c->stream>>>(c->g, L0.z, v, x0 + L0.z.n);
  if ((rc = check_launch(c, "k_to_zebra"))) return rc;
  const int nl = o.levels > 0 ? std::min((int)P.lv.size(), o.levels) : (int)P.lv.size();
  if ((rc = mg_vcycle<T>(c, 0, nl, o))) return rc;
  k_from_zebra<T><<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, L0.z, P.fluid, x0, z);
  return check_launch(c, "k_from_zebra");
}

// z = M^-1 v: one V-cycle in FP32 (precision 0) or FP64.
int mg_precondition(Ctx *c, const double *v, double *z, const vfs_solve_opts &o) {
  return o.precision == 0 ? mg_apply<float>(c, v, z, o) : mg_apply<double>(c, v, z, o);
}

// One smoothing sweep of the finest level (both colours), for timing.
int mg_sweep_fine(Ctx *c, int precision) {
  return precision == 0 ? mg_smooth<float>(c, 0, 1, false) : mg_smooth<double>(c, 0, 1, false);
}

}  // namespace vfs
