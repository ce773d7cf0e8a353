// Pressure-Poisson path for sm_100a: operator assembly (PoissonLHSNew), right-hand side
// (PoissonRHS2_hypre + Remove_Nullspace_Scale), the solve (flexible GMRES in FP64 with
// a geometric multigrid preconditioner in FP32 or FP64), and the velocity correction
// (UpdatePressure, Projection) and divergence check.
//
// Unknowns live on the grid layout (mx*my*mz doubles); a cell is an unknown when the
// reference would give it a Poisson DOF (setup_lidx2, poisson.c:182): interior and
// nvert < 1.  Every solver vector is exactly zero on the other points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "vfs_internal.cuh"

namespace vfs {

__constant__ int c_off[NSLOT][3] = {
    {0, 0, 0},  {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
    {1, 1, 0},  {1, -1, 0},  {-1, 1, 0},  {-1, -1, 0}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1},
    {0, -1, -1}, {1, 0, 1},  {1, 0, -1},  {-1, 0, 1}, {-1, 0, -1}};

__device__ __forceinline__ int slot_of(int di, int dj, int dk) {
  // inverse of c_off (poisson.c:951-969)
  if (dk == 0) {
    if (dj == 0) return di == 0 ? CP : (di > 0 ? EP : WP);
    if (di == 0) return dj > 0 ? NP : SP;
    if (di > 0) return dj > 0 ? NE : SE;
    return dj > 0 ? NW : SW;
  }
  if (di == 0 && dj == 0) return dk > 0 ? TP : BP;
  if (di == 0) return dj > 0 ? (dk > 0 ? TN : BN) : (dk > 0 ? TS : BS);
  return di > 0 ? (dk > 0 ? TE : BE) : (dk > 0 ? TW : BW);
}

// Linear index of the Poisson unknown a stencil slot refers to, or -1 (lidx2 with the
// periodic Gid copy of setup_lidx2, poisson.c:270-300).
__device__ __forceinline__ long long unknown_at(const Grid &g, const uint8_t *nv, int i, int j, int k) {
  i = wrapi(g, i); j = wrapj(g, j); k = wrapk(g, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return -1;
  long long p = lidx(g, i, j, k);
  return nv[p] >= 1 ? -1 : p;
}

// g_ab of PoissonLHSNew (poisson.c:1098-1132) at point (i,j,k), taking the face metrics
// from the periodic image (a,b,c) on a periodic ghost plane.
struct GAB { double v[9]; };  // g11 g12 g13 g21 g22 g23 g31 g32 g33
__device__ GAB gab_at(const Grid &g, const Metrics &m, int i, int j, int k) {
  const long long s = lidx(g, wrapi(g, i), wrapj(g, j), wrapk(g, k));
  GAB r;
  const double ix = m.icsi.x[s], iy = m.icsi.y[s], iz = m.icsi.z[s];
  r.v[0] = (ix * ix + iy * iy + iz * iz) * m.iaj[s];
  r.v[1] = (m.ieta.x[s] * ix + m.ieta.y[s] * iy + m.ieta.z[s] * iz) * m.iaj[s];
  r.v[2] = (m.izet.x[s] * ix + m.izet.y[s] * iy + m.izet.z[s] * iz) * m.iaj[s];
  const double jx = m.jeta.x[s], jy = m.jeta.y[s], jz = m.jeta.z[s];
  r.v[3] = (m.jcsi.x[s] * jx + m.jcsi.y[s] * jy + m.jcsi.z[s] * jz) * m.jaj[s];
  r.v[4] = (jx * jx + jy * jy + jz * jz) * m.jaj[s];
  r.v[5] = (m.jzet.x[s] * jx + m.jzet.y[s] * jy + m.jzet.z[s] * jz) * m.jaj[s];
  const double kx = m.kzet.x[s], ky = m.kzet.y[s], kz = m.kzet.z[s];
  r.v[6] = (m.kcsi.x[s] * kx + m.kcsi.y[s] * ky + m.kcsi.z[s] * kz) * m.kaj[s];
  r.v[7] = (m.keta.x[s] * kx + m.keta.y[s] * ky + m.keta.z[s] * kz) * m.kaj[s];
  r.v[8] = (kx * kx + ky * ky + kz * kz) * m.kaj[s];
  return r;
}

struct StencilCtx {
  const Grid *g;
  const uint8_t *nv;
  int i, j, k;
  double vol[NSLOT];
  __device__ int nvat(int di, int dj, int dk) const {
    return nv[lidx(*g, i + di, j + dj, k + dk)];
  }
  __device__ void add(int di, int dj, int dk, double v) { vol[slot_of(di, dj, dk)] += v; }
};

// Cross-derivative contribution of one face of the cell (poisson.c:1163-1215 pattern):
// face between the cell and its neighbour at d (unit offset along the face normal),
// cross direction e, coefficient G, overall sign s (+1 for the "x+1 - x" blocks, -1
// for the "x - x-1" blocks).  `ecoord`, `em` and `eper` describe the cross direction.
__device__ void cross_term(StencilCtx &S, const int d[3], const int e[3], int ecoord, int em,
                           int eper, double G, double s) {
  const int nplus = S.nvat(e[0], e[1], e[2]) + S.nvat(d[0] + e[0], d[1] + e[1], d[2] + e[2]);
  const int nminus = S.nvat(-e[0], -e[1], -e[2]) + S.nvat(d[0] - e[0], d[1] - e[1], d[2] - e[2]);
  if ((ecoord == em - 2 && !eper) || nplus > 0) {
    if (nminus == 0 && ecoord != 1) {
      const double v = G * 0.5;
      S.add(0, 0, 0, s * v);
      S.add(d[0], d[1], d[2], s * v);
      S.add(-e[0], -e[1], -e[2], -s * v);
      S.add(d[0] - e[0], d[1] - e[1], d[2] - e[2], -s * v);
    }
  } else if ((ecoord == 1 && !eper) || nminus > 0) {
    if (nplus == 0) {
      const double v = G * 0.5;
      S.add(e[0], e[1], e[2], s * v);
      S.add(d[0] + e[0], d[1] + e[1], d[2] + e[2], s * v);
      S.add(0, 0, 0, -s * v);
      S.add(d[0], d[1], d[2], -s * v);
    }
  } else {
    const double v = G * 0.25;
    S.add(e[0], e[1], e[2], s * v);
    S.add(d[0] + e[0], d[1] + e[1], d[2] + e[2], s * v);
    S.add(-e[0], -e[1], -e[2], -s * v);
    S.add(d[0] - e[0], d[1] - e[1], d[2] - e[2], -s * v);
  }
}

// Main (normal-derivative) term of one face: vol[CP] -= G, vol[nb] += G.
__device__ __forceinline__ void main_term(StencilCtx &S, const int d[3], double G) {
  S.vol[CP] -= G;
  S.add(d[0], d[1], d[2], G);
}

// One thread per cell: the 19 matrix entries of a fluid cell's row, assembled in the
// order of PoissonLHSNew (poisson.c:1155-1560) so every entry is bit-identical, then the
// MatSetValues filter (|v| > 1e-10 and a valid column, or the diagonal; INSERT keeps the
// last slot that names a column) of poisson.c:1608-1612.
__global__ void k_poisson_coef(Grid g, Metrics m, const uint8_t *__restrict__ nv, double *coef,
                               uint8_t *fluid, double *invdiag) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  const long long N = g.N;
  const bool interior = !(i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1);
  if (!interior || nv[p] != 0) {
    for (int s = 0; s < NSLOT; s++) coef[s * N + p] = 0;
    fluid[p] = 0;
    invdiag[p] = 0;
    return;
  }
  StencilCtx S;
  S.g = &g; S.nv = nv; S.i = i; S.j = j; S.k = k;
  for (int s = 0; s < NSLOT; s++) S.vol[s] = 0;
  const GAB G0 = gab_at(g, m, i, j, k);
  const int dxp[3] = {1, 0, 0}, dxm[3] = {-1, 0, 0};
  const int dyp[3] = {0, 1, 0}, dym[3] = {0, -1, 0};
  const int dzp[3] = {0, 0, 1}, dzm[3] = {0, 0, -1};
  // i+1 - i
  if (S.nvat(1, 0, 0) == 0 && (i != mx - 2 || g.iper)) {
    main_term(S, dxp, G0.v[0]);
    cross_term(S, dxp, dyp, j, my, g.jper, G0.v[1], 1.0);
    cross_term(S, dxp, dzp, k, mz, g.kper, G0.v[2], 1.0);
  }
  // i - i-1
  if (S.nvat(-1, 0, 0) == 0 && (i != 1 || g.iper)) {
    const GAB Gm = gab_at(g, m, i - 1, j, k);
    main_term(S, dxm, Gm.v[0]);
    cross_term(S, dxm, dyp, j, my, g.jper, Gm.v[1], -1.0);
    cross_term(S, dxm, dzp, k, mz, g.kper, Gm.v[2], -1.0);
  }
  // j+1 - j
  if (S.nvat(0, 1, 0) == 0 && (j != my - 2 || g.jper)) {
    cross_term(S, dyp, dxp, i, mx, g.iper, G0.v[3], 1.0);
    main_term(S, dyp, G0.v[4]);
    cross_term(S, dyp, dzp, k, mz, g.kper, G0.v[5], 1.0);
  }
  // j - j-1
  if (S.nvat(0, -1, 0) == 0 && (j != 1 || g.jper)) {
    const GAB Gm = gab_at(g, m, i, j - 1, k);
    cross_term(S, dym, dxp, i, mx, g.iper, Gm.v[3], -1.0);
    main_term(S, dym, Gm.v[4]);
    cross_term(S, dym, dzp, k, mz, g.kper, Gm.v[5], -1.0);
  }
  // k+1 - k
  if (S.nvat(0, 0, 1) == 0 && (k != mz - 2 || g.kper)) {
    cross_term(S, dzp, dxp, i, mx, g.iper, G0.v[6], 1.0);
    cross_term(S, dzp, dyp, j, my, g.jper, G0.v[7], 1.0);
    main_term(S, dzp, G0.v[8]);
  }
  // k - k-1
  if (S.nvat(0, 0, -1) == 0 && (k != 1 || g.kper)) {
    const GAB Gm = gab_at(g, m, i, j, k - 1);
    cross_term(S, dzm, dxp, i, mx, g.iper, Gm.v[6], -1.0);
    cross_term(S, dzm, dyp, j, my, g.jper, Gm.v[7], -1.0);
    main_term(S, dzm, Gm.v[8]);
  }
  // MatSetValues filter with INSERT semantics
  long long col[NSLOT];
  bool set[NSLOT];
  for (int s = 0; s < NSLOT; s++) {
    col[s] = unknown_at(g, nv, i + c_off[s][0], j + c_off[s][1], k + c_off[s][2]);
    set[s] = (fabs(S.vol[s]) > 1.e-10 && col[s] >= 0) || s == CP;
  }
  for (int s = 0; s < NSLOT; s++) {
    if (!set[s]) continue;
    for (int t = s + 1; t < NSLOT; t++)
      if (set[t] && col[t] == col[s]) { set[s] = false; break; }
  }
  // A slot overwritten by a later one contributes nothing; the later slot carries the
  // inserted value.  The diagonal is the entry whose column is the cell itself.
  double diag = 0;
  for (int s = 0; s < NSLOT; s++) {
    double v = set[s] ? S.vol[s] : 0.0;
    coef[s * N + p] = v;
    if (set[s] && col[s] == p) diag = v;
  }
  fluid[p] = 1;
  invdiag[p] = diag != 0 ? 1.0 / diag : 0.0;
}

// Neighbour index of slot s for an unknown (valid only where the coefficient is non-zero;
// the index is always inside the array).
__device__ __forceinline__ long long nb_index(const Grid &g, int i, int j, int k, int s) {
  return lidx(g, wrapi(g, i + c_off[s][0]), wrapj(g, j + c_off[s][1]), wrapk(g, k + c_off[s][2]));
}

// y = A x on the grid layout (FP64).
__global__ void k_apply64(Grid g, const double *__restrict__ coef, const uint8_t *__restrict__ fluid,
                          const double *__restrict__ x, double *__restrict__ y) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  if (!fluid[p]) { y[p] = 0; return; }
  const int mx = g.mx, my = g.my;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  double s = 0;
#pragma unroll
  for (int t = 0; t < NSLOT; t++) {
    const double c = coef[t * g.N + p];
    if (c != 0.0) s += c * x[nb_index(g, i, j, k, t)];
  }
  y[p] = s;
}

int poisson_apply_dev(Ctx *c, const double *x, double *y) {
  k_apply64<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->ps.coef, c->ps.fluid, x, y);
  return check_launch(c, "k_apply64");
}

// ------------------------------------------------------------------ multigrid
// Fine-level smoother / residual in type T on the 19-point operator.
template <typename T>
__device__ __forceinline__ T apply_row(const Grid &g, const T *__restrict__ coef, const T *__restrict__ x,
                                       long long p, int i, int j, int k) {
  T s = 0;
#pragma unroll
  for (int t = 0; t < NSLOT; t++) {
    const T cf = coef[t * g.N + p];
    if (cf != T(0)) s += cf * x[nb_index(g, i, j, k, t)];
  }
  return s;
}

// One Chebyshev step on the fine level: r = D^-1 (b - A x), d = c1*d + c2*r, xo = x + d.
template <typename T>
__global__ void k_cheb_fine(Grid g, const T *__restrict__ coef, const T *__restrict__ invd,
                            const uint8_t *__restrict__ fluid, const T *__restrict__ b,
                            const T *__restrict__ x, T *__restrict__ xo, T *__restrict__ d, T c1,
                            T c2, int x_is_zero) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  if (!fluid[p]) { xo[p] = 0; d[p] = 0; return; }
  const int mx = g.mx, my = g.my;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  T ax = x_is_zero ? T(0) : apply_row<T>(g, coef, x, p, i, j, k);
  T r = invd[p] * (b[p] - ax);
  T dn = (x_is_zero ? T(0) : c1 * d[p]) + c2 * r;
  d[p] = dn;
  xo[p] = (x_is_zero ? T(0) : x[p]) + dn;
}

// y-line Jacobi smoothing on the fine level (the wall-normal direction of the stretched
// channel grids carries the strongest coupling, which point smoothers cannot damp).
// One thread per (i,k) column solves the tridiagonal system of its fluid cells along j
// (Thomas algorithm; the j-1 / j+1 couplings inside the column, everything else taken
// from the previous iterate), then x <- x + omega (x_line - x).  Consecutive threads
// own consecutive i, so every j-step of the sweep is a coalesced row access.
template <typename T>
__global__ void k_yline_fine(Grid g, const T *__restrict__ coef, const uint8_t *__restrict__ fluid,
                             const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ xn,
                             T *__restrict__ cp, T *__restrict__ dp, T omega, int x_is_zero) {
  const int ni = g.mx - 2, nk = g.mz - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ni * nk) return;
  const int i = 1 + (int)(t % ni), k = 1 + (int)(t / ni);
  const long long sy = g.mx, N = g.N;
  const int jn = g.my - 2;
  T pc = 0, pd = 0;
  for (int j = 1; j <= jn; j++) {
    const long long p = lidx(g, i, j, k);
    T a = 0, bb = 1, cc = 0, r = 0;
    if (fluid[p] && coef[CP * N + p] != T(0)) {  // a fluid cell without fluid neighbours keeps 0
      bb = coef[CP * N + p];
      if (j > 1) a = coef[SP * N + p];
      if (j < jn) cc = coef[NP * N + p];
      r = b[p];
      if (!x_is_zero) {
#pragma unroll
        for (int s = 1; s < NSLOT; s++) {
          if ((s == SP && j > 1) || (s == NP && j < jn)) continue;
          const T cf = coef[s * N + p];
          if (cf != T(0)) r -= cf * x[nb_index(g, i, j, k, s)];
        }
      }
    }
    const T den = bb - a * pc;
    pc = cc / den;
    pd = (r - a * pd) / den;
    cp[p] = pc;
    dp[p] = pd;
  }
  T xnext = 0;
  for (int j = jn; j >= 1; j--) {
    const long long p = lidx(g, i, j, k);
    const T xv = dp[p] - cp[p] * xnext;
    xnext = xv;
    if (!fluid[p]) { xn[p] = 0; continue; }
    xn[p] = x_is_zero ? omega * xv : x[p] + omega * (xv - x[p]);
  }
  (void)sy;
}

// Coarse-level layout: interior cells only, (k*ny + j)*nx + i, periodic wrap in the
// periodic directions, closed (zero conductance) otherwise.
struct CL {
  int nx, ny, nz, ip, jp, kp;
  long long n;
};
__device__ __forceinline__ long long cidx(const CL &L, int i, int j, int k) {
  return ((long long)k * L.ny + j) * L.nx + i;
}

template <typename T>
__device__ __forceinline__ T capply(const CL &L, const T *cx, const T *cy, const T *cz, const T *diag,
                                    const T *x, long long p, int i, int j, int k) {
  T s = diag[p] * x[p];
  // +i / -i
  if (i + 1 < L.nx) s += cx[p] * x[p + 1];
  else if (L.ip) s += cx[p] * x[p - (L.nx - 1)];
  if (i > 0) s += cx[p - 1] * x[p - 1];
  else if (L.ip) s += cx[p + (L.nx - 1)] * x[p + (L.nx - 1)];
  const long long sy = L.nx, sz = (long long)L.nx * L.ny;
  if (j + 1 < L.ny) s += cy[p] * x[p + sy];
  else if (L.jp) s += cy[p] * x[p - (L.ny - 1) * sy];
  if (j > 0) s += cy[p - sy] * x[p - sy];
  else if (L.jp) s += cy[p + (L.ny - 1) * sy] * x[p + (L.ny - 1) * sy];
  if (k + 1 < L.nz) s += cz[p] * x[p + sz];
  else if (L.kp) s += cz[p] * x[p - (L.nz - 1) * sz];
  if (k > 0) s += cz[p - sz] * x[p - sz];
  else if (L.kp) s += cz[p + (L.nz - 1) * sz] * x[p + (L.nz - 1) * sz];
  return s;
}

// y-line Jacobi on a coarse level (7-point conductances, ghost-free layout).
template <typename T>
__global__ void k_yline_coarse(CL L, const T *cx, const T *cy, const T *cz, const T *diag,
                               const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ xn,
                               T *__restrict__ cp, T *__restrict__ dp, T omega, int x_is_zero) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.nx * L.nz) return;
  const int i = (int)(t % L.nx), k = (int)(t / L.nx);
  const long long sy = L.nx, sz = (long long)L.nx * L.ny;
  T pc = 0, pd = 0;
  for (int j = 0; j < L.ny; j++) {
    const long long p = cidx(L, i, j, k);
    T a = 0, bb = 1, cc = 0, r = 0;
    if (diag[p] != T(0)) {
      bb = diag[p];
      if (j > 0) a = cy[p - sy];
      if (j + 1 < L.ny) cc = cy[p];
      r = b[p];
      if (!x_is_zero) {
        if (i + 1 < L.nx) r -= cx[p] * x[p + 1];
        else if (L.ip) r -= cx[p] * x[p - (L.nx - 1)];
        if (i > 0) r -= cx[p - 1] * x[p - 1];
        else if (L.ip) r -= cx[p + (L.nx - 1)] * x[p + (L.nx - 1)];
        if (k + 1 < L.nz) r -= cz[p] * x[p + sz];
        else if (L.kp) r -= cz[p] * x[p - (L.nz - 1) * sz];
        if (k > 0) r -= cz[p - sz] * x[p - sz];
        else if (L.kp) r -= cz[p + (L.nz - 1) * sz] * x[p + (L.nz - 1) * sz];
        if (L.jp) {  // the periodic wrap of the column is taken explicitly
          if (j == 0) r -= cy[p + (L.ny - 1) * sy] * x[p + (L.ny - 1) * sy];
          if (j == L.ny - 1) r -= cy[p] * x[p - (L.ny - 1) * sy];
        }
      }
    }
    const T den = bb - a * pc;
    pc = cc / den;
    pd = (r - a * pd) / den;
    cp[p] = pc;
    dp[p] = pd;
  }
  T xnext = 0;
  for (int j = L.ny - 1; j >= 0; j--) {
    const long long p = cidx(L, i, j, k);
    const T xv = dp[p] - cp[p] * xnext;
    xnext = xv;
    if (diag[p] == T(0)) { xn[p] = 0; continue; }
    xn[p] = x_is_zero ? omega * xv : x[p] + omega * (xv - x[p]);
  }
}

template <typename T>
__global__ void k_cheb_coarse(CL L, const T *cx, const T *cy, const T *cz, const T *diag,
                              const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ xo,
                              T *__restrict__ d, T c1, T c2, int x_is_zero) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= L.n) return;
  if (diag[p] == T(0)) { xo[p] = 0; d[p] = 0; return; }
  int i = (int)(p % L.nx);
  long long q = p / L.nx;
  int j = (int)(q % L.ny);
  int k = (int)(q / L.ny);
  T ax = x_is_zero ? T(0) : capply<T>(L, cx, cy, cz, diag, x, p, i, j, k);
  T r = (b[p] - ax) / diag[p];
  T dn = (x_is_zero ? T(0) : c1 * d[p]) + c2 * r;
  d[p] = dn;
  xo[p] = (x_is_zero ? T(0) : x[p]) + dn;
}

// Residual of the fine level summed over the 8 children of each level-1 cell.
template <typename T>
__global__ void k_restrict_fine(Grid g, CL L1, const T *__restrict__ coef, const uint8_t *__restrict__ fluid,
                                const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ bc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= L1.n) return;
  int I = (int)(p % L1.nx);
  long long q = p / L1.nx;
  int J = (int)(q % L1.ny);
  int K = (int)(q / L1.ny);
  T s = 0;
  for (int c = 0; c < 2; c++)
    for (int b2 = 0; b2 < 2; b2++)
      for (int a = 0; a < 2; a++) {
        const int i = 2 * I + 1 + a, j = 2 * J + 1 + b2, k = 2 * K + 1 + c;
        const long long f = lidx(g, i, j, k);
        if (!fluid[f]) continue;
        s += b[f] - apply_row<T>(g, coef, x, f, i, j, k);
      }
  bc[p] = s;
}

template <typename T>
__global__ void k_restrict_coarse(CL L, CL Lc, const T *cx, const T *cy, const T *cz, const T *diag,
                                  const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ bc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= Lc.n) return;
  int I = (int)(p % Lc.nx);
  long long q = p / Lc.nx;
  int J = (int)(q % Lc.ny);
  int K = (int)(q / Lc.ny);
  T s = 0;
  for (int c = 0; c < 2; c++)
    for (int b2 = 0; b2 < 2; b2++)
      for (int a = 0; a < 2; a++) {
        const int i = 2 * I + a, j = 2 * J + b2, k = 2 * K + c;
        const long long f = cidx(L, i, j, k);
        if (diag[f] == T(0)) continue;
        s += b[f] - capply<T>(L, cx, cy, cz, diag, x, f, i, j, k);
      }
  bc[p] = s;
}

// x_fine += x_coarse (piecewise-constant prolongation, transpose of the restriction).
template <typename T>
__global__ void k_prolong_fine(Grid g, CL L1, const uint8_t *__restrict__ fluid, T *x, const T *__restrict__ xc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  if (!fluid[p]) return;
  const int mx = g.mx, my = g.my;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  x[p] += xc[cidx(L1, (i - 1) >> 1, (j - 1) >> 1, (k - 1) >> 1)];
}
template <typename T>
__global__ void k_prolong_coarse(CL L, CL Lc, const T *diag, T *x, const T *__restrict__ xc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= L.n) return;
  if (diag[p] == T(0)) return;
  int i = (int)(p % L.nx);
  long long q = p / L.nx;
  int j = (int)(q % L.ny);
  int k = (int)(q / L.ny);
  x[p] += xc[cidx(Lc, i >> 1, j >> 1, k >> 1)];
}

// Level-1 conductances from the fine operator's 7-point couplings (symmetrised, clipped
// at zero): C = 0.5 * sum of the four fine face couplings on the coarse face.
__global__ void k_build_l1(Grid g, CL L1, const double *__restrict__ coef, const uint8_t *__restrict__ fluid,
                           double *cx, double *cy, double *cz) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= L1.n) return;
  int I = (int)(p % L1.nx);
  long long q = p / L1.nx;
  int J = (int)(q % L1.ny);
  int K = (int)(q / L1.ny);
  const long long N = g.N;
  double sx = 0, sy = 0, sz = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      {  // x face: fine cells (2I+2, 2J+1+u, 2K+1+v) -> +i
        const int i = 2 * I + 2, j = 2 * J + 1 + u, k = 2 * K + 1 + v;
        const long long f = lidx(g, i, j, k);
        const long long e = lidx(g, wrapi(g, i + 1), j, k);
        if (i + 1 <= g.mx - 2 || g.iper)
          if (fluid[f] && fluid[e]) sx += fmax(0.0, 0.5 * (coef[EP * N + f] + coef[WP * N + e]));
      }
      {
        const int i = 2 * I + 1 + u, j = 2 * J + 2, k = 2 * K + 1 + v;
        const long long f = lidx(g, i, j, k);
        const long long e = lidx(g, i, wrapj(g, j + 1), k);
        if (j + 1 <= g.my - 2 || g.jper)
          if (fluid[f] && fluid[e]) sy += fmax(0.0, 0.5 * (coef[NP * N + f] + coef[SP * N + e]));
      }
      {
        const int i = 2 * I + 1 + u, j = 2 * J + 1 + v, k = 2 * K + 2;
        const long long f = lidx(g, i, j, k);
        const long long e = lidx(g, i, j, wrapk(g, k + 1));
        if (k + 1 <= g.mz - 2 || g.kper)
          if (fluid[f] && fluid[e]) sz += fmax(0.0, 0.5 * (coef[TP * N + f] + coef[BP * N + e]));
      }
    }
  cx[p] = 0.5 * sx;
  cy[p] = 0.5 * sy;
  cz[p] = 0.5 * sz;
}

// Coarser conductances from the level below (same rule), and the diagonal.
__global__ void k_build_coarse(CL L, CL Lc, const double *cx, const double *cy, const double *cz,
                               double *ccx, double *ccy, double *ccz) {
  // cx/cy/cz: the finer level's conductances (op64 rows 0..2)
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= Lc.n) return;
  int I = (int)(p % Lc.nx);
  long long q = p / Lc.nx;
  int J = (int)(q % Lc.ny);
  int K = (int)(q / Lc.ny);
  double sx = 0, sy = 0, sz = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      sx += cx[cidx(L, 2 * I + 1, 2 * J + u, 2 * K + v)];
      sy += cy[cidx(L, 2 * I + u, 2 * J + 1, 2 * K + v)];
      sz += cz[cidx(L, 2 * I + u, 2 * J + v, 2 * K + 1)];
    }
  ccx[p] = 0.5 * sx;
  ccy[p] = 0.5 * sy;
  ccz[p] = 0.5 * sz;
}

__global__ void k_coarse_diag(CL L, double *cx, double *cy, double *cz, double *diag) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= L.n) return;
  int i = (int)(p % L.nx);
  long long q = p / L.nx;
  int j = (int)(q % L.ny);
  int k = (int)(q / L.ny);
  const long long sy = L.nx, sz = (long long)L.nx * L.ny;
  // close faces leaving a non-periodic domain
  if (i == L.nx - 1 && !L.ip) cx[p] = 0;
  if (j == L.ny - 1 && !L.jp) cy[p] = 0;
  if (k == L.nz - 1 && !L.kp) cz[p] = 0;
  double s = cx[p] + cy[p] + cz[p];
  s += (i > 0) ? cx[p - 1] : (L.ip ? cx[p + L.nx - 1] : 0.0);
  s += (j > 0) ? cy[p - sy] : (L.jp ? cy[p + (L.ny - 1) * sy] : 0.0);
  s += (k > 0) ? cz[p - sz] : (L.kp ? cz[p + (L.nz - 1) * sz] : 0.0);
  diag[p] = -s;
}

__global__ void k_cast_d2f(long long n, const double *a, float *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) b[p] = (float)a[p];
}
__global__ void k_cast_f2d(long long n, const float *a, double *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) b[p] = (double)a[p];
}

// Gershgorin bound of D^-1 A (max over rows of sum |a_ij| / |a_ii|) for the fine level.
__global__ void k_gersh_fine(Grid g, const double *coef, const double *invd, const uint8_t *fluid, double *parts) {
  __shared__ double sh[256];
  double mval = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    if (!fluid[p]) continue;
    double s = 0;
    for (int t = 0; t < NSLOT; t++) s += fabs(coef[t * g.N + p]);
    mval = fmax(mval, s * fabs(invd[p]));
  }
  sh[threadIdx.x] = mval;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// ------------------------------------------------------------------ reductions
// Partial sums of up to NV dot products <v_i, w> plus <w,w>, one pass over w.
template <int NV>
__global__ void k_multidot(long long n, const double *__restrict__ V, int nv, const double *__restrict__ w,
                           double *parts) {
  // parts layout: [nv+1][gridDim.x]
  __shared__ double sh[NV + 1][128];
  double acc[NV + 1];
#pragma unroll
  for (int t = 0; t <= NV; t++) acc[t] = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += stride) {
    const double wp = w[p];
#pragma unroll
    for (int t = 0; t < NV; t++)
      if (t < nv) acc[t] += V[(long long)t * n + p] * wp;
    acc[NV] += wp * wp;
  }
  for (int t = 0; t <= NV; t++) sh[t][threadIdx.x] = acc[t];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int t = 0; t <= NV; t++) sh[t][threadIdx.x] += sh[t][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int t = 0; t < nv; t++) parts[(long long)t * gridDim.x + blockIdx.x] = sh[t][0];
    parts[(long long)nv * gridDim.x + blockIdx.x] = sh[NV][0];
  }
}

__global__ void k_sum_rows(const double *parts, int nrows, int ncols, double *out) {
  int r = blockIdx.x;
  if (r >= nrows) return;
  __shared__ double sh[256];
  double s = 0;
  for (int q = threadIdx.x; q < ncols; q += blockDim.x) s += parts[(long long)r * ncols + q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[r] = sh[0];
}

// w -= sum_i h_i v_i
__global__ void k_orth_update(long long n, const double *__restrict__ V, int nv, const double *__restrict__ h,
                              double *__restrict__ w) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double s = w[p];
  for (int t = 0; t < nv; t++) s -= h[t] * V[(long long)t * n + p];
  w[p] = s;
}
__global__ void k_scale_copy(long long n, const double *a, double s, double *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) b[p] = a[p] * s;
}
// x += sum_i y_i Z_i
__global__ void k_lincomb_add(long long n, const double *__restrict__ Z, int m, const double *__restrict__ y,
                              double *__restrict__ x) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double s = x[p];
  for (int t = 0; t < m; t++) s += y[t] * Z[(long long)t * n + p];
  x[p] = s;
}
// r = b - y
__global__ void k_sub(long long n, const double *b, const double *y, double *r) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) r[p] = b[p] - y[p];
}

static const int kRedBlocks = 148 * 2;

// Dots <V_t, w> for t < nv and <w, w>; results in c->red_host[0..nv].
static int multidot(Ctx *c, const double *V, int nv, const double *w, double *out) {
  int rc;
  const long long n = c->g.N;
  if ((rc = ensure_red(c, (nv + 1) * kRedBlocks + 64 + nv + 1))) return rc;
  double *parts = c->red;
  double *res = c->red + (nv + 1) * kRedBlocks;
  if (nv <= 8) k_multidot<8><<<kRedBlocks, 128, 0, c->stream>>>(n, V, nv, w, parts);
  else if (nv <= 16) k_multidot<16><<<kRedBlocks, 128, 0, c->stream>>>(n, V, nv, w, parts);
  else if (nv <= 32) k_multidot<32><<<kRedBlocks, 128, 0, c->stream>>>(n, V, nv, w, parts);
  else return set_err(c, VFS_ERR_INVALID, "FGMRES restart above 32 is not supported");
  if ((rc = check_launch(c, "k_multidot"))) return rc;
  k_sum_rows<<<nv + 1, 256, 0, c->stream>>>(parts, nv + 1, kRedBlocks, res);
  if ((rc = check_launch(c, "k_sum_rows"))) return rc;
  cudaMemcpyAsync(c->red_host, res, sizeof(double) * (nv + 1), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "multidot sync failed");
  for (int t = 0; t <= nv; t++) out[t] = c->red_host[t];
  return VFS_OK;
}


// ------------------------------------------------------------------ LHS set-up
__global__ void k_count_fluid(long long n, const uint8_t *fluid, const double *aj, double *parts) {
  __shared__ double s1[256], s2[256];
  double a = 0, b = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += stride)
    if (fluid[p]) { a += 1.0; b += aj[p]; }
  s1[threadIdx.x] = a; s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { parts[blockIdx.x] = s1[0]; parts[gridDim.x + blockIdx.x] = s2[0]; }
}

static CL clevel(const Ctx *c, const MGLevel &L) {
  CL r;
  r.nx = L.nx; r.ny = L.ny; r.nz = L.nz; r.n = L.n;
  r.ip = c->g.iper; r.jp = c->g.jper; r.kp = c->g.kper;
  return r;
}

static void free_levels(Poisson &P) {
  for (size_t l = 1; l < P.lv.size(); l++) {
    MGLevel &L = P.lv[l];
    cudaFree(L.op64); cudaFree(L.op32); cudaFree(L.x64); cudaFree(L.x32);
  }
  P.lv.clear();
}

static double gersh_max(Ctx *c) {
  k_gersh_fine<<<kRedBlocks, 256, 0, c->stream>>>(c->g, c->ps.coef, c->ps.invdiag, c->ps.fluid, c->red);
  check_launch(c, "k_gersh_fine");
  std::vector<double> h(kRedBlocks);
  cudaMemcpyAsync(h.data(), c->red, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  double m = 0;
  for (double v : h) m = std::max(m, v);
  return m;
}

int poisson_lhs(Ctx *c) {
  Poisson &P = c->ps;
  const Grid &g = c->g;
  const long long N = g.N;
  int rc;
  if (!P.coef) {
    bool ok = cudaMalloc(&P.coef, sizeof(double) * NSLOT * N) == cudaSuccess;
    ok &= cudaMalloc(&P.coef32, sizeof(float) * NSLOT * N) == cudaSuccess;
    ok &= cudaMalloc(&P.invdiag, sizeof(double) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.invdiag32, sizeof(float) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.fluid, N) == cudaSuccess;
    ok &= cudaMalloc(&P.f32, sizeof(float) * N * 6) == cudaSuccess;
    ok &= cudaMalloc(&P.f64, sizeof(double) * N * 6) == cudaSuccess;
    ok &= cudaMalloc(&P.w, sizeof(double) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.r, sizeof(double) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.t, sizeof(double) * N) == cudaSuccess;
    if (!ok) return set_err(c, VFS_ERR_CUDA, "poisson_lhs: allocation failed");
    cudaMemsetAsync(P.f32, 0, sizeof(float) * N * 6, c->stream);
    cudaMemsetAsync(P.f64, 0, sizeof(double) * N * 6, c->stream);
    cudaMemsetAsync(P.w, 0, sizeof(double) * N, c->stream);
    cudaMemsetAsync(P.r, 0, sizeof(double) * N, c->stream);
    cudaMemsetAsync(P.t, 0, sizeof(double) * N, c->stream);
  }
  k_poisson_coef<<<nblocks(N, 128), 128, 0, c->stream>>>(g, metrics(c), c->nv, P.coef, P.fluid, P.invdiag);
  if ((rc = check_launch(c, "k_poisson_coef"))) return rc;
  k_cast_d2f<<<nblocks(NSLOT * N, 256), 256, 0, c->stream>>>(NSLOT * N, P.coef, P.coef32);
  if ((rc = check_launch(c, "k_cast_d2f"))) return rc;
  k_cast_d2f<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.invdiag, P.invdiag32);
  if ((rc = check_launch(c, "k_cast_d2f"))) return rc;
  // fluid-cell count and sum of aj (Remove_Nullspace / Remove_Nullspace_Scale)
  if ((rc = ensure_red(c, 2 * kRedBlocks + 64))) return rc;
  k_count_fluid<<<kRedBlocks, 256, 0, c->stream>>>(N, P.fluid, c->f[VFS_AJ][0], c->red);
  if ((rc = check_launch(c, "k_count_fluid"))) return rc;
  double cnt = 0, saj = 0;
  if ((rc = reduce_sum(c, c->red, kRedBlocks, &cnt))) return rc;
  if ((rc = reduce_sum(c, c->red + kRedBlocks, kRedBlocks, &saj))) return rc;
  P.nfluid = (long long)llround(cnt);
  P.sum_aj = saj;
  P.lmax0 = gersh_max(c);

  // Multigrid hierarchy: coarsen by 2 while every interior dimension stays even.
  free_levels(P);
  MGLevel L0;
  L0.nx = g.mx - 2; L0.ny = g.my - 2; L0.nz = g.mz - 2;
  L0.n = N;
  P.lv.push_back(L0);
  const int maxlev = 8;
  while ((int)P.lv.size() < maxlev) {
    const MGLevel F = P.lv.back();
    if (F.nx % 2 || F.ny % 2 || F.nz % 2 || F.nx < 4 || F.ny < 4 || F.nz < 4) break;
    MGLevel L;
    L.nx = F.nx / 2; L.ny = F.ny / 2; L.nz = F.nz / 2;
    L.n = (long long)L.nx * L.ny * L.nz;
    bool ok = cudaMalloc(&L.op64, sizeof(double) * L.n * 4) == cudaSuccess;
    ok &= cudaMalloc(&L.op32, sizeof(float) * L.n * 4) == cudaSuccess;
    ok &= cudaMalloc(&L.x64, sizeof(double) * L.n * 6) == cudaSuccess;
    ok &= cudaMalloc(&L.x32, sizeof(float) * L.n * 6) == cudaSuccess;
    if (!ok) return set_err(c, VFS_ERR_CUDA, "poisson_lhs: level allocation failed");
    L.b64 = L.x64 + L.n; L.d64 = L.b64 + L.n; L.t64 = L.d64 + L.n;
    L.b32 = L.x32 + L.n; L.d32 = L.b32 + L.n; L.t32 = L.d32 + L.n;
    cudaMemsetAsync(L.x64, 0, sizeof(double) * L.n * 6, c->stream);
    cudaMemsetAsync(L.x32, 0, sizeof(float) * L.n * 6, c->stream);
    double *cx = L.op64, *cy = cx + L.n, *cz = cy + L.n, *dg = cz + L.n;
    CL Lc = clevel(c, L);
    if (P.lv.size() == 1) {
      k_build_l1<<<nblocks(L.n, 128), 128, 0, c->stream>>>(g, Lc, P.coef, P.fluid, cx, cy, cz);
    } else {
      const double *f = F.op64;
      k_build_coarse<<<nblocks(L.n, 128), 128, 0, c->stream>>>(clevel(c, F), Lc, f, f + F.n, f + 2 * F.n, cx, cy, cz);
    }
    if ((rc = check_launch(c, "k_build_level"))) return rc;
    k_coarse_diag<<<nblocks(L.n, 128), 128, 0, c->stream>>>(Lc, cx, cy, cz, dg);
    if ((rc = check_launch(c, "k_coarse_diag"))) return rc;
    k_cast_d2f<<<nblocks(4 * L.n, 256), 256, 0, c->stream>>>(4 * L.n, L.op64, L.op32);
    if ((rc = check_launch(c, "k_cast_d2f"))) return rc;
    P.lv.push_back(L);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "poisson_lhs failed");
  P.built = true;
  return VFS_OK;
}

// ------------------------------------------------------------------ V-cycle
// Chebyshev polynomial smoothing of D^-1 A on [lmin, lmax] (the classical three-term
// recurrence): step coefficients c1 (momentum) and c2 (residual weight) per step.
static void cheb_coeffs(double lmax, int steps, std::vector<double> &c1, std::vector<double> &c2) {
  const double hi = 1.1 * lmax, lo = hi / 8.0;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  c1.assign(steps, 0.0); c2.assign(steps, 0.0);
  c1[0] = 0.0; c2[0] = 1.0 / theta;
  for (int s = 1; s < steps; s++) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    c1[s] = rn * rho;
    c2[s] = 2.0 * rn / delta;
    rho = rn;
  }
}

template <typename T> struct LvPtr;
template <> struct LvPtr<float> {
  static float *x(MGLevel &L) { return L.x32; }
  static float *b(MGLevel &L) { return L.b32; }
  static float *d(MGLevel &L) { return L.d32; }
  static float *t(MGLevel &L) { return L.t32; }
  static const float *op(MGLevel &L) { return L.op32; }
};
template <> struct LvPtr<double> {
  static double *x(MGLevel &L) { return L.x64; }
  static double *b(MGLevel &L) { return L.b64; }
  static double *d(MGLevel &L) { return L.d64; }
  static double *t(MGLevel &L) { return L.t64; }
  static const double *op(MGLevel &L) { return L.op64; }
};

template <typename T> struct FineOps;
template <> struct FineOps<float> {
  static const float *coef(Poisson &P) { return P.coef32; }
  static const float *invd(Poisson &P) { return P.invdiag32; }
  static float *work(Poisson &P) { return P.f32; }
};
template <> struct FineOps<double> {
  static const double *coef(Poisson &P) { return P.coef; }
  static const double *invd(Poisson &P) { return P.invdiag; }
  static double *work(Poisson &P) { return P.f64; }
};

// Smoothing of level l: damped y-line Jacobi sweeps (omega = 0.8); x is updated in place
// (ping-pong through t, the Thomas coefficients in the two scratch slots after it).
static const double kLineOmega = 0.8;
template <typename T>
static int smooth(Ctx *c, int l, int steps, bool x_zero) {
  Poisson &P = c->ps;
  int rc;
  if (l == 0) {
    const long long N = c->g.N;
    T *w = FineOps<T>::work(P);
    T *b = w, *x = w + N, *xt = w + 2 * N, *cp = w + 4 * N, *dp = w + 5 * N;
    const long long cols = (long long)(c->g.mx - 2) * (c->g.mz - 2);
    for (int s = 0; s < steps; s++) {
      const bool z = x_zero && s == 0;
      k_yline_fine<T><<<nblocks(cols, 128), 128, 0, c->stream>>>(c->g, FineOps<T>::coef(P), P.fluid, b, x, xt, cp, dp,
                                                                (T)kLineOmega, z ? 1 : 0);
      if ((rc = check_launch(c, "k_yline_fine"))) return rc;
      std::swap(x, xt);
    }
    if (x != w + N) cudaMemcpyAsync(w + N, x, sizeof(T) * N, cudaMemcpyDeviceToDevice, c->stream);
    return VFS_OK;
  }
  MGLevel &L = P.lv[l];
  CL cl = clevel(c, L);
  const T *op = LvPtr<T>::op(L);
  T *x = LvPtr<T>::x(L), *xt = LvPtr<T>::t(L);
  T *cp = LvPtr<T>::x(L) + 4 * L.n, *dp = LvPtr<T>::x(L) + 5 * L.n;
  const long long cols = (long long)L.nx * L.nz;
  for (int s = 0; s < steps; s++) {
    const bool z = x_zero && s == 0;
    k_yline_coarse<T><<<nblocks(cols, 128), 128, 0, c->stream>>>(cl, op, op + L.n, op + 2 * L.n, op + 3 * L.n,
                                                                LvPtr<T>::b(L), x, xt, cp, dp, (T)kLineOmega,
                                                                z ? 1 : 0);
    if ((rc = check_launch(c, "k_yline_coarse"))) return rc;
    std::swap(x, xt);
  }
  if (x != LvPtr<T>::x(L)) cudaMemcpyAsync(LvPtr<T>::x(L), x, sizeof(T) * L.n, cudaMemcpyDeviceToDevice, c->stream);
  return VFS_OK;
}

// V-cycle on level l for the right-hand side already in the level's b slot.
template <typename T>
static int vcycle(Ctx *c, int l, const vfs_solve_opts &o) {
  Poisson &P = c->ps;
  const int nl = std::min((int)P.lv.size(), o.levels);
  int rc;
  if (l == nl - 1) return smooth<T>(c, l, o.coarse_iters, true);
  if ((rc = smooth<T>(c, l, o.pre_smooth, true))) return rc;
  MGLevel &C = P.lv[l + 1];
  CL cc = clevel(c, C);
  if (l == 0) {
    const long long N = c->g.N;
    T *w = FineOps<T>::work(P);
    k_restrict_fine<T><<<nblocks(C.n, 128), 128, 0, c->stream>>>(c->g, cc, FineOps<T>::coef(P), P.fluid, w, w + N,
                                                                LvPtr<T>::b(C));
  } else {
    MGLevel &F = P.lv[l];
    const T *op = LvPtr<T>::op(F);
    k_restrict_coarse<T><<<nblocks(C.n, 128), 128, 0, c->stream>>>(clevel(c, F), cc, op, op + F.n, op + 2 * F.n,
                                                                  op + 3 * F.n, LvPtr<T>::b(F), LvPtr<T>::x(F),
                                                                  LvPtr<T>::b(C));
  }
  if ((rc = check_launch(c, "k_restrict"))) return rc;
  if ((rc = vcycle<T>(c, l + 1, o))) return rc;
  if (l == 0) {
    T *w = FineOps<T>::work(P);
    k_prolong_fine<T><<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, cc, P.fluid, w + c->g.N, LvPtr<T>::x(C));
  } else {
    MGLevel &F = P.lv[l];
    const T *op = LvPtr<T>::op(F);
    k_prolong_coarse<T><<<nblocks(F.n, 256), 256, 0, c->stream>>>(clevel(c, F), cc, op + 3 * F.n, LvPtr<T>::x(F),
                                                                  LvPtr<T>::x(C));
  }
  if ((rc = check_launch(c, "k_prolong"))) return rc;
  return smooth<T>(c, l, o.post_smooth, false);
}

// z = M^-1 v (one V-cycle, FP32 or FP64), v and z on the grid layout in FP64.
static int precondition(Ctx *c, const double *v, double *z, const vfs_solve_opts &o) {
  Poisson &P = c->ps;
  const long long N = c->g.N;
  int rc;
  if (o.precision == 0) {
    k_cast_d2f<<<nblocks(N, 256), 256, 0, c->stream>>>(N, v, P.f32);
    if ((rc = check_launch(c, "k_cast_d2f"))) return rc;
    if ((rc = vcycle<float>(c, 0, o))) return rc;
    k_cast_f2d<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.f32 + N, z);
    return check_launch(c, "k_cast_f2d");
  }
  cudaMemcpyAsync(P.f64, v, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream);
  if ((rc = vcycle<double>(c, 0, o))) return rc;
  cudaMemcpyAsync(z, P.f64 + N, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream);
  return VFS_OK;
}

// ------------------------------------------------------------------ RHS
// PoissonRHS2_hypre (poisson_hypre.c:330-360): b = div(Ucont) / dt * st at fluid cells,
// with the periodic neighbour of the first interior face taken from its image.
__global__ void k_poisson_rhs(Grid g, CV3 uc, const uint8_t *__restrict__ fluid, double *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  if (!fluid[p]) { b[p] = 0; return; }
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  const long long sy = mx, sz = (long long)mx * my;
  const double coeff = 1.0;  // time_coeff() (poisson.c:17) without levelset/RANS
  double val = 0;
  val -= uc.x[p];
  if (i == 1 && g.iper) val += uc.x[p - 1 + (mx - 2)];
  else val += uc.x[p - 1];
  val -= uc.y[p];
  if (j == 1 && g.jper) val += uc.y[p - sy + (long long)(my - 2) * sy];
  else val += uc.y[p - sy];
  val -= uc.z[p];
  if (k == 1 && g.kper) val += uc.z[p - sz + (long long)(mz - 2) * sz];
  else val += uc.z[p - sz];
  val *= -1.0 / g.dt * g.st * coeff;
  b[p] = val;
}

// b += -sum(b) * aj / sum(aj) on fluid cells (Remove_Nullspace_Scale, poisson_hypre.c:110).
__global__ void k_shift_scaled(long long n, const uint8_t *fluid, const double *aj, double sum, double sum_aj,
                               double *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n || !fluid[p]) return;
  double val = -sum * aj[p] / sum_aj;
  b[p] += val;
}
// x += val on fluid cells (Remove_Nullspace, poisson_hypre.c:194).
__global__ void k_shift(long long n, const uint8_t *fluid, double val, double *x) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n || !fluid[p]) return;
  x[p] += val;
}

__global__ void k_sum_fluid(long long n, const uint8_t *fluid, const double *a, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += stride)
    if (fluid[p]) s += a[p];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

static int sum_fluid(Ctx *c, const double *a, double *out) {
  int rc;
  if ((rc = ensure_red(c, kRedBlocks + 64))) return rc;
  k_sum_fluid<<<kRedBlocks, 256, 0, c->stream>>>(c->g.N, c->ps.fluid, a, c->red);
  if ((rc = check_launch(c, "k_sum_fluid"))) return rc;
  return reduce_sum(c, c->red, kRedBlocks, out);
}

// VolumeFlux(user, Ucont, ...) (poisson.c:3306-3500) without sharp-interface IB nodes
// (immersed = 0): the flux through every interior face between a fluid cell and a
// non-fluid cell is set to zero.  The face index is the lower cell of the pair, as in
// the reference loops over interior cells (i <= mx-2 always holds there).
__global__ void k_volume_flux_blocked(Grid g, const uint8_t *__restrict__ nv, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i = (int)(p % g.mx);
  long long q = p / g.mx;
  int j = (int)(q % g.my);
  int k = (int)(q / g.my);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  const bool f0 = nv[p] == 0;
  if (f0) {
    if (nv[p + 1] > 0) uc.x[p] = 0;
    if (nv[p + sy] > 0) uc.y[p] = 0;
    if (nv[p + sz] > 0) uc.z[p] = 0;
  } else {
    if (nv[p + 1] == 0) uc.x[p] = 0;
    if (nv[p + sy] == 0) uc.y[p] = 0;
    if (nv[p + sz] == 0) uc.z[p] = 0;
  }
}

int volume_flux(Ctx *c) {
  if (c->g.immersed) return set_err(c, VFS_ERR_INVALID, "VolumeFlux: IB-node flux balance is not on this path yet");
  k_volume_flux_blocked<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->nv, field3(c, VFS_UCONT));
  return check_launch(c, "k_volume_flux_blocked");
}

int poisson_rhs(Ctx *c) {
  int rc;
  double *b = c->f[VFS_B][0];
  if ((rc = periodic_copy3(c, field3(c, VFS_UCONT)))) return rc;
  k_poisson_rhs<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_UCONT)), c->ps.fluid, b);
  if ((rc = check_launch(c, "k_poisson_rhs"))) return rc;
  double sum = 0;
  if ((rc = sum_fluid(c, b, &sum))) return rc;
  k_shift_scaled<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, c->ps.fluid, c->f[VFS_AJ][0], sum,
                                                             c->ps.sum_aj, b);
  return check_launch(c, "k_shift_scaled");
}

// ------------------------------------------------------------------ FGMRES
// Right-preconditioned flexible GMRES (Saad 1993) in FP64 with classical Gram-Schmidt
// and one re-orthogonalisation pass.  Solves A phi = b for the fluid unknowns, starting
// from phi = 0 as HYPRE does with a zero initial vector (Petsc_to_Hypre_Vector of a fresh
// Phi2), then removes the mean (Remove_Nullspace) and fills the grid Phi like
// Convert_Phi2_Phi (poisson.c:92): non-fluid interior cells 0, periodic ghosts from
// their images, other ghosts 0.
int poisson_solve(Ctx *c, const vfs_solve_opts *oin, vfs_solve_stats *st) {
  vfs_solve_opts o;
  memset(&o, 0, sizeof(o));
  o.precision = 0; o.restart = 30; o.max_iter = 200; o.levels = 4; o.pre_smooth = 2; o.post_smooth = 2;
  o.coarse_iters = 16; o.rtol = 1e-10; o.atol = 0.0;
  if (oin) {
    o.precision = oin->precision;
    if (oin->restart > 0) o.restart = oin->restart;
    if (oin->max_iter > 0) o.max_iter = oin->max_iter;
    if (oin->levels > 0) o.levels = oin->levels;
    if (oin->pre_smooth > 0) o.pre_smooth = oin->pre_smooth;
    if (oin->post_smooth > 0) o.post_smooth = oin->post_smooth;
    if (oin->coarse_iters > 0) o.coarse_iters = oin->coarse_iters;
    if (oin->rtol > 0) o.rtol = oin->rtol;
    if (oin->atol > 0) o.atol = oin->atol;
  }
  if (o.restart > 32) o.restart = 32;
  Poisson &P = c->ps;
  const long long N = c->g.N;
  int rc;
  if (P.restart < o.restart) {
    cudaFree(P.V); cudaFree(P.Z);
    P.V = P.Z = nullptr;
    if (cudaMalloc(&P.V, sizeof(double) * N * (o.restart + 1)) != cudaSuccess ||
        cudaMalloc(&P.Z, sizeof(double) * N * o.restart) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "poisson_solve: Krylov basis allocation failed");
    P.restart = o.restart;
  }
  cudaEventRecord(c->ev0, c->stream);
  double *x = c->f[VFS_PHI][0];
  const double *b = c->f[VFS_B][0];
  cudaMemsetAsync(x, 0, sizeof(double) * N, c->stream);
  const int m = o.restart;
  std::vector<double> H((m + 1) * m), cs(m), sn(m), gv(m + 1), y(m), h(m + 2), h2(m + 2);
  double bnorm = 0;
  {
    double dd[1];
    if ((rc = multidot(c, nullptr, 0, b, dd))) return rc;
    bnorm = sqrt(dd[0]);
  }
  vfs_solve_stats s;
  memset(&s, 0, sizeof(s));
  s.r0 = bnorm;
  const double tol = std::max(o.rtol * bnorm, o.atol);
  int it = 0;
  bool conv = bnorm <= tol;
  double rnorm = bnorm;
  while (!conv && it < o.max_iter) {
    // r = b - A x
    if ((rc = poisson_apply_dev(c, x, P.t))) return rc;
    k_sub<<<nblocks(N, 256), 256, 0, c->stream>>>(N, b, P.t, P.r);
    if ((rc = check_launch(c, "k_sub"))) return rc;
    double rr[1];
    if ((rc = multidot(c, nullptr, 0, P.r, rr))) return rc;
    double beta = sqrt(rr[0]);
    rnorm = beta;
    if (beta <= tol) { conv = true; break; }
    k_scale_copy<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.r, 1.0 / beta, P.V);
    if ((rc = check_launch(c, "k_scale_copy"))) return rc;
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int jdone = 0;
    for (int j = 0; j < m && it < o.max_iter; j++) {
      double *Vj = P.V + (long long)j * N, *Zj = P.Z + (long long)j * N;
      if ((rc = precondition(c, Vj, Zj, o))) return rc;
      if ((rc = poisson_apply_dev(c, Zj, P.w))) return rc;
      // CGS with one re-orthogonalisation pass
      if ((rc = multidot(c, P.V, j + 1, P.w, h.data()))) return rc;
      cudaMemcpyAsync(c->red + 8, h.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, c->stream);
      k_orth_update<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.V, j + 1, c->red + 8, P.w);
      if ((rc = check_launch(c, "k_orth_update"))) return rc;
      if ((rc = multidot(c, P.V, j + 1, P.w, h2.data()))) return rc;
      cudaMemcpyAsync(c->red + 8, h2.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, c->stream);
      k_orth_update<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.V, j + 1, c->red + 8, P.w);
      if ((rc = check_launch(c, "k_orth_update"))) return rc;
      double nn[1];
      if ((rc = multidot(c, nullptr, 0, P.w, nn))) return rc;
      for (int t = 0; t <= j; t++) H[t * m + j] = h[t] + h2[t];
      const double hn = sqrt(nn[0]);
      H[(j + 1) * m + j] = hn;
      if (hn > 0) {
        k_scale_copy<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.w, 1.0 / hn, P.V + (long long)(j + 1) * N);
        if ((rc = check_launch(c, "k_scale_copy"))) return rc;
      }
      // Givens rotations
      for (int t = 0; t < j; t++) {
        const double a = H[t * m + j], bb = H[(t + 1) * m + j];
        H[t * m + j] = cs[t] * a + sn[t] * bb;
        H[(t + 1) * m + j] = -sn[t] * a + cs[t] * bb;
      }
      const double a = H[j * m + j], bb = H[(j + 1) * m + j];
      const double den = sqrt(a * a + bb * bb);
      cs[j] = den > 0 ? a / den : 1.0;
      sn[j] = den > 0 ? bb / den : 0.0;
      H[j * m + j] = den;
      H[(j + 1) * m + j] = 0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      it++;
      jdone = j + 1;
      rnorm = fabs(gv[j + 1]);
      if (rnorm <= tol || hn == 0) break;
    }
    // back substitution and update x += Z y
    for (int t = jdone - 1; t >= 0; t--) {
      double sum = gv[t];
      for (int u = t + 1; u < jdone; u++) sum -= H[t * m + u] * y[u];
      y[t] = sum / H[t * m + t];
    }
    cudaMemcpyAsync(c->red + 8, y.data(), sizeof(double) * jdone, cudaMemcpyHostToDevice, c->stream);
    k_lincomb_add<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.Z, jdone, c->red + 8, x);
    if ((rc = check_launch(c, "k_lincomb_add"))) return rc;
    if (rnorm <= tol) {
      // confirm with the true residual
      if ((rc = poisson_apply_dev(c, x, P.t))) return rc;
      k_sub<<<nblocks(N, 256), 256, 0, c->stream>>>(N, b, P.t, P.r);
      if ((rc = check_launch(c, "k_sub"))) return rc;
      double r2[1];
      if ((rc = multidot(c, nullptr, 0, P.r, r2))) return rc;
      rnorm = sqrt(r2[0]);
      conv = rnorm <= tol * 1.0000001 || rnorm <= 2 * tol;
    }
  }
  // Remove_Nullspace: phi += -mean(phi) over fluid cells
  double sum = 0;
  if ((rc = sum_fluid(c, x, &sum))) return rc;
  const double val = -sum / (double)P.nfluid;
  k_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.fluid, val, x);
  if ((rc = check_launch(c, "k_shift"))) return rc;
  // Convert_Phi2_Phi: periodic ghosts take their images (x is 0 elsewhere off-fluid)
  if ((rc = periodic_copy1(c, x))) return rc;
  cudaEventRecord(c->ev1, c->stream);
  cudaEventSynchronize(c->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  s.iterations = it;
  s.converged = conv ? 1 : 0;
  s.rfinal = rnorm;
  s.ms = ms;
  if (st) *st = s;
  return conv ? VFS_OK : set_err(c, VFS_ERR_NOT_CONVERGED, "poisson_solve: iteration cap reached");
}

// ------------------------------------------------------------------ UpdatePressure
// poisson.c:3144-3305: P += Phi on fluid cells, P = 0 where nvert > 1.1, then the
// periodic ghosts of P and Phi take their images.
__global__ void k_update_pressure(Grid g, const uint8_t *__restrict__ nv, const double *__restrict__ phi, double *P) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i = (int)(p % g.mx);
  long long q = p / g.mx;
  int j = (int)(q % g.my);
  int k = (int)(q / g.my);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  if (nv[p] == 0) P[p] += phi[p];
  if (nv[p] >= 2) P[p] = 0;
}

int update_pressure(Ctx *c) {
  int rc;
  k_update_pressure<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->nv, c->f[VFS_PHI][0], c->f[VFS_P][0]);
  if ((rc = check_launch(c, "k_update_pressure"))) return rc;
  if ((rc = periodic_copy1(c, c->f[VFS_P][0]))) return rc;
  return periodic_copy1(c, c->f[VFS_PHI][0]);
}

// ------------------------------------------------------------------ Projection
// poisson.c:2780-2970 (levelset off): Ucont -= G(Phi) * dt * st on faces whose two
// cells are fluid, with one-sided cross differences next to solids and walls.
__device__ __forceinline__ double cross_phi(const double *phi, long long a0, long long a1, long long dp,
                                            int ecoord, int em, int eper, int nplus, int nminus) {
  // a0, a1: the two face cells; dp: stride of the cross direction
  if ((ecoord == em - 2 && !eper) || nplus > 0) {
    if (nminus == 0 && ecoord != 1) return (phi[a0] + phi[a1] - phi[a0 - dp] - phi[a1 - dp]) * 0.5;
    return 0.;
  } else if ((ecoord == 1 && !eper) || nminus > 0) {
    if (nplus == 0) return (phi[a0 + dp] + phi[a1 + dp] - phi[a0] - phi[a1]) * 0.5;
    return 0.;
  }
  return (phi[a0 + dp] + phi[a1 + dp] - phi[a0 - dp] - phi[a1 - dp]) * 0.25;
}

__global__ void k_projection(Grid g, Metrics m, const uint8_t *__restrict__ nv, const double *__restrict__ phi, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) return;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const double coeff = 1.0, r1 = 1.0, r2 = 1.0, r3 = 1.0;
  const double fac = g.dt * g.st;
  if (i < mx - 2 || (g.iper && i == mx - 2)) {
    double dpdc = phi[p + 1] - phi[p];
    if (i == mx - 2 && g.iper) dpdc = phi[p - i + 1] - phi[p];
    const double dpde = cross_phi(phi, p, p + sx, sy, j, my, g.jper, nv[p + sy] + nv[p + sy + sx], nv[p - sy] + nv[p - sy + sx]);
    const double dpdz = cross_phi(phi, p, p + sx, sz, k, mz, g.kper, nv[p + sz] + nv[p + sz + sx], nv[p - sz] + nv[p - sz + sx]);
    if (nv[p] + nv[p + 1] == 0) {
      const double ix = m.icsi.x[p], iy = m.icsi.y[p], iz = m.icsi.z[p], a = m.iaj[p];
      uc.x[p] -= (dpdc * (ix * ix + iy * iy + iz * iz) * a +
                  dpde * (m.ieta.x[p] * ix + m.ieta.y[p] * iy + m.ieta.z[p] * iz) * a +
                  dpdz * (m.izet.x[p] * ix + m.izet.y[p] * iy + m.izet.z[p] * iz) * a) *
                 g.dt * g.st / coeff / r1;
    }
  }
  if (j < my - 2 || (g.jper && j == my - 2)) {
    const double dpdc = cross_phi(phi, p, p + sy, sx, i, mx, g.iper, nv[p + sx] + nv[p + sy + sx], nv[p - sx] + nv[p + sy - sx]);
    double dpde;
    if (j == my - 2 && g.jper) dpde = phi[p - (long long)j * sy + sy] - phi[p];
    else dpde = phi[p + sy] - phi[p];
    const double dpdz = cross_phi(phi, p, p + sy, sz, k, mz, g.kper, nv[p + sz] + nv[p + sz + sy], nv[p - sz] + nv[p - sz + sy]);
    if (nv[p] + nv[p + sy] == 0 || nv[p] + nv[p + sy] == 5) {
      const double jx = m.jeta.x[p], jy = m.jeta.y[p], jz = m.jeta.z[p], a = m.jaj[p];
      uc.y[p] -= (dpdc * (m.jcsi.x[p] * jx + m.jcsi.y[p] * jy + m.jcsi.z[p] * jz) * a +
                  dpde * (jx * jx + jy * jy + jz * jz) * a +
                  dpdz * (m.jzet.x[p] * jx + m.jzet.y[p] * jy + m.jzet.z[p] * jz) * a) *
                 g.dt * g.st / coeff / r2;
    }
  }
  if (k < mz - 2 || (g.kper && k == mz - 2)) {
    const double dpdc = cross_phi(phi, p, p + sz, sx, i, mx, g.iper, nv[p + sx] + nv[p + sz + sx], nv[p - sx] + nv[p + sz - sx]);
    const double dpde = cross_phi(phi, p, p + sz, sy, j, my, g.jper, nv[p + sy] + nv[p + sz + sy], nv[p - sy] + nv[p + sz - sy]);
    double dpdz;
    if (k == mz - 2 && g.kper) dpdz = phi[p - (long long)k * sz + sz] - phi[p];
    else dpdz = phi[p + sz] - phi[p];
    if (nv[p] + nv[p + sz] == 0) {
      const double kx = m.kzet.x[p], ky = m.kzet.y[p], kz = m.kzet.z[p], a = m.kaj[p];
      uc.z[p] -= (dpdc * (m.kcsi.x[p] * kx + m.kcsi.y[p] * ky + m.kcsi.z[p] * kz) * a +
                  dpde * (m.keta.x[p] * kx + m.keta.y[p] * ky + m.keta.z[p] * kz) * a +
                  dpdz * (kx * kx + ky * ky + kz * kz) * a) *
                 g.dt * g.st / coeff / r3;
    }
  }
  (void)fac;
}

// Component-wise periodic copy after Projection (poisson.c:3013-3046): a component is
// copied only when its own direction is periodic at the point.
__global__ void k_periodic_copy_comp(Grid g, V3 u) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i = (int)(p % g.mx);
  long long q = p / g.mx;
  int j = (int)(q % g.my);
  int k = (int)(q / g.my);
  int ii = wrapi(g, i), jj = wrapj(g, j), kk = wrapk(g, k);
  if (ii == i && jj == j && kk == k) return;
  long long s = lidx(g, ii, jj, kk);
  if (ii != i) u.x[p] = u.x[s];
  if (jj != j) u.y[p] = u.y[s];
  if (kk != k) u.z[p] = u.z[s];
}

int projection(Ctx *c) {
  int rc;
  k_projection<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), c->nv, c->f[VFS_PHI][0],
                                                           field3(c, VFS_UCONT));
  if ((rc = check_launch(c, "k_projection"))) return rc;
  if (c->g.iper || c->g.jper || c->g.kper) {
    k_periodic_copy_comp<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
    if ((rc = check_launch(c, "k_periodic_copy_comp"))) return rc;
  }
  return contra2cart(c);
}

// ------------------------------------------------------------------ Divergence
// main.c:1083-1090: max |(dU + dV + dW) * aj| over interior cells with no solid in the
// 7-point neighbourhood.
__global__ void k_divergence(Grid g, CV3 uc, const double *__restrict__ aj, const uint8_t *__restrict__ nv,
                             double *parts) {
  __shared__ double sh[256];
  double mval = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    int i = (int)(p % g.mx);
    long long q = p / g.mx;
    int j = (int)(q % g.my);
    int k = (int)(q / g.my);
    if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) continue;
    double d = fabs((uc.x[p] - uc.x[p - 1] + uc.y[p] - uc.y[p - sy] + uc.z[p] - uc.z[p - sz]) * aj[p]);
    if (nv[p] + nv[p + sz] + nv[p - sz] + nv[p + sy] + nv[p - sy] + nv[p + 1] + nv[p - 1] > 0) d = 0.;
    mval = fmax(mval, d);
  }
  sh[threadIdx.x] = mval;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

int divergence(Ctx *c, double *maxdiv) {
  int rc;
  if ((rc = ensure_red(c, kRedBlocks + 64))) return rc;
  k_divergence<<<kRedBlocks, 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_UCONT)), c->f[VFS_AJ][0], c->nv, c->red);
  if ((rc = check_launch(c, "k_divergence"))) return rc;
  cudaMemcpyAsync(c->red_host, c->red, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "divergence sync failed");
  double m = 0;
  for (int q = 0; q < kRedBlocks; q++) m = std::max(m, c->red_host[q]);
  *maxdiv = m;
  return VFS_OK;
}

}  // namespace vfs

// ------------------------------------------------------------------ diagnostics
namespace vfs {
// Launches one kernel of the path `reps` times on the context's stream (no host sync),
// so a caller can bracket it with events recorded on that stream.
int run_kernel(Ctx *c, int which, int reps) {
  const Grid &g = c->g;
  Poisson &P = c->ps;
  int rc = VFS_OK;
  if ((which >= 3) && !P.built && (rc = poisson_lhs(c))) return rc;
  Metrics m = metrics(c);
  for (int r = 0; r < reps; r++) {
    switch (which) {
      case 0: extern void launch_face_flux(Ctx *); launch_face_flux(c); break;
      case 1: extern void launch_fp(Ctx *); launch_fp(c); break;
      case 2: extern void launch_rhs(Ctx *); launch_rhs(c); break;
      case 3:
        k_apply64<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, P.coef, P.fluid, c->f[VFS_PHI][0], P.t);
        break;
      case 4: {
        float *w = P.f32;
        const long long cols = (long long)(g.mx - 2) * (g.mz - 2);
        k_yline_fine<float><<<nblocks(cols, 128), 128, 0, c->stream>>>(g, P.coef32, P.fluid, w, w + g.N, w + 2 * g.N,
                                                                      w + 4 * g.N, w + 5 * g.N, 0.8f, 0);
        break;
      }
      case 5: {
        double *w = P.f64;
        const long long cols = (long long)(g.mx - 2) * (g.mz - 2);
        k_yline_fine<double><<<nblocks(cols, 128), 128, 0, c->stream>>>(g, P.coef, P.fluid, w, w + g.N, w + 2 * g.N,
                                                                       w + 4 * g.N, w + 5 * g.N, 0.8, 0);
        break;
      }
      case 6:
        k_projection<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, c->f[VFS_PHI][0], field3(c, VFS_UCONT));
        break;
      default: return set_err(c, VFS_ERR_INVALID, "run_kernel: unknown kernel id");
    }
    if ((rc = check_launch(c, "run_kernel"))) return rc;
  }
  return VFS_OK;
}
}  // namespace vfs

extern "C" int vfs_run_kernel(vfs_ctx *ctx, int which, int reps) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || reps < 0) return vfs::set_err(c, VFS_ERR_INVALID, "vfs_run_kernel: bad argument");
  cudaSetDevice(c->device);
  return vfs::run_kernel(c, which, reps);
}

extern "C" int vfs_get_stream(vfs_ctx *ctx, void **stream) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !stream) return vfs::set_err(c, VFS_ERR_INVALID, "vfs_get_stream: bad argument");
  *stream = (void *)c->stream;
  return VFS_OK;
}
