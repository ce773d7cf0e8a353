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
                               uint8_t *fluid) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const long long N = g.N;
  const bool interior = !(i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1);
  if (!interior || nv[p] != 0) {
    for (int s = 0; s < NSLOT; s++) coef[s * N + p] = 0;
    fluid[p] = 0;
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
  // inserted value.
  for (int s = 0; s < NSLOT; s++) coef[s * N + p] = set[s] ? S.vol[s] : 0.0;
  fluid[p] = 1;
}

// Neighbour index of slot s for an unknown (valid only where the coefficient is non-zero;
// the index is always inside the array).
__device__ __forceinline__ long long nb_index(const Grid &g, int i, int j, int k, int s) {
  return lidx(g, wrapi(g, i + c_off[s][0]), wrapj(g, j + c_off[s][1]), wrapk(g, k + c_off[s][2]));
}

// (A x)[p] on the grid layout from the first NS stencil slots: NS = 7 when every cross
// slot of the operator is zero (orthogonal grids), else 19.  A skipped slot is zero, so
// both forms give the same sums.  Rows of non-unknowns are all zero.
template <int NS>
__device__ __forceinline__ double apply_row64(const Grid &g, const double *__restrict__ coef,
                                              const double *__restrict__ x, long long p) {
  // 32-bit index arithmetic (grids below 2^31 points)
  const unsigned up = (unsigned)p, umx = (unsigned)g.mx, umy = (unsigned)g.my;
  const unsigned q = up / umx;
  const int i = (int)(up - q * umx);
  const unsigned kk = q / umy;
  const int j = (int)(q - kk * umy), k = (int)kk;
  double s = 0;
#pragma unroll
  for (int t = 0; t < NS; t++) {
    const double c = coef[t * g.N + p];
    if (c != 0.0) s += c * x[nb_index(g, i, j, k, t)];
  }
  return s;
}

// y = A x on the grid layout (FP64).
template <int NS>
__global__ void k_apply(Grid g, const double *__restrict__ coef, const double *__restrict__ x,
                        double *__restrict__ y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  y[p] = apply_row64<NS>(g, coef, x, p);
}

// y = A^T x: every stencil entry of row p scattered onto its neighbour (atomics).
__global__ void k_apply_t(Grid g, int ns, const double *__restrict__ coef, const double *__restrict__ x, double *y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const double xp = x[p];
  if (xp == 0.0) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  for (int t = 0; t < ns; t++) {
    const double c = coef[t * g.N + p];
    if (c != 0.0) atomicAdd(y + nb_index(g, i, j, k, t), c * xp);
  }
}

int poisson_set_transpose(Ctx *c, bool on) {
  c->ps.transpose = on;
  return VFS_OK;
}

int poisson_apply_dev(Ctx *c, const double *x, double *y) {
  if (c->ps.transpose) {
    cudaMemsetAsync(y, 0, sizeof(double) * c->g.N, c->stream);
    c->launches++, k_apply_t<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->ps.nslot, c->ps.coef, x, y);
    return check_launch(c, "k_apply_t");
  }
  if (c->ps.nslot == 7) c->launches++, k_apply<7><<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->ps.coef, x, y);
  else c->launches++, k_apply<NSLOT><<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->ps.coef, x, y);
  return check_launch(c, "k_apply");
}

// ------------------------------------------------------------------ Krylov kernels
// The FGMRES vectors are exactly zero off the unknowns, so every dot product runs over
// the whole grid layout.  Reductions are deterministic: per-thread sums in a fixed order,
// warp shuffles, a fixed-order sum over warps, then k_sum_rows over the block partials.
#ifndef VFS_KRY_BLOCKS_PER_SM
#define VFS_KRY_BLOCKS_PER_SM 4
#endif
// Two resident blocks per SM cap the basis kernels at 128 registers (their 32-vector
// branch spills; the common ones fit): the step went from 35.6 to 34.5 ms against one
// block per SM at 250 registers (256 x 192 x 256, mixed, graph form).
#ifndef VFS_KRY_MINB
#define VFS_KRY_MINB 2
#endif
static const int kKryBlocks = 148 * VFS_KRY_BLOCKS_PER_SM;
// Blocks of the basis passes: a fixed multiple of the SM count, grid-stride (one point
// pair per thread over the whole vector measured 7 % slower per step on the B200).
static const int kKryThreads = 256;
static int kry_grid(const Ctx *c) {
  (void)c;
  return kKryBlocks;
}

// Block sums of rows 0..nv-1 and of row NV (stored as row nv) of acc into
// parts[row * gridDim.x + blockIdx.x].
template <int NV>
__device__ __forceinline__ void block_sums(const double (&acc)[NV + 1], int nv, double *__restrict__ parts) {
  __shared__ double sh[NV + 1][kKryThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t <= NV; t++) {
    double v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[t][warp] = v;
  }
  __syncthreads();
  for (int t = threadIdx.x; t <= NV; t += blockDim.x) {
    if (t < nv || t == NV) {
      double s = 0;
      for (int w = 0; w < kKryThreads / 32; w++) s += sh[t][w];
      parts[(long long)(t == NV ? nv : t) * gridDim.x + blockIdx.x] = s;
    }
  }
}

// The Krylov kernels below stream the basis two points at a time (16-byte loads): the
// basis vectors are stored ldv apart, ldv a multiple of 32, and every other vector is a
// separate allocation, so pair loads are aligned; an odd last point is done alone.

static const int kRedBlocks = 148 * 2;
// Number of non-zero cross-derivative slots (7..18) of the operator.
__global__ void k_count_cross(long long N, const double *__restrict__ coef, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += stride)
    for (int t = NE; t < NSLOT; t++) s += coef[t * N + p] != 0.0 ? 1.0 : 0.0;
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
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

int poisson_lhs(Ctx *c) {
  Poisson &P = c->ps;
  const Grid &g = c->g;
  const long long N = g.N;
  int rc;
  if (!P.coef) {
    bool ok = cudaMalloc(&P.coef, sizeof(double) * NSLOT * N) == cudaSuccess;
    ok &= cudaMalloc(&P.fluid, N) == cudaSuccess;
    ok &= cudaMalloc(&P.w, sizeof(double) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.r, sizeof(double) * N) == cudaSuccess;
    ok &= cudaMalloc(&P.t, sizeof(double) * N) == cudaSuccess;
    if (!ok) return set_err(c, VFS_ERR_CUDA, "poisson_lhs: allocation failed");
    cudaMemsetAsync(P.w, 0, sizeof(double) * N, c->stream);
    cudaMemsetAsync(P.r, 0, sizeof(double) * N, c->stream);
    cudaMemsetAsync(P.t, 0, sizeof(double) * N, c->stream);
  }
  c->launches++, k_poisson_coef<<<nblocks(N, 128), 128, 0, c->stream>>>(g, metrics(c), c->nv, P.coef, P.fluid);
  if ((rc = check_launch(c, "k_poisson_coef"))) return rc;
  // fluid-cell count and sum of aj (Remove_Nullspace / Remove_Nullspace_Scale)
  if ((rc = ensure_red(c, 2 * kRedBlocks + 64))) return rc;
  c->launches++, k_count_fluid<<<kRedBlocks, 256, 0, c->stream>>>(N, P.fluid, c->f[VFS_AJ][0], c->red);
  if ((rc = check_launch(c, "k_count_fluid"))) return rc;
  double cnt = 0, saj = 0;
  if ((rc = reduce_sum(c, c->red, kRedBlocks, &cnt))) return rc;
  if ((rc = reduce_sum(c, c->red + kRedBlocks, kRedBlocks, &saj))) return rc;
  P.nfluid = (long long)llround(cnt);
  P.sum_aj = saj;
  // the apply reads only slots CP..BP when no row has a cross-derivative entry
  c->launches++, k_count_cross<<<kRedBlocks, 256, 0, c->stream>>>(N, P.coef, c->red);
  if ((rc = check_launch(c, "k_count_cross"))) return rc;
  double ncross = 0;
  if ((rc = reduce_sum(c, c->red, kRedBlocks, &ncross))) return rc;
  P.nslot = ncross == 0 ? 7 : NSLOT;
  if ((rc = mg_setup(c))) return rc;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "poisson_lhs failed");
  P.built = true;
  P.guess = false;  // a fresh Phi2 with the unknown numbering (poisson.c:280-282)
  c->setup_epoch++;
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
  int i, j, k;
  dijk(g, p, i, j, k);
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

// b += -sum(b) * aj / sum(aj) on fluid cells (Remove_Nullspace_Scale, poisson_hypre.c:110),
// sum(b) from the device scalars.
__global__ void k_shift_scaled(long long n, const uint8_t *fluid, const double *aj, const double *__restrict__ ds,
                               double sum_aj, double *b) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n || !fluid[p]) return;
  const double sum = ds[DS_BSUM];
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
  __shared__ double sh[8];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = (p < n && fluid[p]) ? a[p] : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < 8; w++) t += sh[w];
    parts[blockIdx.x] = t;
  }
}

// VolumeFlux(user, Ucont, ...) (poisson.c:3306-3500) without sharp-interface IB nodes
// (immersed = 0): the flux through every interior face between a fluid cell and a
// non-fluid cell is set to zero.  The face index is the lower cell of the pair, as in
// the reference loops over interior cells (i <= mx-2 always holds there).
__global__ void k_volume_flux_blocked(Grid g, const uint8_t *__restrict__ nv, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
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
  if (c->g.immersed) {  // poisson_hypre.c:564
    int rc;
    if (c->tape && (rc = tape_vflux(c))) return rc;
    return volume_flux_ibm(c, nullptr, nullptr);
  }
  c->launches++, k_volume_flux_blocked<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->nv, field3(c, VFS_UCONT));
  return check_launch(c, "k_volume_flux_blocked");
}

// The local part of the right-hand side: periodic Ucont ghosts, then b = div(Ucont)/dt*st.
int poisson_rhs_local(Ctx *c) {
  int rc;
  if ((rc = periodic_copy3(c, field3(c, VFS_UCONT)))) return rc;
  c->launches++, k_poisson_rhs<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_UCONT)), c->ps.fluid,
                                                             c->f[VFS_B][0]);
  return check_launch(c, "k_poisson_rhs");
}

int poisson_rhs(Ctx *c) {
  int rc;
  double *b = c->f[VFS_B][0];
  if ((rc = poisson_rhs_local(c))) return rc;
  const int nb = (int)nblocks(c->g.N, 256);
  if ((rc = ensure_red(c, nb + 64))) return rc;
  c->launches++, k_sum_fluid<<<nb, 256, 0, c->stream>>>(c->g.N, c->ps.fluid, b, c->red);
  if ((rc = check_launch(c, "k_sum_fluid"))) return rc;
  if ((rc = reduce_to(c, c->red, nb, c->ds + DS_BSUM))) return rc;
  c->launches++, k_shift_scaled<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, c->ps.fluid, c->f[VFS_AJ][0], c->ds,
                                                             c->ps.sum_aj, b);
  return check_launch(c, "k_shift_scaled");
}

// ------------------------------------------------------------------ FGMRES
// x = x on the unknowns, 0 elsewhere (the periodic ghost copies), with the block sums of
// <b, b> in parts[blockIdx.x].
__global__ void __launch_bounds__(256) k_guess(long long n, const uint8_t *__restrict__ fluid,
                                               const double *__restrict__ b, double *__restrict__ x,
                                               double *__restrict__ parts) {
  __shared__ double sh[8];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double v2 = 0;
  if (p < n) {
    if (!fluid[p]) x[p] = 0.0;
    v2 = b[p] * b[p];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v2 += __shfl_down_sync(0xffffffffu, v2, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < 8; w++) s += sh[w];
    parts[blockIdx.x] = s;
  }
}

// ------------------------------------------------------------------ device-driven FGMRES
// The same FGMRES as a sequence of kernels that read the iteration state from the device
// (KryDev): the Gram-Schmidt decisions, the Hessenberg matrix, the Givens rotations and the
// convergence tests run in one-thread kernels, and every kernel that depends on a
// decision reads its flag (Guard) and returns at once when it does not apply.  Launched
// from a host loop that reads the two loop flags, or captured into a graph whose two
// loops are conditional WHILE nodes that the control kernels set, with the same kernels
// and therefore the same results.

// Run when (*flag != 0) == want; without a flag always.
struct Guard {
  const int *flag;
  int want;
};
__device__ __forceinline__ bool guard_off(const Guard &q) { return q.flag && ((*q.flag != 0) != (q.want != 0)); }
static Guard always() { return Guard{nullptr, 0}; }

// base + (*j + off) * ldv (base when j is null).
template <typename B>
struct DynPtrT {
  B *base;
  long long ldv;
  const int *j;
  int off;
  __device__ __forceinline__ B *get() const { return j ? base + (long long)(*j + off) * ldv : base; }
};
using DynPtr = DynPtrT<double>;

// Two consecutive basis entries as FP64 (the FP32 basis of precision 2 is widened on load
// and rounded on store; every sum and product is FP64).
__device__ __forceinline__ double2 ld2(const double *__restrict__ p, long long i) {
  return reinterpret_cast<const double2 *>(p)[i];
}
__device__ __forceinline__ double2 ld2(const float *__restrict__ p, long long i) {
  const float2 f = reinterpret_cast<const float2 *>(p)[i];
  return make_double2((double)f.x, (double)f.y);
}
__device__ __forceinline__ void st2(double *__restrict__ p, long long i, double2 v) {
  reinterpret_cast<double2 *>(p)[i] = v;
}
__device__ __forceinline__ void st2(float *__restrict__ p, long long i, double2 v) {
  reinterpret_cast<float2 *>(p)[i] = make_float2((float)v.x, (float)v.y);
}

// Sets a graph conditional from the device (only in a captured solve).
__device__ __forceinline__ void set_cond(unsigned long long h, int use, int v) {
  if (use) cudaGraphSetConditional((cudaGraphConditionalHandle)h, v ? 1u : 0u);
}

template <int NS>
__global__ void k_apply_dyn(Grid g, const double *__restrict__ coef, DynPtr x, double *__restrict__ y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  y[p] = apply_row64<NS>(g, coef, x.get(), p);
}
// The inner operator of precision 2: FP32 vectors, the FP64 coefficients, FP64 products and
// sum, the result rounded to FP32 (FP32 coefficients measured 20-40 % more iterations:
// iterative refinement converges at the rate of the inner operator's error).
template <int NS>
__global__ void k_apply32_dyn(Grid g, const double *__restrict__ coef, DynPtrT<float> xp, float *__restrict__ y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const float *__restrict__ x = xp.get();
  const unsigned up = (unsigned)p, umx = (unsigned)g.mx, umy = (unsigned)g.my;
  const unsigned q = up / umx;
  const int i = (int)(up - q * umx);
  const unsigned kk = q / umy;
  const int j = (int)(q - kk * umy), k = (int)kk;
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < NS; t++) {
    const double c = coef[t * g.N + p];
    if (c != 0.0) s += c * (double)x[nb_index(g, i, j, k, t)];
  }
  y[p] = (float)s;
}
__global__ void k_apply_t_dyn(Grid g, int ns, const double *__restrict__ coef, DynPtr x, double *y, Guard q) {
  if (guard_off(q)) return;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const double xp = x.get()[p];
  if (xp == 0.0) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  for (int t = 0; t < ns; t++) {
    const double c = coef[t * g.N + p];
    if (c != 0.0) atomicAdd(y + nb_index(g, i, j, k, t), c * xp);
  }
}
__global__ void k_zero_g(long long n, double *y, Guard q) {
  if (guard_off(q)) return;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) y[p] = 0.0;
}

// <V_t, w> (t < nv) and <w, w> with nv = j + 1 from the device state (B: the basis type,
// FP64, or FP32 for precision 2; the sums are FP64).
template <int NV, typename B>
__device__ __forceinline__ void multidot_body(long long N, long long ldv, const B *__restrict__ V, int nv,
                                              const B *__restrict__ w, double *__restrict__ parts) {
  double acc[NV + 1];
#pragma unroll
  for (int t = 0; t <= NV; t++) acc[t] = 0;
  const long long N2 = N >> 1, stride = (long long)gridDim.x * blockDim.x;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long p2 = tid; p2 < N2; p2 += stride) {
    const double2 wp = ld2(w, p2);
#pragma unroll
    for (int t = 0; t < NV; t++) {
      if (t < nv) {
        const double2 v = ld2(V + t * ldv, p2);
        acc[t] += v.x * wp.x + v.y * wp.y;
      }
    }
    acc[NV] += wp.x * wp.x + wp.y * wp.y;
  }
  if ((N & 1) && tid == 0) {
    const long long p = N - 1;
    const double wp = (double)w[p];
#pragma unroll
    for (int t = 0; t < NV; t++)
      if (t < nv) acc[t] += (double)V[t * ldv + p] * wp;
    acc[NV] += wp * wp;
  }
  block_sums<NV>(acc, nv, parts);
}
template <typename B>
__global__ void __launch_bounds__(kKryThreads, VFS_KRY_MINB) k_multidot_dyn(long long N, long long ldv,
                                                                             const B *__restrict__ V,
                                                                             const KryDev *__restrict__ kd,
                                                                             const B *__restrict__ w,
                                                                             double *__restrict__ parts) {
  const int nv = kd->j + 1;
  if (nv <= 4) multidot_body<4>(N, ldv, V, nv, w, parts);
  else if (nv <= 8) multidot_body<8>(N, ldv, V, nv, w, parts);
  else if (nv <= 16) multidot_body<16>(N, ldv, V, nv, w, parts);
  else multidot_body<32>(N, ldv, V, nv, w, parts);
}

// w -= sum_t h_t V_t (h = kd->hdev), with <V_t, w> and <w, w> of the result.
template <int NV, typename B>
__device__ __forceinline__ void update_dots_body(long long N, long long ldv, const B *__restrict__ V, int nv,
                                                 const double *__restrict__ h, B *__restrict__ w,
                                                 double *__restrict__ parts) {
  double hr[NV], acc[NV + 1];
#pragma unroll
  for (int t = 0; t < NV; t++) hr[t] = t < nv ? h[t] : 0.0;
#pragma unroll
  for (int t = 0; t <= NV; t++) acc[t] = 0;
  const long long N2 = N >> 1, stride = (long long)gridDim.x * blockDim.x;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long p2 = tid; p2 < N2; p2 += stride) {
    double2 v[NV];
#pragma unroll
    for (int t = 0; t < NV; t++) v[t] = t < nv ? ld2(V + t * ldv, p2) : make_double2(0.0, 0.0);
    double2 s = ld2(w, p2);
#pragma unroll
    for (int t = 0; t < NV; t++) { s.x -= hr[t] * v[t].x; s.y -= hr[t] * v[t].y; }
    st2(w, p2, s);
    if (sizeof(B) == 4) s = ld2(w, p2);  // the stored (rounded) values enter the dots
#pragma unroll
    for (int t = 0; t < NV; t++) acc[t] += v[t].x * s.x + v[t].y * s.y;
    acc[NV] += s.x * s.x + s.y * s.y;
  }
  if ((N & 1) && tid == 0) {
    const long long p = N - 1;
    double s = (double)w[p];
#pragma unroll
    for (int t = 0; t < NV; t++)
      if (t < nv) s -= hr[t] * (double)V[t * ldv + p];
    w[p] = (B)s;
    s = (double)w[p];
#pragma unroll
    for (int t = 0; t < NV; t++)
      if (t < nv) acc[t] += (double)V[t * ldv + p] * s;
    acc[NV] += s * s;
  }
  block_sums<NV>(acc, nv, parts);
}
template <typename B>
__global__ void __launch_bounds__(kKryThreads, VFS_KRY_MINB) k_update_dots_dyn(long long N, long long ldv,
                                                                                const B *__restrict__ V,
                                                                                const KryDev *__restrict__ kd,
                                                                                B *__restrict__ w,
                                                                                double *__restrict__ parts, Guard q) {
  if (guard_off(q)) return;
  const int nv = kd->j + 1;
  if (nv <= 4) update_dots_body<4>(N, ldv, V, nv, kd->hdev, w, parts);
  else if (nv <= 8) update_dots_body<8>(N, ldv, V, nv, kd->hdev, w, parts);
  else if (nv <= 16) update_dots_body<16>(N, ldv, V, nv, kd->hdev, w, parts);
  else update_dots_body<32>(N, ldv, V, nv, kd->hdev, w, parts);
}

// out = (w - sum_t h_t V_t) * scale (h = kd->hdev, scale = kd->scale).
template <int NV, typename B>
__device__ __forceinline__ void update_scale_body(long long N, long long ldv, const B *__restrict__ V, int nv,
                                                  const double *__restrict__ h, const B *__restrict__ w,
                                                  double scale, B *__restrict__ out) {
  double hr[NV];
#pragma unroll
  for (int t = 0; t < NV; t++) hr[t] = t < nv ? h[t] : 0.0;
  const long long N2 = N >> 1, stride = (long long)gridDim.x * blockDim.x;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long p2 = tid; p2 < N2; p2 += stride) {
    double2 v[NV];
#pragma unroll
    for (int t = 0; t < NV; t++) v[t] = t < nv ? ld2(V + t * ldv, p2) : make_double2(0.0, 0.0);
    double2 s = ld2(w, p2);
#pragma unroll
    for (int t = 0; t < NV; t++) { s.x -= hr[t] * v[t].x; s.y -= hr[t] * v[t].y; }
    s.x *= scale; s.y *= scale;
    st2(out, p2, s);
  }
  if ((N & 1) && tid == 0) {
    const long long p = N - 1;
    double s = (double)w[p];
#pragma unroll
    for (int t = 0; t < NV; t++)
      if (t < nv) s -= hr[t] * (double)V[t * ldv + p];
    out[p] = (B)(s * scale);
  }
}
template <typename B>
__global__ void __launch_bounds__(kKryThreads, VFS_KRY_MINB) k_update_scale_dyn(long long N, long long ldv,
                                                                                 const B *__restrict__ V,
                                                                                 const KryDev *__restrict__ kd,
                                                                                 const B *__restrict__ w,
                                                                                 DynPtrT<B> out, Guard q) {
  if (guard_off(q)) return;
  const int nv = kd->j + 1;
  B *o = out.get();
  if (nv <= 4) update_scale_body<4>(N, ldv, V, nv, kd->hdev, w, kd->scale, o);
  else if (nv <= 8) update_scale_body<8>(N, ldv, V, nv, kd->hdev, w, kd->scale, o);
  else if (nv <= 16) update_scale_body<16>(N, ldv, V, nv, kd->hdev, w, kd->scale, o);
  else update_scale_body<32>(N, ldv, V, nv, kd->hdev, w, kd->scale, o);
}

// Rows 0..nrows-1 of the block partials summed in a fixed order; nrows = j + 2 (the nv
// dot products and the norm) from the device state.
__global__ void k_sum_rows_dyn(const double *parts, const KryDev *kd, int ncols, double *out, Guard q) {
  if (guard_off(q)) return;
  const int r = blockIdx.x;
  if (r >= kd->j + 2) return;
  __shared__ double sh[256];
  double s = 0;
  for (int t = threadIdx.x; t < ncols; t += blockDim.x) s += parts[(long long)r * ncols + t];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[r] = sh[0];
}

// Sum of n partials (one block, fixed order, as k_sum_parts) into out, guarded.
__global__ void __launch_bounds__(1024) k_sum_parts_g(const double *parts, int n, double *out, Guard q) {
  if (guard_off(q)) return;
  __shared__ double sh[32];
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int t = threadIdx.x;
  for (; t + 7 * 1024 < n; t += 8 * 1024) {
#pragma unroll
    for (int u = 0; u < 8; u++) s[u] += parts[t + u * 1024];
  }
  for (; t < n; t += 1024) s[0] += parts[t];
  double v = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = sh[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) out[0] = v;
  }
}

// r = b - A x with the block sums of <r, r>, guarded.
template <int NS>
__global__ void __launch_bounds__(256) k_residual_g(Grid g, const double *__restrict__ coef,
                                                    const double *__restrict__ b, const double *__restrict__ x,
                                                    double *__restrict__ r, double *__restrict__ parts, Guard q) {
  if (guard_off(q)) return;
  __shared__ double sh[8];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double v2 = 0;
  if (p < g.N) {
    const double v = b[p] - apply_row64<NS>(g, coef, x, p);
    r[p] = v;
    v2 = v * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v2 += __shfl_down_sync(0xffffffffu, v2, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < 8; w++) s += sh[w];
    parts[blockIdx.x] = s;
  }
}
// r = b - r (r holding A x) and the partial sums of <r, r>, guarded (grid-stride).
__global__ void k_sub_norm_g(long long n, const double *__restrict__ b, double *r, double *parts, Guard q) {
  if (guard_off(q)) return;
  __shared__ double sh[256];
  double s = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const double v = b[p] - r[p];
    r[p] = v;
    s += v * v;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// dst = src * (*scale), guarded (FP64 arithmetic, stored in dst's type).
template <typename S, typename D>
__global__ void k_scale_copy_dyn(long long n, const S *__restrict__ src, const double *__restrict__ scale,
                                 DynPtrT<D> dst, Guard q) {
  if (guard_off(q)) return;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) dst.get()[p] = (D)((double)src[p] * (*scale));
}
// x += sum_t y_t Z_t for t < kd->jdone (y = kd->y); x is FP64 whatever Z's type.
template <typename B>
__global__ void k_lincomb_add_dyn(long long n, long long ldv, const B *__restrict__ Z,
                                  const KryDev *__restrict__ kd, double *__restrict__ x) {
  const int m = kd->jdone;
  if (m <= 0) return;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double s = x[p];
  for (int t = 0; t < m; t++) s += kd->y[t] * (double)Z[(long long)t * ldv + p];
  x[p] = s;
}
// x += -sum / nfluid on the fluid cells (sum = ds[DS_PHISUM]).
__global__ void k_shift_mean(long long n, const uint8_t *fluid, const double *__restrict__ ds, double nfluid,
                             double *x) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n || !fluid[p]) return;
  const double val = -ds[DS_PHISUM] / nfluid;
  x[p] += val;
}

// ---- control kernels (one thread)
// After the initial residual (kd->rr) and, with a starting guess, <b, b> (kd->bb).
__global__ void k_kry_init(KryDev *kd, double rtol, double atol, int warm, int maxit, int m, unsigned long long h_outer,
                           int use_graph, double inner_rtol) {
  kd->inner_rtol = inner_rtol;
  kd->rnorm = sqrt(kd->rr);
  kd->bnorm = warm ? sqrt(kd->bb) : kd->rnorm;
  kd->r0 = kd->rnorm;
  kd->tol = fmax(rtol * kd->bnorm, atol);
  kd->it = 0;
  kd->cycles = 0;
  kd->maxit = maxit;
  kd->m = m;
  kd->conv = kd->bnorm <= kd->tol;
  kd->fresh = 1;
  kd->jdone = 0;
  kd->outer_go = !kd->conv && kd->it < maxit;
  set_cond(h_outer, use_graph, kd->outer_go);
}
// Start of a restart cycle (kd->rr holds <r, r> of a new residual unless kd->fresh).
__global__ void k_kry_cycle(KryDev *kd, unsigned long long h_inner, int use_graph) {
  kd->cycles++;
  if (!kd->fresh) kd->rnorm = sqrt(kd->rr);
  kd->fresh = 0;
  const double beta = kd->rnorm;
  kd->beta = beta;
  kd->j = 0;
  kd->jdone = 0;
  kd->check = 0;
  if (beta <= kd->tol) {
    kd->conv = 1;
    kd->inner_go = 0;
    kd->scale = 0;
  } else {
    kd->scale = 1.0 / beta;
    for (int t = 0; t <= kd->m; t++) kd->gv[t] = 0.0;
    kd->gv[0] = beta;
    kd->inner_go = kd->it < kd->maxit;
  }
  set_cond(h_inner, use_graph, kd->inner_go);
}
// After h = V^T w and h[nv] = <w, w>: one Gram-Schmidt pass, or re-orthogonalise.
__global__ void k_kry_ctl_a(KryDev *kd) {
  const int j = kd->j, nv = j + 1, m = kd->m;
  double proj0 = 0;
  for (int t = 0; t < nv; t++) proj0 += kd->h[t] * kd->h[t];
  const double hn2_0 = kd->h[nv] - proj0;  // |w - V h|^2 for orthonormal V
  for (int t = 0; t < nv; t++) kd->hdev[t] = kd->h[t];
  kd->degen = 0;
  if (hn2_0 > 0.5 * kd->h[nv]) {
    for (int t = 0; t < nv; t++) kd->H[t * m + j] = kd->h[t];
    kd->hn = sqrt(hn2_0);
    kd->scale = 1.0 / kd->hn;
    kd->reorth = 0;
  } else {
    kd->reorth = 1;
  }
}
// After w -= V h and h2 = V^T w: the second pass.
__global__ void k_kry_ctl_b(KryDev *kd) {
  if (!kd->reorth) return;
  const int j = kd->j, nv = j + 1, m = kd->m;
  const double ww = kd->h2[nv];
  double proj = 0;
  for (int t = 0; t < nv; t++) proj += kd->h2[t] * kd->h2[t];
  const double hn2 = ww - proj;  // |w - V h2|^2 for orthonormal V
  for (int t = 0; t < nv; t++) {
    kd->hdev[t] = kd->h2[t];
    kd->H[t * m + j] = kd->h[t] + kd->h2[t];
  }
  if (hn2 > 1e-4 * ww) {
    kd->hn = sqrt(hn2);
    kd->scale = 1.0 / kd->hn;
    kd->degen = 0;
  } else {
    kd->degen = 1;  // w nearly in span(V): form w - V h2 and take its norm
  }
}
// After the explicit w -= V h2 (degenerate case).
__global__ void k_kry_ctl_c(KryDev *kd) {
  if (!kd->degen) return;
  const int nv = kd->j + 1;
  kd->hn = sqrt(fmax(kd->h3[nv], 0.0));
  kd->scale = kd->hn > 0 ? 1.0 / kd->hn : 0.0;
}
// Hessenberg column j: Givens rotations, residual estimate, loop control.
__global__ void k_kry_givens(KryDev *kd, unsigned long long h_inner, int use_graph) {
  const int j = kd->j, m = kd->m;
  double *H = kd->H;
  H[(j + 1) * m + j] = kd->hn;
  for (int t = 0; t < j; t++) {
    const double a = H[t * m + j], bb = H[(t + 1) * m + j];
    H[t * m + j] = kd->cs[t] * a + kd->sn[t] * bb;
    H[(t + 1) * m + j] = -kd->sn[t] * a + kd->cs[t] * bb;
  }
  const double a = H[j * m + j], bb = H[(j + 1) * m + j];
  const double den = sqrt(a * a + bb * bb);
  kd->cs[j] = den > 0 ? a / den : 1.0;
  kd->sn[j] = den > 0 ? bb / den : 0.0;
  H[j * m + j] = den;
  H[(j + 1) * m + j] = 0;
  kd->gv[j + 1] = -kd->sn[j] * kd->gv[j];
  kd->gv[j] = kd->cs[j] * kd->gv[j];
  kd->it++;
  kd->jdone = j + 1;
  kd->rnorm = fabs(kd->gv[j + 1]);
  // precision 2 also ends the cycle (an iterative-refinement sweep) once the FP32 Arnoldi
  // estimate has fallen by inner_rtol; the next cycle restarts from the FP64 residual
  const bool stop = kd->rnorm <= kd->tol || kd->hn == 0 || kd->rnorm <= kd->inner_rtol * kd->beta;
  kd->j = j + 1;
  kd->inner_go = !stop && kd->j < m && kd->it < kd->maxit;
  set_cond(h_inner, use_graph, kd->inner_go);
}
// Back substitution (y into hdev for the update) and the test for the true residual.
__global__ void k_kry_backsub(KryDev *kd) {
  const int jd = kd->jdone, m = kd->m;
  for (int t = jd - 1; t >= 0; t--) {
    double sum = kd->gv[t];
    for (int u = t + 1; u < jd; u++) sum -= kd->H[t * m + u] * kd->y[u];
    kd->y[t] = sum / kd->H[t * m + t];
  }
  kd->check = (jd > 0 && kd->rnorm <= kd->tol) ? 1 : 0;
}
// After the confirming residual (when kd->check): convergence and the outer loop.
__global__ void k_kry_confirm(KryDev *kd, unsigned long long h_outer, int use_graph) {
  if (kd->check) {
    kd->rnorm = sqrt(kd->rr);
    kd->fresh = 1;
    kd->conv = kd->rnorm <= kd->tol * 1.0000001 || kd->rnorm <= 2 * kd->tol;
  }
  kd->outer_go = !kd->conv && kd->it < kd->maxit;
  set_cond(h_outer, use_graph, kd->outer_go);
}

// ---- host side
static DynPtr dyn(double *base, long long ldv, const int *j, int off) { return DynPtr{base, ldv, j, off}; }

// r = b - A x and <r, r> into *rr, under guard q.
static int residual_dev(Ctx *c, const double *b, double *x, double *r, double *rr, Guard q) {
  Poisson &P = c->ps;
  const long long N = c->g.N;
  int rc;
  if (P.transpose) {
    c->launches++, k_zero_g<<<nblocks(N, 256), 256, 0, c->stream>>>(N, r, q);
    c->launches++, k_apply_t_dyn<<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.nslot, P.coef, dyn(x, 0, nullptr, 0), r, q);
    c->launches++, k_sub_norm_g<<<kKryBlocks, 256, 0, c->stream>>>(N, b, r, c->red, q);
    if ((rc = check_launch(c, "residual (transposed)"))) return rc;
    c->launches++, k_sum_parts_g<<<1, 1024, 0, c->stream>>>(c->red, kKryBlocks, rr, q);
    return check_launch(c, "k_sum_parts_g");
  }
  const int nb = (int)nblocks(N, 256);
  if (P.nslot == 7)
    c->launches++, k_residual_g<7><<<nb, 256, 0, c->stream>>>(c->g, P.coef, b, x, r, c->red, q);
  else
    c->launches++, k_residual_g<NSLOT><<<nb, 256, 0, c->stream>>>(c->g, P.coef, b, x, r, c->red, q);
  if ((rc = check_launch(c, "k_residual_g"))) return rc;
  c->launches++, k_sum_parts_g<<<1, 1024, 0, c->stream>>>(c->red, nb, rr, q);
  return check_launch(c, "k_sum_parts_g");
}

// w = A z_j (z_j = Z + j ldv with j from the device state).
static int apply_dyn(Ctx *c, double *Z, double *w) {
  Poisson &P = c->ps;
  const long long N = c->g.N;
  KryDev *kd = c->kd;
  if (P.transpose) {
    c->launches++, k_zero_g<<<nblocks(N, 256), 256, 0, c->stream>>>(N, w, always());
    c->launches++, k_apply_t_dyn<<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.nslot, P.coef,
                                                                          dyn(Z, P.ldv, &kd->j, 0), w, always());
    return check_launch(c, "k_apply_t_dyn");
  }
  if (P.nslot == 7)
    c->launches++, k_apply_dyn<7><<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.coef, dyn(Z, P.ldv, &kd->j, 0), w);
  else
    c->launches++, k_apply_dyn<NSLOT><<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.coef, dyn(Z, P.ldv, &kd->j, 0), w);
  return check_launch(c, "k_apply_dyn");
}
static int apply32_dyn(Ctx *c, float *Z, float *w) {
  Poisson &P = c->ps;
  const long long N = c->g.N;
  const DynPtrT<float> z{Z, P.ldv, &c->kd->j, 0};
  if (P.nslot == 7)
    c->launches++, k_apply32_dyn<7><<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.coef, z, w);
  else
    c->launches++, k_apply32_dyn<NSLOT><<<nblocks(N, 256), 256, 0, c->stream>>>(c->g, P.coef, z, w);
  return check_launch(c, "k_apply32_dyn");
}

// One Arnoldi step of the device-driven FGMRES (body of the inner loop), on the basis of
// type B (FP64; FP32 for precision 2, whose preconditioner and operator apply are FP32).
template <typename B>
static int kry_body_t(Ctx *c, const vfs_solve_opts &o, unsigned long long h_inner, int use_graph, B *V, B *Z, B *w) {
  Poisson &P = c->ps;
  KryDev *kd = c->kd;
  const long long N = c->g.N;
  const int kg = kry_grid(c);
  int rc;
  if (sizeof(B) == 4) {
    if ((rc = mg_precondition_dyn32(c, (const float *)V, (float *)Z, P.ldv, &kd->j, o))) return rc;  // z_j = M^-1 v_j
    if ((rc = apply32_dyn(c, (float *)Z, (float *)w))) return rc;                                     // w = A z_j
  } else {
    if ((rc = mg_precondition_dyn(c, (const double *)V, (double *)Z, P.ldv, &kd->j, o))) return rc;
    if ((rc = apply_dyn(c, (double *)Z, (double *)w))) return rc;
  }
  c->launches++, k_multidot_dyn<B><<<kg, kKryThreads, 0, c->stream>>>(N, P.ldv, V, kd, w, c->red);
  c->launches++, k_sum_rows_dyn<<<kKryMax + 2, 256, 0, c->stream>>>(c->red, kd, kg, kd->h, always());
  c->launches++, k_kry_ctl_a<<<1, 1, 0, c->stream>>>(kd);
  if ((rc = check_launch(c, "FGMRES Gram-Schmidt"))) return rc;
  const Guard reorth{&kd->reorth, 1}, degen{&kd->degen, 1}, plain{&kd->degen, 0};
  c->launches++, k_update_dots_dyn<B><<<kg, kKryThreads, 0, c->stream>>>(N, P.ldv, V, kd, w, c->red, reorth);
  c->launches++, k_sum_rows_dyn<<<kKryMax + 2, 256, 0, c->stream>>>(c->red, kd, kg, kd->h2, reorth);
  c->launches++, k_kry_ctl_b<<<1, 1, 0, c->stream>>>(kd);
  c->launches++, k_update_dots_dyn<B><<<kg, kKryThreads, 0, c->stream>>>(N, P.ldv, V, kd, w, c->red, degen);
  c->launches++, k_sum_rows_dyn<<<kKryMax + 2, 256, 0, c->stream>>>(c->red, kd, kg, kd->h3, degen);
  c->launches++, k_kry_ctl_c<<<1, 1, 0, c->stream>>>(kd);
  if ((rc = check_launch(c, "FGMRES re-orthogonalisation"))) return rc;
  const DynPtrT<B> next{V, P.ldv, &kd->j, 1};
  c->launches++, k_update_scale_dyn<B><<<kg, kKryThreads, 0, c->stream>>>(N, P.ldv, V, kd, w, next, plain);
  c->launches++, k_scale_copy_dyn<B, B><<<nblocks(N, 256), 256, 0, c->stream>>>(N, w, &kd->scale, next, degen);
  c->launches++, k_kry_givens<<<1, 1, 0, c->stream>>>(kd, h_inner, use_graph);
  return check_launch(c, "FGMRES Givens");
}

static bool fp32_inner(const vfs_solve_opts &o) { return o.precision == 2; }

static int kry_body(Ctx *c, const vfs_solve_opts &o, unsigned long long h_inner, int use_graph) {
  Poisson &P = c->ps;
  return fp32_inner(o) ? kry_body_t<float>(c, o, h_inner, use_graph, P.V32, P.Z32, P.w32)
                       : kry_body_t<double>(c, o, h_inner, use_graph, P.V, P.Z, P.w);
}

static int kry_cycle_start(Ctx *c, const vfs_solve_opts &o, const double *b, double *x, unsigned long long h_inner,
                           int use_graph) {
  Poisson &P = c->ps;
  KryDev *kd = c->kd;
  const long long N = c->g.N;
  int rc;
  if ((rc = residual_dev(c, b, x, P.r, &kd->rr, Guard{&kd->fresh, 0}))) return rc;
  c->launches++, k_kry_cycle<<<1, 1, 0, c->stream>>>(kd, h_inner, use_graph);
  if (fp32_inner(o))
    c->launches++, k_scale_copy_dyn<double, float><<<nblocks(N, 256), 256, 0, c->stream>>>(
        N, P.r, &kd->scale, DynPtrT<float>{P.V32, P.ldv, nullptr, 0}, Guard{&kd->inner_go, 1});
  else
    c->launches++, k_scale_copy_dyn<double, double><<<nblocks(N, 256), 256, 0, c->stream>>>(
        N, P.r, &kd->scale, dyn(P.V, P.ldv, nullptr, 0), Guard{&kd->inner_go, 1});
  return check_launch(c, "FGMRES cycle start");
}

static int kry_cycle_end(Ctx *c, const vfs_solve_opts &o, const double *b, double *x, unsigned long long h_outer,
                         int use_graph) {
  Poisson &P = c->ps;
  KryDev *kd = c->kd;
  const long long N = c->g.N;
  int rc;
  c->launches++, k_kry_backsub<<<1, 1, 0, c->stream>>>(kd);
  if (fp32_inner(o))
    c->launches++, k_lincomb_add_dyn<float><<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.ldv, P.Z32, kd, x);
  else
    c->launches++, k_lincomb_add_dyn<double><<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.ldv, P.Z, kd, x);
  if ((rc = check_launch(c, "FGMRES update"))) return rc;
  if ((rc = residual_dev(c, b, x, P.r, &kd->rr, Guard{&kd->check, 1}))) return rc;
  c->launches++, k_kry_confirm<<<1, 1, 0, c->stream>>>(kd, h_outer, use_graph);
  return check_launch(c, "FGMRES confirm");
}

// Reads one int of the device state (host loop of the stream form).
static int read_flag(Ctx *c, const int *dev, int *out) {
  cudaMemcpyAsync(&c->kd_host->inner_go, dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "FGMRES: flag read failed");
  *out = c->kd_host->inner_go;
  return VFS_OK;
}

// A WHILE conditional node on the graph being captured on c->stream, its body captured
// on cap_streams[level] (c->stream switched to it until while_end).
struct WhileLoop {
  cudaGraphNode_t node;
  cudaStream_t outer;
};
static int cond_handle(Ctx *c, cudaGraphConditionalHandle *h) {
  cudaStreamCaptureStatus st;
  cudaGraph_t graph;
  if (cudaStreamGetCaptureInfo(c->stream, &st, nullptr, &graph, nullptr, nullptr) != cudaSuccess ||
      st != cudaStreamCaptureStatusActive)
    return set_err(c, VFS_ERR_CUDA, "step graph: stream not capturing");
  if (cudaGraphConditionalHandleCreate(h, graph, 0, 0) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "step graph: conditional handle creation failed");
  return VFS_OK;
}
static int while_begin(Ctx *c, int level, cudaGraphConditionalHandle h, WhileLoop &w) {
  cudaStreamCaptureStatus st;
  cudaGraph_t graph;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  if (cudaStreamGetCaptureInfo(c->stream, &st, nullptr, &graph, &deps, &ndeps) != cudaSuccess ||
      st != cudaStreamCaptureStatusActive)
    return set_err(c, VFS_ERR_CUDA, "step graph: stream not capturing");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  if (cudaGraphAddNode(&w.node, graph, deps, ndeps, &p) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "step graph: conditional node creation failed");
  if (cudaStreamUpdateCaptureDependencies(c->stream, &w.node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "step graph: capture dependencies");
  cudaGraph_t body = p.conditional.phGraph_out[0];
  if (!c->cap_streams[level] && cudaStreamCreateWithFlags(&c->cap_streams[level], cudaStreamNonBlocking) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "step graph: stream creation failed");
  if (cudaStreamBeginCaptureToGraph(c->cap_streams[level], body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
      cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "step graph: body capture failed");
  w.outer = c->stream;
  c->stream = c->cap_streams[level];
  return VFS_OK;
}
static int while_end(Ctx *c, WhileLoop &w) {
  cudaGraph_t body = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &body);
  c->stream = w.outer;
  if (e != cudaSuccess) return set_err(c, VFS_ERR_CUDA, std::string("step graph: body capture: ") + cudaGetErrorString(e));
  return VFS_OK;
}

// Right-preconditioned flexible GMRES (Saad 1993) in FP64 with classical Gram-Schmidt,
// re-orthogonalised where the first pass loses more than half the norm.  Solves A phi = b
// for the fluid unknowns, then removes the mean (Remove_Nullspace) and fills the grid Phi
// like Convert_Phi2_Phi (poisson.c:92): non-fluid interior cells 0, periodic ghosts from
// their images, other ghosts 0.
// Initial guess: the reference hands HYPRE's GMRES the persistent Phi2, created zero once
// with the unknown numbering (poisson.c:280-282) and holding the previous solution after
// every solve (poisson_hypre.c:571, 604).  Here the previous solution is the grid Phi on
// the unknowns (P.guess), so the first solve after the operator is built starts from 0
// and later ones from the last Phi; zero_guess = 1 always starts from 0.  The target is
// rtol * ||b|| either way, as in HYPRE's GMRES.
// The iteration runs on the device (KryDev); the host drives its two loops by reading
// their flags, or, while a step is captured, the loops are conditional WHILE nodes.
// The solver options with defaults filled in (precision 2 falls back to 0 for the
// transposed operator, which has no FP32 form).
static vfs_solve_opts solve_opts(const Ctx *c, const vfs_solve_opts *oin) {
  vfs_solve_opts o;
  memset(&o, 0, sizeof(o));
  o.precision = 0; o.restart = 30; o.max_iter = 200; o.levels = 0; o.pre_smooth = 3; o.post_smooth = 3;
  o.coarse_iters = 4; o.rtol = 1e-10; o.atol = 0.0;
  if (oin) {
    o.precision = oin->precision;
    if (oin->restart > 0) o.restart = oin->restart;
    if (oin->max_iter > 0) o.max_iter = oin->max_iter;
    if (oin->levels > 0) o.levels = oin->levels;
    if (oin->pre_smooth > 0) o.pre_smooth = oin->pre_smooth;
    if (oin->post_smooth > 0) o.post_smooth = oin->post_smooth;
    if (oin->coarse_iters > 0) o.coarse_iters = oin->coarse_iters;
    o.zero_guess = oin->zero_guess;
    if (oin->rtol > 0) o.rtol = oin->rtol;
    if (oin->atol > 0) o.atol = oin->atol;
  }
  if (o.restart > kKryMax) o.restart = kKryMax;
  if (o.pre_smooth < 1) o.pre_smooth = 1;
  if (o.coarse_iters < 1) o.coarse_iters = 1;
  if (o.precision == 2 && c->ps.transpose) o.precision = 0;
  return o;
}

// The inner tolerance of precision 2: an FP32 cycle reduces its residual estimate by at
// most this factor before the FP64 residual is formed again (FP32 keeps about 7 digits).
static const double kInnerRtol = 1e-5;

// Allocates the solver's workspace for options o (the Krylov basis, and for precision 2
// its FP32 form); outside a stream capture.
int poisson_prepare(Ctx *c, const vfs_solve_opts *oin) {
  const vfs_solve_opts o = solve_opts(c, oin);
  Poisson &P = c->ps;
  const long long N = c->g.N;
  const bool f32 = o.precision == 2;
  if (P.restart >= o.restart && (!f32 || P.restart32 >= o.restart)) return VFS_OK;
  if (c->capturing) return set_err(c, VFS_ERR_STATE, "poisson_solve: Krylov basis not allocated before capture");
  c->setup_epoch++;  // a captured step graph holds the old buffers
  P.ldv = (N + 31) / 32 * 32;
  if (P.restart < o.restart) {
    cudaFree(P.V); cudaFree(P.Z);
    P.V = P.Z = nullptr;
    P.restart = 0;
    if (cudaMalloc(&P.V, sizeof(double) * P.ldv * (o.restart + 1)) != cudaSuccess ||
        cudaMalloc(&P.Z, sizeof(double) * P.ldv * o.restart) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "poisson_solve: Krylov basis allocation failed");
    P.restart = o.restart;
  }
  if (!f32) return VFS_OK;
  if (P.restart32 < o.restart) {
    cudaFree(P.V32); cudaFree(P.Z32); cudaFree(P.w32);
    P.V32 = P.Z32 = P.w32 = nullptr;
    P.restart32 = 0;
    if (cudaMalloc(&P.V32, sizeof(float) * P.ldv * (o.restart + 1)) != cudaSuccess ||
        cudaMalloc(&P.Z32, sizeof(float) * P.ldv * o.restart) != cudaSuccess ||
        cudaMalloc(&P.w32, sizeof(float) * P.ldv) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "poisson_solve: FP32 Krylov basis allocation failed");
    P.restart32 = o.restart;
  }
  return VFS_OK;
}

int poisson_solve(Ctx *c, const vfs_solve_opts *oin, vfs_solve_stats *st) {
  const vfs_solve_opts o = solve_opts(c, oin);
  Poisson &P = c->ps;
  const long long N = c->g.N;
  int rc;
  if ((rc = poisson_prepare(c, &o))) return rc;
  if ((rc = ensure_red(c, 34 * std::max(kKryBlocks, kry_grid(c)) + (int)nblocks(N, 256) + 64))) return rc;
  if (!c->capturing) cudaEventRecord(c->ev0, c->stream);
  KryDev *kd = c->kd;
  double *x = c->f[VFS_PHI][0];
  const double *b = c->f[VFS_B][0];
  const bool warm = P.guess && !o.zero_guess && !P.transpose;
  if (warm) {
    const int nb = (int)nblocks(N, 256);
    c->launches++, k_guess<<<nb, 256, 0, c->stream>>>(N, P.fluid, b, x, c->red);
    c->launches++, k_sum_parts_g<<<1, 1024, 0, c->stream>>>(c->red, nb, &kd->bb, always());
    if ((rc = check_launch(c, "k_guess"))) return rc;
  } else {
    cudaMemsetAsync(x, 0, sizeof(double) * N, c->stream);
  }
  if ((rc = residual_dev(c, b, x, P.r, &kd->rr, always()))) return rc;  // from x = 0: r = b
  const int m = o.restart;
  const int use_graph = c->capturing ? 1 : 0;
  cudaGraphConditionalHandle h_outer = 0, h_inner = 0;
  if (use_graph && (rc = cond_handle(c, &h_outer))) return rc;
  c->launches++, k_kry_init<<<1, 1, 0, c->stream>>>(kd, o.rtol, o.atol, warm ? 1 : 0, o.max_iter, m,
                                                     (unsigned long long)h_outer, use_graph,
                                                     o.precision == 2 ? kInnerRtol : 0.0);
  if ((rc = check_launch(c, "k_kry_init"))) return rc;
  if (use_graph) {
    WhileLoop w0, w1;
    if ((rc = while_begin(c, 0, h_outer, w0))) return rc;
    if ((rc = cond_handle(c, &h_inner))) return rc;
    const long long l0 = c->launches;
    if ((rc = kry_cycle_start(c, o, b, x, (unsigned long long)h_inner, 1))) return rc;
    if ((rc = while_begin(c, 1, h_inner, w1))) return rc;
    const long long l1 = c->launches;
    if ((rc = kry_body(c, o, (unsigned long long)h_inner, 1))) return rc;
    c->sg.body_launches = c->launches - l1;
    if ((rc = while_end(c, w1))) return rc;
    if ((rc = kry_cycle_end(c, o, b, x, (unsigned long long)h_outer, 1))) return rc;
    c->sg.cycle_launches = c->launches - l0 - c->sg.body_launches;
    if ((rc = while_end(c, w0))) return rc;
  } else {
    for (;;) {
      int go = 0;
      if ((rc = read_flag(c, &kd->outer_go, &go))) return rc;
      if (!go) break;
      if ((rc = kry_cycle_start(c, o, b, x, 0, 0))) return rc;
      for (;;) {
        if ((rc = read_flag(c, &kd->inner_go, &go))) return rc;
        if (!go) break;
        if ((rc = kry_body(c, o, 0, 0))) return rc;
      }
      if ((rc = kry_cycle_end(c, o, b, x, 0, 0))) return rc;
    }
  }
  // Remove_Nullspace: phi += -mean(phi) over fluid cells
  {
    const int nb = (int)nblocks(N, 256);
    c->launches++, k_sum_fluid<<<nb, 256, 0, c->stream>>>(N, P.fluid, x, c->red);
    if ((rc = check_launch(c, "k_sum_fluid"))) return rc;
    if ((rc = reduce_to(c, c->red, nb, c->ds + DS_PHISUM))) return rc;
    c->launches++, k_shift_mean<<<nblocks(N, 256), 256, 0, c->stream>>>(N, P.fluid, c->ds, (double)P.nfluid, x);
    if ((rc = check_launch(c, "k_shift_mean"))) return rc;
  }
  // Convert_Phi2_Phi: periodic ghosts take their images (x is 0 elsewhere off-fluid)
  if ((rc = periodic_copy1(c, x))) return rc;
  if (!P.transpose) P.guess = true;
  if (c->capturing) return VFS_OK;  // statistics after the replay
  cudaEventRecord(c->ev1, c->stream);
  cudaMemcpyAsync(c->kd_host, kd, sizeof(KryDev), cudaMemcpyDeviceToHost, c->stream);
  if (cudaEventSynchronize(c->ev1) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "poisson_solve: failed");
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  vfs_solve_stats s;
  memset(&s, 0, sizeof(s));
  s.iterations = c->kd_host->it;
  s.converged = c->kd_host->conv ? 1 : 0;
  s.rfinal = c->kd_host->rnorm;
  s.r0 = c->kd_host->r0;
  s.ms = ms;
  if (st) *st = s;
  return s.converged ? VFS_OK : set_err(c, VFS_ERR_NOT_CONVERGED, "poisson_solve: iteration cap reached");
}

// ------------------------------------------------------------------ UpdatePressure
// poisson.c:3144-3305: P += Phi on fluid cells, P = 0 where nvert > 1.1, then the
// periodic ghosts of P and Phi take their images.
__global__ void k_update_pressure(Grid g, const uint8_t *__restrict__ nv, const double *__restrict__ phi, double *P) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  if (nv[p] == 0) P[p] += phi[p];
  if (nv[p] >= 2) P[p] = 0;
}

int update_pressure(Ctx *c) {
  int rc;
  c->launches++, k_update_pressure<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->nv, c->f[VFS_PHI][0], c->f[VFS_P][0]);
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

// Projection at interior point p with the face-metric products G (9 x N, k_gab) and
// the face Jacobians; with kUpdate the same thread first applies UpdatePressure to P
// (the two touch disjoint data: UpdatePressure reads Phi and writes P, Projection reads
// Phi and writes Ucont), so one pass serves both.
template <bool kUpdate>
__global__ void __launch_bounds__(256) k_projection(Grid g, const double *__restrict__ G,
                                                    const double *__restrict__ iaj, const double *__restrict__ jaj,
                                                    const double *__restrict__ kaj, const uint8_t *__restrict__ nv,
                                                    const double *__restrict__ phi, V3 uc, double *P) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) return;
  if (kUpdate) {  // poisson.c:3144-3305
    if (nv[p] == 0) P[p] += phi[p];
    if (nv[p] >= 2) P[p] = 0;
  }
  const long long sx = 1, sy = mx, sz = (long long)mx * my, N = g.N;
  const double coeff = 1.0, r1 = 1.0, r2 = 1.0, r3 = 1.0;
  if (i < mx - 2 || (g.iper && i == mx - 2)) {
    double dpdc = phi[p + 1] - phi[p];
    if (i == mx - 2 && g.iper) dpdc = phi[p - i + 1] - phi[p];
    const double dpde = cross_phi(phi, p, p + sx, sy, j, my, g.jper, nv[p + sy] + nv[p + sy + sx], nv[p - sy] + nv[p - sy + sx]);
    const double dpdz = cross_phi(phi, p, p + sx, sz, k, mz, g.kper, nv[p + sz] + nv[p + sz + sx], nv[p - sz] + nv[p - sz + sx]);
    if (nv[p] + nv[p + 1] == 0) {
      const double a = iaj[p];
      uc.x[p] -= (dpdc * __ldcs(G + p) * a + dpde * __ldcs(G + N + p) * a + dpdz * __ldcs(G + 2 * N + p) * a) *
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
      const double a = jaj[p];
      uc.y[p] -= (dpdc * __ldcs(G + 3 * N + p) * a + dpde * __ldcs(G + 4 * N + p) * a +
                  dpdz * __ldcs(G + 5 * N + p) * a) *
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
      const double a = kaj[p];
      uc.z[p] -= (dpdc * __ldcs(G + 6 * N + p) * a + dpde * __ldcs(G + 7 * N + p) * a +
                  dpdz * __ldcs(G + 8 * N + p) * a) *
                 g.dt * g.st / coeff / r3;
    }
  }
}

static void launch_projection(Ctx *c, bool update_p) {
  const Grid &g = c->g;
  if (update_p)
    c->launches++, k_projection<true><<<nblocks(g.N, 256), 256, 0, c->stream>>>(
        g, c->gab, c->f[VFS_IAJ][0], c->f[VFS_JAJ][0], c->f[VFS_KAJ][0], c->nv, c->f[VFS_PHI][0],
        field3(c, VFS_UCONT), c->f[VFS_P][0]);
  else
    c->launches++, k_projection<false><<<nblocks(g.N, 256), 256, 0, c->stream>>>(
        g, c->gab, c->f[VFS_IAJ][0], c->f[VFS_JAJ][0], c->f[VFS_KAJ][0], c->nv, c->f[VFS_PHI][0],
        field3(c, VFS_UCONT), nullptr);
}

// Component-wise periodic copy after Projection (poisson.c:3013-3046): a component is
// copied only when its own direction is periodic at the point.
__global__ void k_periodic_copy_comp(Grid g, V3 u) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  int ii = wrapi(g, i), jj = wrapj(g, j), kk = wrapk(g, k);
  if (ii == i && jj == j && kk == k) return;
  long long s = lidx(g, ii, jj, kk);
  if (ii != i) u.x[p] = u.x[s];
  if (jj != j) u.y[p] = u.y[s];
  if (kk != k) u.z[p] = u.z[s];
}

int projection(Ctx *c) {
  int rc;
  if ((rc = ensure_gab(c))) return rc;
  launch_projection(c, false);
  if ((rc = check_launch(c, "k_projection"))) return rc;
  if (c->g.iper || c->g.jper || c->g.kper) {
    c->launches++, k_periodic_copy_comp<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
    if ((rc = check_launch(c, "k_periodic_copy_comp"))) return rc;
  }
  return contra2cart(c);
}

// UpdatePressure, Projection and its Contra2Cart as the step runs them (solvers.c:1341-1342):
// UpdatePressure's P += Phi fused into the projection kernel, the periodic ghosts of P and
// of the projected Ucont, then Contra2Cart; with fuse_divergence the Contra2Cart interior
// kernel also forms the block maxima of Divergence (main.c:1083-1090) on the same Ucont
// (valid when nothing changes Ucont between Contra2Cart and Divergence: no IB nodes), and
// divergence_finish reduces them.  Phi's periodic ghosts, which UpdatePressure also
// refreshes, already hold their images from the end of the Poisson solve.
int correction(Ctx *c, bool fuse_divergence) {
  int rc;
  if ((rc = ensure_gab(c))) return rc;
  launch_projection(c, true);
  if ((rc = check_launch(c, "k_projection"))) return rc;
  if ((rc = periodic_copy1(c, c->f[VFS_P][0]))) return rc;
  if (c->g.iper || c->g.jper || c->g.kper) {
    c->launches++, k_periodic_copy_comp<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
    if ((rc = check_launch(c, "k_periodic_copy_comp"))) return rc;
  }
  if (fuse_divergence && (rc = ensure_red(c, (int)nblocks(c->g.N, 256) + 64))) return rc;
  return contra2cart_div(c, fuse_divergence);
}

// ------------------------------------------------------------------ Divergence
// main.c:1083-1090: max |(dU + dV + dW) * aj| over interior cells with no solid in the
// 7-point neighbourhood.
// One point per thread; the block maxima go to parts[blockIdx.x].
__global__ void k_divergence(Grid g, CV3 uc, const double *__restrict__ aj, const uint8_t *__restrict__ nv,
                             double *parts) {
  __shared__ double sh[8];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  double mval = 0;
  if (p < g.N) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2) {
      double d = fabs((uc.x[p] - uc.x[p - 1] + uc.y[p] - uc.y[p - sy] + uc.z[p] - uc.z[p - sz]) * aj[p]);
      if (nv[p] + nv[p + sz] + nv[p - sz] + nv[p + sy] + nv[p - sy] + nv[p + 1] + nv[p - 1] > 0) d = 0.;
      mval = d;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mval = fmax(mval, __shfl_down_sync(0xffffffffu, mval, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mval;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int w = 0; w < 8; w++) m = fmax(m, sh[w]);
    parts[blockIdx.x] = m;
  }
}

// Maximum of n block maxima (one block).
// Maximum of n block partials (non-negative) in one block of 1024 threads, eight loads in
// flight per thread.
__global__ void __launch_bounds__(1024) k_max_parts(const double *parts, int n, double *out) {
  __shared__ double sh[32];
  double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int q = threadIdx.x;
  for (; q + 7 * 1024 < n; q += 8 * 1024) {
#pragma unroll
    for (int u = 0; u < 8; u++) m[u] = fmax(m[u], parts[q + u * 1024]);
  }
  for (; q < n; q += 1024) m[0] = fmax(m[0], parts[q]);
  double t = fmax(fmax(fmax(m[0], m[1]), fmax(m[2], m[3])), fmax(fmax(m[4], m[5]), fmax(m[6], m[7])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x < 32) {
    t = sh[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
    if (threadIdx.x == 0) out[0] = t;
  }
}

int divergence(Ctx *c, double *maxdiv) {
  int rc;
  const int nb = (int)nblocks(c->g.N, 256);
  if ((rc = ensure_red(c, nb + 64))) return rc;
  c->launches++, k_divergence<<<nb, 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_UCONT)), c->f[VFS_AJ][0], c->nv, c->red + 64);
  if ((rc = check_launch(c, "k_divergence"))) return rc;
  return divergence_finish(c, maxdiv);
}

// Maximum of the block maxima of Divergence (in c->red + 64, one per block of 256 points)
// into the device scalar; read back into *maxdiv unless capturing.
int divergence_finish(Ctx *c, double *maxdiv) {
  int rc;
  const int nb = (int)nblocks(c->g.N, 256);
  c->launches++, k_max_parts<<<1, 1024, 0, c->stream>>>(c->red + 64, nb, c->ds + DS_MAXDIV);
  if ((rc = check_launch(c, "k_max_parts"))) return rc;
  if (c->capturing || !maxdiv) return VFS_OK;
  if ((rc = ds_fetch(c))) return rc;
  *maxdiv = c->ds_out[DS_MAXDIV];
  return VFS_OK;
}

}  // namespace vfs

// ------------------------------------------------------------------ diagnostics
namespace vfs {
// Launches one kernel of the path `reps` times on the context's stream (no host sync),
// so a caller can bracket it with events recorded on that stream.
int run_kernel(Ctx *c, int which, int reps) {
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
        rc = poisson_apply_dev(c, c->f[VFS_PHI][0], P.t);
        if (rc) return rc;
        break;
      case 4: rc = mg_sweep_fine(c, 0); if (rc) return rc; break;
      case 5: rc = mg_sweep_fine(c, 1); if (rc) return rc; break;
      case 7: rc = formfunction2_split(c, 1.0, false, 0.0); if (rc) return rc; break;
      case 8: rc = formfunction2(c, 1.0, false, 0.0); if (rc) return rc; break;
      case 11: rc = formfunction2_onepass(c, 1.0, false, 0.0); if (rc) return rc; break;
      case 12: rc = pressure_gradient(c); if (rc) return rc; break;
      case 13:
        if ((rc = ensure_gab(c))) return rc;
        launch_projection(c, true);
        if ((rc = check_launch(c, "k_projection"))) return rc;
        break;
      case 14: {
        extern int contra2cart_interior_div(Ctx *);
        if ((rc = contra2cart_interior_div(c))) return rc;
        break;
      }
      case 9:
      case 10: {  // one multigrid V-cycle (the preconditioner) on B, FP32 or FP64, into a work vector
        vfs_solve_opts o;
        memset(&o, 0, sizeof(o));
        o.precision = which == 9 ? 0 : 1;
        o.pre_smooth = 3; o.post_smooth = 3; o.coarse_iters = 4;
        rc = mg_precondition(c, c->f[VFS_B][0], P.t, o);
        if (rc) return rc;
        break;
      }
      case 6:
        if ((rc = ensure_gab(c))) return rc;
        launch_projection(c, false);
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
