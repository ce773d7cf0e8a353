// Momentum predictor kernels for sm_100a: Contra2Cart, Formfunction_2, Pressure_Gradient,
// Calc_k_Flux, the wall/periodic part of FormBCS and the 4-stage RungeKutta driver.
//
// All arithmetic is FP64 in the reference's operation order (the library is compiled
// with --fmad=false), so pointwise outputs match the reference bit for bit; only
// reductions differ in summation order.
#include <cmath>
#include <cstdio>

#include "vfs_internal.cuh"

namespace vfs {

__device__ __forceinline__ double dot3(double ax, double ay, double az, double bx, double by, double bz) {
  return ax * bx + ay * by + az * bz;
}

// ------------------------------------------------------------------ periodic copies
// Shell kernel: every point with a periodic-boundary index copies the value of its
// periodic image (all flagged directions at once), as the reference's copy loops do
// (e.g. momentum.c:641-669, rhs.c:161-181).  Sources are never flagged points, so the
// copy is order independent.
// One thread per point of the ghost planes of the periodic directions (points on two such
// planes appear twice and write the same value); each takes the value of its periodic
// image, whose indices are all interior or non-periodic ghosts, so no thread reads a
// point another one writes.
__global__ void k_periodic_copy(Grid g, double *a, double *b, double *c) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ni = g.iper ? 2LL * g.my * g.mz : 0, nj = g.jper ? 2LL * g.mx * g.mz : 0;
  const long long nk = g.kper ? 2LL * g.mx * g.my : 0;
  int i, j, k;
  if (t < ni) {
    const long long r = t >> 1;
    i = (t & 1) ? g.mx - 1 : 0; j = (int)(r % g.my); k = (int)(r / g.my);
  } else if ((t -= ni) < nj) {
    const long long r = t >> 1;
    j = (t & 1) ? g.my - 1 : 0; i = (int)(r % g.mx); k = (int)(r / g.mx);
  } else if ((t -= nj) < nk) {
    const long long r = t >> 1;
    k = (t & 1) ? g.mz - 1 : 0; i = (int)(r % g.mx); j = (int)(r / g.mx);
  } else {
    return;
  }
  const long long p = lidx(g, i, j, k);
  const long long s = lidx(g, wrapi(g, i), wrapj(g, j), wrapk(g, k));
  a[p] = a[s];
  if (b) b[p] = b[s];
  if (c) c[p] = c[s];
}

static long long ghost_points(const Grid &g) {
  return (g.iper ? 2LL * g.my * g.mz : 0) + (g.jper ? 2LL * g.mx * g.mz : 0) + (g.kper ? 2LL * g.mx * g.my : 0);
}

int periodic_copy3(Ctx *c, V3 v) {
  if (!(c->g.iper || c->g.jper || c->g.kper)) return VFS_OK;
  c->launches++, k_periodic_copy<<<nblocks(ghost_points(c->g), 256), 256, 0, c->stream>>>(c->g, v.x, v.y, v.z);
  return check_launch(c, "k_periodic_copy");
}
int periodic_copy1(Ctx *c, double *s) {
  if (!(c->g.iper || c->g.jper || c->g.kper)) return VFS_OK;
  c->launches++, k_periodic_copy<<<nblocks(ghost_points(c->g), 256), 256, 0, c->stream>>>(c->g, s, nullptr, nullptr);
  return check_launch(c, "k_periodic_copy");
}

// ------------------------------------------------------------------ Contra2Cart
// Interior Cartesian velocity from averaged face fluxes by Cramer's rule on the centre
// metrics (rhs.c:186-233).  Cells with nvert >= 0.1 keep their value.
__global__ void k_contra2cart_interior(Grid g, CV3 uc, CV3 csi, CV3 eta, CV3 zet,
                                       const uint8_t *__restrict__ nv, V3 ucat) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  if (nv[p] != 0) return;
  const double m00 = csi.x[p], m01 = csi.y[p], m02 = csi.z[p];
  const double m10 = eta.x[p], m11 = eta.y[p], m12 = eta.z[p];
  const double m20 = zet.x[p], m21 = zet.y[p], m22 = zet.z[p];
  const double q0 = 0.5 * (uc.x[p - 1] + uc.x[p]);
  const double q1 = 0.5 * (uc.y[p - g.mx] + uc.y[p]);
  const double q2 = 0.5 * (uc.z[p - (long long)g.mx * g.my] + uc.z[p]);
  const double det = m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) +
                     m02 * (m10 * m21 - m11 * m20);
  const double det0 = q0 * (m11 * m22 - m12 * m21) - q1 * (m01 * m22 - m02 * m21) +
                      q2 * (m01 * m12 - m02 * m11);
  const double det1 = -q0 * (m10 * m22 - m12 * m20) + q1 * (m00 * m22 - m02 * m20) -
                      q2 * (m00 * m12 - m02 * m10);
  const double det2 = q0 * (m10 * m21 - m11 * m20) - q1 * (m00 * m21 - m01 * m20) +
                      q2 * (m00 * m11 - m01 * m10);
  ucat.x[p] = det0 / det;
  ucat.y[p] = det1 / det;
  ucat.z[p] = det2 / det;
}

// k_contra2cart_interior plus the block maxima of Divergence (main.c:1083-1090) on the
// same Ucont: |(dU + dV + dW) aj| at interior cells with no solid in the 7-point
// neighbourhood, 0 elsewhere; one partial per block of 256 threads in parts[blockIdx.x]
// (the layout k_divergence writes).
__global__ void __launch_bounds__(256) k_contra2cart_div(Grid g, CV3 uc, CV3 csi, CV3 eta, CV3 zet,
                                                         const double *__restrict__ aj,
                                                         const uint8_t *__restrict__ nv, V3 ucat, double *parts) {
  __shared__ double sh[8];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  double dmax = 0;
  if (p < g.N) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2) {
      const double ux0 = uc.x[p - 1], ux1 = uc.x[p], uy0 = uc.y[p - sy], uy1 = uc.y[p];
      const double uz0 = uc.z[p - sz], uz1 = uc.z[p];
      if (nv[p] + nv[p + sz] + nv[p - sz] + nv[p + sy] + nv[p - sy] + nv[p + 1] + nv[p - 1] == 0)
        dmax = fabs((ux1 - ux0 + uy1 - uy0 + uz1 - uz0) * aj[p]);
      if (nv[p] == 0) {
        const double m00 = csi.x[p], m01 = csi.y[p], m02 = csi.z[p];
        const double m10 = eta.x[p], m11 = eta.y[p], m12 = eta.z[p];
        const double m20 = zet.x[p], m21 = zet.y[p], m22 = zet.z[p];
        const double q0 = 0.5 * (ux0 + ux1), q1 = 0.5 * (uy0 + uy1), q2 = 0.5 * (uz0 + uz1);
        const double det = m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) +
                           m02 * (m10 * m21 - m11 * m20);
        const double det0 = q0 * (m11 * m22 - m12 * m21) - q1 * (m01 * m22 - m02 * m21) +
                            q2 * (m01 * m12 - m02 * m11);
        const double det1 = -q0 * (m10 * m22 - m12 * m20) + q1 * (m00 * m22 - m02 * m20) -
                            q2 * (m00 * m12 - m02 * m10);
        const double det2 = q0 * (m10 * m21 - m11 * m20) - q1 * (m00 * m21 - m01 * m20) +
                            q2 * (m00 * m11 - m01 * m10);
        ucat.x[p] = det0 / det;
        ucat.y[p] = det1 / det;
        ucat.z[p] = det2 / det;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = dmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0;
    for (int w = 0; w < 8; w++) mx = fmax(mx, sh[w]);
    parts[blockIdx.x] = mx;
  }
}

// Covariant metric inverse (Calculate_Covariant_metrics, rhs2.c:538).
__device__ void covariant(const double g[3][3], double G[3][3]) {
  const double a11 = g[0][0], a12 = g[0][1], a13 = g[0][2];
  const double a21 = g[1][0], a22 = g[1][1], a23 = g[1][2];
  const double a31 = g[2][0], a32 = g[2][1], a33 = g[2][2];
  double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
  G[0][0] = (a33 * a22 - a32 * a23) / det, G[0][1] = -(a33 * a12 - a32 * a13) / det, G[0][2] = (a23 * a12 - a22 * a13) / det;
  G[1][0] = -(a33 * a21 - a31 * a23) / det, G[1][1] = (a33 * a11 - a31 * a13) / det, G[1][2] = -(a23 * a11 - a21 * a13) / det;
  G[2][0] = (a32 * a21 - a31 * a22) / det, G[2][1] = -(a32 * a11 - a31 * a12) / det, G[2][2] = (a22 * a11 - a21 * a12) / det;
}

// Reader of a 3-component field for the boundary rules (the transposed kernel evaluates
// them with unit-vector readers instead, ProbeAcc).
struct FieldAcc {
  CV3 a;
  __device__ __forceinline__ double operator()(long long q, int c) const { return c == 0 ? a.x[q] : (c == 1 ? a.y[q] : a.z[q]); }
};

// Slip-wall ghost: mirror the neighbour's old velocity about the wall normal taken from
// the covariant metric column `col` of the neighbour cell (rhs.c:384-478).
template <class UO>
__device__ void slip_ghost(long long nb, int col, double sgn, const Metrics &m, const UO &uo, double *o) {
  double g[3][3], G[3][3];
  g[0][0] = m.csi.x[nb], g[0][1] = m.csi.y[nb], g[0][2] = m.csi.z[nb];
  g[1][0] = m.eta.x[nb], g[1][1] = m.eta.y[nb], g[1][2] = m.eta.z[nb];
  g[2][0] = m.zet.x[nb], g[2][1] = m.zet.y[nb], g[2][2] = m.zet.z[nb];
  covariant(g, G);
  double nx = G[0][col], ny = G[1][col], nz = G[2][col];
  if (sgn < 0) nx = -nx, ny = -ny, nz = -nz;
  double sum = sqrt(nx * nx + ny * ny + nz * nz);
  nx /= sum, ny /= sum, nz /= sum;
  double un = uo(nb, 0) * nx + uo(nb, 1) * ny + uo(nb, 2) * nz;
  o[0] = uo(nb, 0) - 2 * un * nx;
  o[1] = uo(nb, 1) - 2 * un * ny;
  o[2] = uo(nb, 2) - 2 * un * nz;
}

// Boundary part of Contra2Cart_2 (rhs.c:291-675), phase 1: every point the reference's
// boundary loop assigns gets its new value in `out` (reads the pre-loop snapshot `ucat`),
// `flag` marks it.  Phase 2 (k_bc_commit) copies the marked values, which reproduces the
// reference's read-from-lUcat / write-to-Ucat semantics exactly.
// The rule at point p as a function of the readers lu (the snapshot) and uo (Ucat_o):
// whether it assigns p, and the value v.
template <class LU, class UO>
__device__ __forceinline__ bool contra2cart_bc_rule(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv,
                                                    const LU &lu, const UO &uo, long long p, int i, int j, int k,
                                                    double v[3]) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const int *bc = g.bc;
  bool w = false;
  if (nv[p] == 3) {  // (int)(nvert+0.1)==3 and fixed bodies (rhs.c:296-299)
    v[0] = 0; v[1] = 0; v[2] = 0;
    return true;
  }
  // every rule below acts on a ghost point or on a cell (1 or mx-2, 1, k)
  if (!(i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1 ||
        (j == 1 && (i == 1 || i == mx - 2))))
    return false;
  v[0] = lu(p, 0); v[1] = lu(p, 1); v[2] = lu(p, 2);
  int solid_flag = 0;
  if (bc[3] == 13 && j == my - 1) {
    v[0] = lu(p - sy, 0); v[2] = lu(p - sy, 2); v[1] = -lu(p - sy, 1); w = true;
  }
  if (bc[3] == 14 && j == my - 1) {
    v[0] = lu(p - sy, 0); v[1] = lu(p - sy, 1); v[2] = -lu(p - sy, 2); w = true;
  }
  if (bc[0] == 10 && i == 0 && (j != 0 && k != 0)) {
    slip_ghost(p + sx, 0, -1.0, m, uo, v); w = true;
    if (nv[p + sx] != 0) v[0] = v[1] = v[2] = 0;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  if (bc[1] == 10 && i == mx - 1 && (j != 0 && k != 0)) {
    slip_ghost(p - sx, 0, 1.0, m, uo, v); w = true;
    if (nv[p - sx] != 0) v[0] = v[1] = v[2] = 0;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  if (bc[2] == 10 && j == 0 && (i != 0 && k != 0)) {
    slip_ghost(p + sy, 1, -1.0, m, uo, v); w = true;
    if (nv[p + sy] != 0) v[0] = v[1] = v[2] = 0;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  if ((bc[3] == 10 || bc[3] == -10) && j == my - 1 && (i != 0 && k != 0)) {
    slip_ghost(p - sy, 1, 1.0, m, uo, v); w = true;
    if (nv[p - sy] != 0) v[0] = v[1] = v[2] = 0;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  // no-slip ghosts (rhs.c:511-534)
  if (i == 0 && bc[0] == 1 && (j != 0 && k != 0)) {
    v[0] = -1 * lu(p + sx, 0); v[1] = -1 * lu(p + sx, 1); v[2] = -1 * lu(p + sx, 2); w = true; solid_flag = 1;
  }
  if (i == mx - 1 && bc[1] == 1 && (j != 0 && k != 0)) {
    v[0] = -1 * lu(p - sx, 0); v[1] = -1 * lu(p - sx, 1); v[2] = -1 * lu(p - sx, 2); w = true; solid_flag = 1;
  }
  if (j == 0 && bc[2] == 1 && (i != 0 && k != 0)) {
    v[0] = -1 * lu(p + sy, 0); v[1] = -1 * lu(p + sy, 1); v[2] = -1 * lu(p + sy, 2); w = true; solid_flag = 1;
  }
  if (j == my - 1 && bc[3] == 1 && (i != 0 && k != 0)) {
    v[0] = -1 * lu(p - sy, 0); v[1] = -1 * lu(p - sy, 1); v[2] = -1 * lu(p - sy, 2); w = true; solid_flag = 1;
  }
  if (k == 0 && bc[4] == 1 && (i != 0 && j != 0)) {
    v[0] = -1 * lu(p + sz, 0); v[1] = -1 * lu(p + sz, 1); v[2] = -1 * lu(p + sz, 2); w = true; solid_flag = 1;
  }
  if (k == mz - 1 && bc[5] == 1 && (i != 0 && j != 0)) {
    v[0] = -1 * lu(p - sz, 0); v[1] = -1 * lu(p - sz, 1); v[2] = -1 * lu(p - sz, 2); w = true; solid_flag = 1;
  }
  if (j == my - 1 && bc[3] == 2) {
    if (solid_flag) { v[0] = 2.0 - uo(p - sy, 0); v[1] = -uo(p - sy, 1); v[2] = -uo(p - sy, 2); }
    else { v[0] = 2.0 - lu(p - sy, 0); v[1] = -lu(p - sy, 1); v[2] = -lu(p - sy, 2); }
    w = true;
  }
  if (j == 0 && bc[2] == 12) {
    v[0] = -lu(p + sy, 0); v[1] = -lu(p + sy, 1); v[2] = 2.0 - lu(p + sy, 2); w = true;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  if (j == my - 1 && bc[3] == 12) {
    v[0] = -lu(p - sy, 0); v[1] = -lu(p - sy, 1); v[2] = 2.0 - lu(p - sy, 2); w = true;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  // outflow (rhs.c:573-597)
  if (bc[3] == 4 && j == my - 1 && (i != 0 && i != mx - 1 && k != 0 && k != mz - 1)) {
    v[0] = lu(p - sy, 0); v[1] = lu(p - sy, 1); v[2] = lu(p - sy, 2); w = true;
  }
  if (bc[5] == 4 && k == mz - 1 && (i != 0 && i != mx - 1 && j != 0 && j != my - 1)) {
    if (nv[p - sz] != 0) { v[0] = v[1] = v[2] = 0; w = true; }
    if (solid_flag) { v[0] = v[1] = v[2] = 0; w = true; }
  }
  // corner cells next to two walls (rhs.c:599-604)
  if (i != 0 && i != mx - 1 && j != 0 && j != my - 2 && k != 0 && k != mz - 2) {
    if (bc[0] <= 1 && bc[2] <= 1 && (i == 1 && j == 1)) { v[0] = v[1] = v[2] = 0; w = true; }
    if (bc[1] <= 1 && bc[2] <= 1 && (i == mx - 2 && j == 1)) { v[0] = v[1] = v[2] = 0; w = true; }
  }
  return w;
}

__device__ __forceinline__ void contra2cart_bc_point(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv,
                                                     CV3 lu, CV3 uo, V3 out, uint8_t *flag, long long p, int i,
                                                     int j, int k) {
  double v[3];
  if (contra2cart_bc_rule(g, m, nv, FieldAcc{lu}, FieldAcc{uo}, p, i, j, k, v)) {
    out.x[p] = v[0]; out.y[p] = v[1]; out.z[p] = v[2];
    flag[p] = 1;
  }
}

__global__ void k_contra2cart_bc(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 lu,
                                 CV3 uo, V3 out, uint8_t *flag) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  contra2cart_bc_point(g, m, nv, lu, uo, out, flag, p, i, j, k);
}

// The points the boundary phase can assign apart from solid (nvert 3) cells: the six
// ghost planes and the cells (1, 1, k), (mx-2, 1, k).  Points on two planes appear twice;
// both threads compute and write the same values.
__host__ __device__ inline long long edge_points(const Grid &g) {
  return 2LL * g.my * g.mz + 2LL * g.mx * g.mz + 2LL * g.mx * g.my + 2LL * g.mz;
}
__device__ __forceinline__ long long edge_point(const Grid &g, long long t, int &i, int &j, int &k) {
  const long long ni = 2LL * g.my * g.mz, nj = 2LL * g.mx * g.mz, nk = 2LL * g.mx * g.my;
  if (t < ni) {
    const long long r = t >> 1;
    i = (t & 1) ? g.mx - 1 : 0; j = (int)(r % g.my); k = (int)(r / g.my);
  } else if ((t -= ni) < nj) {
    const long long r = t >> 1;
    j = (t & 1) ? g.my - 1 : 0; i = (int)(r % g.mx); k = (int)(r / g.mx);
  } else if ((t -= nj) < nk) {
    const long long r = t >> 1;
    k = (t & 1) ? g.mz - 1 : 0; i = (int)(r % g.mx); j = (int)(r / g.mx);
  } else {
    t -= nk;
    i = (t & 1) ? g.mx - 2 : 1; j = 1; k = (int)(t >> 1);
  }
  return lidx(g, i, j, k);
}

__global__ void k_contra2cart_bc_edges(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 lu, CV3 uo, V3 out,
                                       uint8_t *flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= edge_points(g)) return;
  int i, j, k;
  const long long p = edge_point(g, t, i, j, k);
  contra2cart_bc_point(g, m, nv, lu, uo, out, flag, p, i, j, k);
}

// Solid cells (nvert 3) get zero (rhs.c:296-299), through the same two-phase buffer.
__global__ void k_solid_zero(long long n, const long long *__restrict__ idx, V3 out, uint8_t *flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long p = idx[t];
  out.x[p] = 0; out.y[p] = 0; out.z[p] = 0;
  flag[p] = 1;
}

__global__ void k_bc_commit_edges(Grid g, CV3 in, uint8_t *flag, V3 dst) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= edge_points(g)) return;
  int i, j, k;
  const long long p = edge_point(g, t, i, j, k);
  if (!flag[p]) return;
  dst.x[p] = in.x[p]; dst.y[p] = in.y[p]; dst.z[p] = in.z[p];
}
__global__ void k_bc_commit_list(long long n, const long long *__restrict__ idx, CV3 in, V3 dst) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long p = idx[t];
  dst.x[p] = in.x[p]; dst.y[p] = in.y[p]; dst.z[p] = in.z[p];
}
// Flags are cleared after every commit so the next call starts from zero.
__global__ void k_bc_clear_edges(Grid g, uint8_t *flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= edge_points(g)) return;
  int i, j, k;
  flag[edge_point(g, t, i, j, k)] = 0;
}
__global__ void k_bc_clear_list(long long n, const long long *__restrict__ idx, uint8_t *flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) flag[idx[t]] = 0;
}

// Indices of the solid (nvert 3) points, in any order.
__global__ void k_collect_solid(long long n, const uint8_t *__restrict__ nv, long long *idx,
                                unsigned long long *count) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n || nv[p] != 3) return;
  const unsigned long long s = atomicAdd(count, 1ull);
  if (idx) idx[s] = p;
}

__global__ void k_bc_commit(long long n, CV3 in, uint8_t *flag, V3 dst) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (!flag[p]) return;
  dst.x[p] = in.x[p]; dst.y[p] = in.y[p]; dst.z[p] = in.z[p];
  flag[p] = 0;
}

// The solid-point list is built once per nvert field (the count, then the indices).
int solid_list(Ctx *c) {
  if (c->nsolid >= 0) return VFS_OK;
  int rc;
  if ((rc = ensure_red(c, 64))) return rc;
  unsigned long long *cnt = (unsigned long long *)(c->red + 62);
  cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream);
  c->launches++, k_collect_solid<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, c->nv, nullptr, cnt);
  unsigned long long n = 0;
  cudaMemcpyAsync(&n, cnt, sizeof(n), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "solid_list: count failed");
  cudaFree(c->solid);
  c->solid = nullptr;
  if (n > 0) {
    if (cudaMalloc(&c->solid, sizeof(long long) * n) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "solid_list: allocation failed");
    cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream);
    c->launches++, k_collect_solid<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, c->nv, c->solid, cnt);
    if ((rc = check_launch(c, "k_collect_solid"))) return rc;
  }
  c->nsolid = (long long)n;
  c->setup_epoch++;
  return VFS_OK;
}

int contra2cart(Ctx *c) { return contra2cart_div(c, false); }

// The interior kernel of contra2cart_div with the divergence maxima alone (diagnostics).
int contra2cart_interior_div(Ctx *c) {
  const Grid &g = c->g;
  int rc;
  if ((rc = ensure_red(c, (int)nblocks(g.N, 256) + 64))) return rc;
  Metrics m = metrics(c);
  c->launches++, k_contra2cart_div<<<nblocks(g.N, 256), 256, 0, c->stream>>>(
      g, cv(field3(c, VFS_UCONT)), m.csi, m.eta, m.zet, m.aj, c->nv, field3(c, VFS_UCAT), c->red + 64);
  return check_launch(c, "k_contra2cart_div");
}

// Contra2Cart; with_divergence: the interior kernel also writes the block maxima of
// Divergence to c->red + 64 (sized by the caller).
int contra2cart_div(Ctx *c, bool with_divergence) {
  const Grid &g = c->g;
  V3 uc = field3(c, VFS_UCONT), ucat = field3(c, VFS_UCAT);
  int rc;
  if ((rc = periodic_copy3(c, uc))) return rc;
  Metrics m = metrics(c);
  if (with_divergence)
    c->launches++, k_contra2cart_div<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, cv(uc), m.csi, m.eta, m.zet, m.aj,
                                                                               c->nv, ucat, c->red + 64);
  else
    c->launches++, k_contra2cart_interior<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, cv(uc), m.csi, m.eta, m.zet, c->nv,
                                                                                    ucat);
  if ((rc = check_launch(c, "k_contra2cart_interior"))) return rc;
  if ((rc = periodic_copy3(c, ucat))) return rc;
  V3 out{c->bcbuf[0], c->bcbuf[1], c->bcbuf[2]};
  uint8_t *fl = c->bcflag;
  if ((rc = solid_list(c))) return rc;
  // solid points get Ucat = 0, except with moving bodies (rhs.c:298)
  const long long ne = edge_points(g), ns = g.moving ? 0 : c->nsolid;
  c->launches++, k_contra2cart_bc_edges<<<nblocks(ne, 256), 256, 0, c->stream>>>(g, m, c->nv, cv(ucat), cv(field3(c, VFS_UCAT_O)),
                                                                  out, fl);
  if (ns > 0) c->launches++, k_solid_zero<<<nblocks(ns, 256), 256, 0, c->stream>>>(ns, c->solid, out, fl);
  if ((rc = check_launch(c, "k_contra2cart_bc"))) return rc;
  c->launches++, k_bc_commit_edges<<<nblocks(ne, 256), 256, 0, c->stream>>>(g, cv(out), fl, ucat);
  if (ns > 0) c->launches++, k_bc_commit_list<<<nblocks(ns, 256), 256, 0, c->stream>>>(ns, c->solid, cv(out), ucat);
  c->launches++, k_bc_clear_edges<<<nblocks(ne, 256), 256, 0, c->stream>>>(g, fl);
  if (ns > 0) c->launches++, k_bc_clear_list<<<nblocks(ns, 256), 256, 0, c->stream>>>(ns, c->solid, fl);
  if ((rc = check_launch(c, "k_bc_commit"))) return rc;
  return periodic_copy3(c, ucat);
}

// ------------------------------------------------------------------ Contra2Cart transpose
// The adjoint of contra2cart (Ucont, Ucat, Ucat_o -> the same slots), as gathers:
//   Ucont' = C Ucont; Ucat1 = I(Ucont') on the interior fluid cells; Ucat2 = C Ucat1;
//   Ucat3 = B(Ucat2, Ucat_o) on the points the boundary phase assigns; Ucat' = C Ucat3
// (C the periodic ghost copy, I the Cramer's-rule interior, B the boundary rules).  B's
// coefficients come from the rules themselves, evaluated at unit vectors.

// Points the boundary phase visits (edge_point): the ghost planes and (1 or mx-2, 1, k).
__device__ __forceinline__ bool c2c_edge(const Grid &g, int i, int j, int k) {
  return i == 0 || i == g.mx - 1 || j == 0 || j == g.my - 1 || k == 0 || k == g.mz - 1 ||
         (j == 1 && (i == 1 || i == g.mx - 2));
}

// Reader for the coefficient evaluations: component c of point q is 1, all else 0 (q < 0:
// the zero vector).
struct ProbeAcc {
  long long q;
  int c;
  __device__ __forceinline__ double operator()(long long r, int cc) const { return (r == q && cc == c) ? 1.0 : 0.0; }
};

// Points within one step of a point the boundary phase visits (the only ones B^T changes).
__device__ __forceinline__ bool c2c_near(const Grid &g, int i, int j, int k) {
  return i <= 2 || i >= g.mx - 3 || j <= 2 || j >= g.my - 2 || k <= 1 || k >= g.mz - 2;
}

// B^T, first half, at the points near the boundary: l2 = l3 off the assigned points (0 on
// them) plus, over the assigned neighbours p (p = q or one step away: every rule reads
// there), dB_p/dUcat2[q]^T l3[p]; lo (the Ucat_o adjoint) += dB_p/dUcat_o[q]^T l3[p].
// The coefficients are the rule's value at unit vectors (evaluation e = 1..3: Ucat2
// component e-1 of q; 4..6: Ucat_o component e-4; 0: whether p is assigned).  l2 is a
// scratch copy (the next kernel moves it into l3), so that no thread reads an entry
// another has already replaced.
__global__ void k_c2c_bc_adjoint(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 l3, V3 l2, V3 lo) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= g.N) return;
  int i, j, k;
  dijk(g, q, i, j, k);
  const bool solid = nv[q] == 3 && !g.moving;  // k_solid_zero
  if (!c2c_near(g, i, j, k) && !solid) return;
  bool assigned = solid;
  double a[3] = {0.0, 0.0, 0.0}, o[3] = {0.0, 0.0, 0.0};
  if (c2c_near(g, i, j, k)) {
#pragma unroll 1
    for (int n = 0; n < 7; n++) {
      int x[3] = {i, j, k};
      if (n > 0) x[(n - 1) >> 1] += (n & 1) ? 1 : -1;
      if (x[0] < 0 || x[0] >= g.mx || x[1] < 0 || x[1] >= g.my || x[2] < 0 || x[2] >= g.mz) continue;
      if (!c2c_edge(g, x[0], x[1], x[2])) continue;
      const long long p = lidx(g, x[0], x[1], x[2]);
      if (nv[p] == 3) {  // assigned zero
        if (n == 0) assigned = true;
        continue;
      }
      const double l[3] = {l3.x[p], l3.y[p], l3.z[p]};
#pragma unroll 1
      for (int e = 0; e < 7; e++) {
        const ProbeAcc A{(e >= 1 && e <= 3) ? q : -1, e - 1}, B{e >= 4 ? q : -1, e - 4};
        double v[3];
        const bool w = contra2cart_bc_rule(g, m, nv, A, B, p, x[0], x[1], x[2], v);
        if (e == 0) {
          if (!w) break;
          if (n == 0) assigned = true;
          if (l[0] == 0.0 && l[1] == 0.0 && l[2] == 0.0) break;
          continue;
        }
        const double t = v[0] * l[0] + v[1] * l[1] + v[2] * l[2];
        if (e <= 3) a[e - 1] += t;
        else o[e - 4] += t;
      }
    }
  }
  if (!assigned) { a[0] += l3.x[q]; a[1] += l3.y[q]; a[2] += l3.z[q]; }
  l2.x[q] = a[0]; l2.y[q] = a[1]; l2.z[q] = a[2];
  if (o[0] != 0.0 || o[1] != 0.0 || o[2] != 0.0) { lo.x[q] += o[0]; lo.y[q] += o[1]; lo.z[q] += o[2]; }
}

// B^T, second half: the points the first half wrote take their new adjoints.
__global__ void k_c2c_bc_adjoint_commit(Grid g, const uint8_t *__restrict__ nv, CV3 l2, V3 l3) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= g.N) return;
  int i, j, k;
  dijk(g, q, i, j, k);
  if (!c2c_near(g, i, j, k) && !(nv[q] == 3 && !g.moving)) return;
  l3.x[q] = l2.x[q]; l3.y[q] = l2.y[q]; l3.z[q] = l2.z[q];
}

// I^T, per cell: w_d = 0.5 * sum_c K[c][d] / det * lu_c on the cells the interior kernel
// computes (K the cofactors of Cramer's rule: ucat_c = sum_d K[c][d] q_d / det, q_d the
// average of the two d-faces), 0 elsewhere; those cells' lu are consumed (the forward
// overwrites them).
__global__ void k_c2c_interior_adjoint(Grid g, CV3 csi, CV3 eta, CV3 zet, const uint8_t *__restrict__ nv, V3 lu,
                                       V3 w) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2 || nv[p] != 0) {
    w.x[p] = 0; w.y[p] = 0; w.z[p] = 0;
    return;
  }
  const double m00 = csi.x[p], m01 = csi.y[p], m02 = csi.z[p];
  const double m10 = eta.x[p], m11 = eta.y[p], m12 = eta.z[p];
  const double m20 = zet.x[p], m21 = zet.y[p], m22 = zet.z[p];
  const double det = m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) +
                     m02 * (m10 * m21 - m11 * m20);
  const double l0 = lu.x[p], l1 = lu.y[p], l2 = lu.z[p];
  w.x[p] = 0.5 * ((m11 * m22 - m12 * m21) * l0 - (m10 * m22 - m12 * m20) * l1 + (m10 * m21 - m11 * m20) * l2) / det;
  w.y[p] = 0.5 * (-(m01 * m22 - m02 * m21) * l0 + (m00 * m22 - m02 * m20) * l1 - (m00 * m21 - m01 * m20) * l2) / det;
  w.z[p] = 0.5 * ((m01 * m12 - m02 * m11) * l0 - (m00 * m12 - m02 * m10) * l1 + (m00 * m11 - m01 * m10) * l2) / det;
  lu.x[p] = 0; lu.y[p] = 0; lu.z[p] = 0;
}

// I^T, per face: the d-face f between cells f and f + d gathers both cells' w_d.
__global__ void k_c2c_face_gather(Grid g, CV3 w, V3 luc) {
  const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= g.N) return;
  int i, j, k;
  dijk(g, f, i, j, k);
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  const double ax = w.x[f] + (i + 1 < g.mx ? w.x[f + 1] : 0.0);
  const double ay = w.y[f] + (j + 1 < g.my ? w.y[f + sy] : 0.0);
  const double az = w.z[f] + (k + 1 < g.mz ? w.z[f + sz] : 0.0);
  if (ax != 0.0) luc.x[f] += ax;
  if (ay != 0.0) luc.y[f] += ay;
  if (az != 0.0) luc.z[f] += az;
}

// Affine boundary rules (a constant 2.0 in the ghost value) have no transpose of this form.
bool contra2cart_linear(const Grid &g) { return !(g.bc[3] == 2 || g.bc[2] == 12 || g.bc[3] == 12); }

// In place: (luc, lucat, luo) <- the transpose of contra2cart applied to them; tmp: three
// scratch arrays of N.
int contra2cart_adjoint(Ctx *c, V3 luc, V3 lucat, V3 luo, V3 tmp) {
  const Grid &g = c->g;
  int rc;
  if (!contra2cart_linear(g)) return set_err(c, VFS_ERR_INVALID, "contra2cart_adjoint: affine boundary rule");
  Metrics m = metrics(c);
  if ((rc = periodic_copy3_adjoint(c, lucat))) return rc;
  c->launches++, k_c2c_bc_adjoint<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, cv(lucat), tmp, luo);
  if ((rc = check_launch(c, "k_c2c_bc_adjoint"))) return rc;
  c->launches++, k_c2c_bc_adjoint_commit<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nv, cv(tmp), lucat);
  if ((rc = check_launch(c, "k_c2c_bc_adjoint_commit"))) return rc;
  if ((rc = periodic_copy3_adjoint(c, lucat))) return rc;
  c->launches++, k_c2c_interior_adjoint<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m.csi, m.eta, m.zet, c->nv,
                                                                                  lucat, tmp);
  if ((rc = check_launch(c, "k_c2c_interior_adjoint"))) return rc;
  c->launches++, k_c2c_face_gather<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, cv(tmp), luc);
  if ((rc = check_launch(c, "k_c2c_face_gather"))) return rc;
  return periodic_copy3_adjoint(c, luc);
}

// ------------------------------------------------------------------ Formfunction_2
// Face-centred velocity gradients in computational space with nvert-aware one-sided
// cross differences, solid = 0.1 (Compute_du_i/j/k, k-omega.c:48-300).
struct Grad9 { double dudc, dvdc, dwdc, dude, dvde, dwde, dudz, dvdz, dwdz; };

__device__ __forceinline__ void cross_diff(CV3 u, long long a0, long long a1, long long bp0,
                                           long long bp1, long long bm0, long long bm1,
                                           bool plus_solid, bool minus_solid, double *d) {
  // a0,a1: the two face cells; bp*/bm*: same cells shifted +/- in the cross direction
  if (plus_solid) {
    d[0] = (u.x[a1] + u.x[a0] - u.x[bm1] - u.x[bm0]) * 0.5;
    d[1] = (u.y[a1] + u.y[a0] - u.y[bm1] - u.y[bm0]) * 0.5;
    d[2] = (u.z[a1] + u.z[a0] - u.z[bm1] - u.z[bm0]) * 0.5;
  } else if (minus_solid) {
    d[0] = (u.x[bp1] + u.x[bp0] - u.x[a1] - u.x[a0]) * 0.5;
    d[1] = (u.y[bp1] + u.y[bp0] - u.y[a1] - u.y[a0]) * 0.5;
    d[2] = (u.z[bp1] + u.z[bp0] - u.z[a1] - u.z[a0]) * 0.5;
  } else {
    d[0] = (u.x[bp1] + u.x[bp0] - u.x[bm1] - u.x[bm0]) * 0.25;
    d[1] = (u.y[bp1] + u.y[bp0] - u.y[bm1] - u.y[bm0]) * 0.25;
    d[2] = (u.z[bp1] + u.z[bp0] - u.z[bm1] - u.z[bm0]) * 0.25;
  }
}

// QUICK flux next to an immersed boundary (momentum.c:734-755 and the j/k analogues):
// variant A when the lower cell is IB/solid, B when the upper cell is.
__device__ __forceinline__ double quick_a(double um, double up, double u0, double u1, double u2) {
  return um * (0.125 * (-u2 - 2. * u1 + 3. * u0) + u1) + up * (0.125 * (-u0 - 2. * u0 + 3. * u1) + u0);
}
__device__ __forceinline__ double quick_b(double um, double up, double um1, double u0, double u1) {
  return um * (0.125 * (-u1 - 2. * u1 + 3. * u0) + u1) + up * (0.125 * (-um1 - 2. * u0 + 3. * u1) + u0);
}

// Viscous face flux component (momentum.c:876-905): (g.du + r.metric) * ajc * nu.
__device__ __forceinline__ double visc_term(double g11, double g21, double g31, double dc, double de,
                                            double dz, double ra, double rb, double rc, double m0,
                                            double m1, double m2, double ajc, double nu) {
  return (g11 * dc + g21 * de + g31 * dz + ra * m0 + rb * m1 + rc * m2) * ajc * (nu);
}

struct FluxOut { double *div[3]; double *visc[3]; };

// Convective (d) and viscous (v) flux of one face of Formfunction_2, following the three
// face loops (momentum.c:671-1415): the i-face between (i,j,k) and (i+1,j,k), and the j
// and k analogues.
template <bool kReg = false>
__device__ __forceinline__ void flux_i(const Grid &g, const Metrics &m, CV3 uc, CV3 u,
                                      const uint8_t *__restrict__ nv, const double *__restrict__ nut, long long p,
                                      int i, int j, int k, double d[3], double v[3]) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const double nu = 1. / g.ren;
  const bool les = g.les != 0;
  (void)sx; (void)sy; (void)sz; (void)mx; (void)my; (void)mz;
  const double ajc = __ldcs(m.iaj + p);
  const double csi0 = __ldcs(m.icsi.x + p), csi1 = __ldcs(m.icsi.y + p), csi2 = __ldcs(m.icsi.z + p);
  const double eta0 = __ldcs(m.ieta.x + p), eta1 = __ldcs(m.ieta.y + p), eta2 = __ldcs(m.ieta.z + p);
  const double zet0 = __ldcs(m.izet.x + p), zet1 = __ldcs(m.izet.y + p), zet2 = __ldcs(m.izet.z + p);
  double dc[3], de[3], dz[3];
  dc[0] = u.x[p + sx] - u.x[p]; dc[1] = u.y[p + sx] - u.y[p]; dc[2] = u.z[p + sx] - u.z[p];
  cross_diff(u, p, p + sx, p + sy, p + sy + sx, p - sy, p - sy + sx,
             !kReg && (nv[p + sy] > 0 || nv[p + sy + sx] > 0),
             !kReg && (nv[p - sy] > 0 || nv[p - sy + sx] > 0), de);
  cross_diff(u, p, p + sx, p + sz, p + sz + sx, p - sz, p - sz + sx,
             !kReg && (nv[p + sz] > 0 || nv[p + sz + sx] > 0),
             !kReg && (nv[p - sz] > 0 || nv[p - sz + sx] > 0), dz);
  const double g11 = csi0 * csi0 + csi1 * csi1 + csi2 * csi2;
  const double g21 = eta0 * csi0 + eta1 * csi1 + eta2 * csi2;
  const double g31 = zet0 * csi0 + zet1 * csi1 + zet2 * csi2;
  const double r11 = dc[0] * csi0 + de[0] * eta0 + dz[0] * zet0;
  const double r21 = dc[1] * csi0 + de[1] * eta0 + dz[1] * zet0;
  const double r31 = dc[2] * csi0 + de[2] * eta0 + dz[2] * zet0;
  const double r12 = dc[0] * csi1 + de[0] * eta1 + dz[0] * zet1;
  const double r22 = dc[1] * csi1 + de[1] * eta1 + dz[1] * zet1;
  const double r32 = dc[2] * csi1 + de[2] * eta1 + dz[2] * zet1;
  const double r13 = dc[0] * csi2 + de[0] * eta2 + dz[0] * zet2;
  const double r23 = dc[1] * csi2 + de[1] * eta2 + dz[1] * zet2;
  const double r33 = dc[2] * csi2 + de[2] * eta2 + dz[2] * zet2;
  int iL = i - 1, iR = i + 2;
  if (!kReg && (i == 0 || i == mx - 2)) {
    if (g.iper) iL = mx - 3, iR = 2;
    else iL = i, iR = i + 1;
  } else if (!kReg && nv[p - 1] + nv[p + 2] > 0) iL = i, iR = i + 1;
  double ucon = uc.x[p];
  if (!kReg && g.iper && (i == 0 || i == mx - 2)) ucon = uc.x[p - i + (mx - 2)];
  const double up = -0.5 * (ucon + fabs(ucon));
  const double um = -0.5 * (ucon - fabs(ucon));
  const long long pL = p - i + iL, pR = p - i + iR;
  if (!kReg && g.immersed && i != mx - 2 && nv[p] > 0) {
    d[0] = quick_a(um, up, u.x[p], u.x[p + 1], u.x[p + 2]);
    d[1] = quick_a(um, up, u.y[p], u.y[p + 1], u.y[p + 2]);
    d[2] = quick_a(um, up, u.z[p], u.z[p + 1], u.z[p + 2]);
  } else if (!kReg && g.immersed && i != 0 && nv[p + 1] > 0) {
    d[0] = quick_b(um, up, u.x[p - 1], u.x[p], u.x[p + 1]);
    d[1] = quick_b(um, up, u.y[p - 1], u.y[p], u.y[p + 1]);
    d[2] = quick_b(um, up, u.z[p - 1], u.z[p], u.z[p + 1]);
  } else {
    const double cu = uc.x[p];
    d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + 1] - u.x[pR]);
    d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + 1] - u.y[pR]);
    d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + 1] - u.z[pR]);
  }
  if (!kReg && nv[p] + nv[p + 1] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
  v[0] = 0; v[1] = 0; v[2] = 0;
  if (les) {
    double nut_f;
    if (!kReg && ((i == 0 && !g.iper) || nv[p] > 0)) nut_f = nut[p + 1];
    else if (!kReg && ((i == mx - 2 && !g.iper) || nv[p + 1] > 0)) nut_f = nut[p];
    else nut_f = 0.5 * (nut[p] + nut[p + 1]);
    v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, csi0, csi1, csi2, ajc, nut_f);
    v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, csi0, csi1, csi2, ajc, nut_f);
    v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, csi0, csi1, csi2, ajc, nut_f);
  }
  v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, csi0, csi1, csi2, ajc, nu);
  v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, csi0, csi1, csi2, ajc, nu);
  v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, csi0, csi1, csi2, ajc, nu);
}

template <bool kReg = false>
__device__ __forceinline__ void flux_j(const Grid &g, const Metrics &m, CV3 uc, CV3 u,
                                      const uint8_t *__restrict__ nv, const double *__restrict__ nut, long long p,
                                      int i, int j, int k, double d[3], double v[3]) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const double nu = 1. / g.ren;
  const bool les = g.les != 0;
  (void)sx; (void)sy; (void)sz; (void)mx; (void)my; (void)mz;
  const double ajc = __ldcs(m.jaj + p);
  const double csi0 = __ldcs(m.jcsi.x + p), csi1 = __ldcs(m.jcsi.y + p), csi2 = __ldcs(m.jcsi.z + p);
  const double eta0 = __ldcs(m.jeta.x + p), eta1 = __ldcs(m.jeta.y + p), eta2 = __ldcs(m.jeta.z + p);
  const double zet0 = __ldcs(m.jzet.x + p), zet1 = __ldcs(m.jzet.y + p), zet2 = __ldcs(m.jzet.z + p);
  double dc[3], de[3], dz[3];
  cross_diff(u, p, p + sy, p + sx, p + sy + sx, p - sx, p + sy - sx,
             !kReg && (nv[p + sx] > 0 || nv[p + sy + sx] > 0),
             !kReg && (nv[p - sx] > 0 || nv[p + sy - sx] > 0), dc);
  de[0] = u.x[p + sy] - u.x[p]; de[1] = u.y[p + sy] - u.y[p]; de[2] = u.z[p + sy] - u.z[p];
  cross_diff(u, p, p + sy, p + sz, p + sz + sy, p - sz, p - sz + sy,
             !kReg && (nv[p + sz] > 0 || nv[p + sz + sy] > 0),
             !kReg && (nv[p - sz] > 0 || nv[p - sz + sy] > 0), dz);
  const double g11 = csi0 * eta0 + csi1 * eta1 + csi2 * eta2;
  const double g21 = eta0 * eta0 + eta1 * eta1 + eta2 * eta2;
  const double g31 = zet0 * eta0 + zet1 * eta1 + zet2 * eta2;
  const double r11 = dc[0] * csi0 + de[0] * eta0 + dz[0] * zet0;
  const double r21 = dc[1] * csi0 + de[1] * eta0 + dz[1] * zet0;
  const double r31 = dc[2] * csi0 + de[2] * eta0 + dz[2] * zet0;
  const double r12 = dc[0] * csi1 + de[0] * eta1 + dz[0] * zet1;
  const double r22 = dc[1] * csi1 + de[1] * eta1 + dz[1] * zet1;
  const double r32 = dc[2] * csi1 + de[2] * eta1 + dz[2] * zet1;
  const double r13 = dc[0] * csi2 + de[0] * eta2 + dz[0] * zet2;
  const double r23 = dc[1] * csi2 + de[1] * eta2 + dz[1] * zet2;
  const double r33 = dc[2] * csi2 + de[2] * eta2 + dz[2] * zet2;
  int jL = j - 1, jR = j + 2;
  if (!kReg && (j == 0 || j == my - 2)) {
    if (g.jper) jL = my - 3, jR = 2;
    else jL = j, jR = j + 1;
  } else if (!kReg && nv[p - sy] + nv[p + 2 * sy] > 0) jL = j, jR = j + 1;
  double ucon = uc.y[p];
  if (!kReg && g.jper && (j == 0 || j == my - 2)) ucon = uc.y[p + (long long)(my - 2 - j) * sy];
  const double up = -0.5 * (ucon + fabs(ucon));
  const double um = -0.5 * (ucon - fabs(ucon));
  const long long pL = p + (long long)(jL - j) * sy, pR = p + (long long)(jR - j) * sy;
  if (!kReg && g.immersed && j != my - 2 && nv[p] > 0) {
    d[0] = quick_a(um, up, u.x[p], u.x[p + sy], u.x[p + 2 * sy]);
    d[1] = quick_a(um, up, u.y[p], u.y[p + sy], u.y[p + 2 * sy]);
    d[2] = quick_a(um, up, u.z[p], u.z[p + sy], u.z[p + 2 * sy]);
  } else if (!kReg && g.immersed && j != 0 && nv[p + sy] > 0) {
    d[0] = quick_b(um, up, u.x[p - sy], u.x[p], u.x[p + sy]);
    d[1] = quick_b(um, up, u.y[p - sy], u.y[p], u.y[p + sy]);
    d[2] = quick_b(um, up, u.z[p - sy], u.z[p], u.z[p + sy]);
  } else {
    const double cu = uc.y[p];
    d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + sy] - u.x[pR]);
    d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + sy] - u.y[pR]);
    d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + sy] - u.z[pR]);
  }
  if (!kReg && nv[p] + nv[p + sy] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
  v[0] = 0; v[1] = 0; v[2] = 0;
  if (les) {
    double nut_f;
    if (!kReg && ((j == 0 && !g.jper) || nv[p] > 0)) nut_f = nut[p + sy];
    else if (!kReg && ((j == my - 2 && !g.jper) || nv[p + sy] > 0)) nut_f = nut[p];
    else nut_f = 0.5 * (nut[p] + nut[p + sy]);
    v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, eta0, eta1, eta2, ajc, nut_f);
    v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, eta0, eta1, eta2, ajc, nut_f);
    v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, eta0, eta1, eta2, ajc, nut_f);
  }
  v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, eta0, eta1, eta2, ajc, nu);
  v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, eta0, eta1, eta2, ajc, nu);
  v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, eta0, eta1, eta2, ajc, nu);
}

template <bool kReg = false>
__device__ __forceinline__ void flux_k(const Grid &g, const Metrics &m, CV3 uc, CV3 u,
                                      const uint8_t *__restrict__ nv, const double *__restrict__ nut, long long p,
                                      int i, int j, int k, double d[3], double v[3]) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const double nu = 1. / g.ren;
  const bool les = g.les != 0;
  (void)sx; (void)sy; (void)sz; (void)mx; (void)my; (void)mz;
  const double ajc = __ldcs(m.kaj + p);
  const double csi0 = __ldcs(m.kcsi.x + p), csi1 = __ldcs(m.kcsi.y + p), csi2 = __ldcs(m.kcsi.z + p);
  const double eta0 = __ldcs(m.keta.x + p), eta1 = __ldcs(m.keta.y + p), eta2 = __ldcs(m.keta.z + p);
  const double zet0 = __ldcs(m.kzet.x + p), zet1 = __ldcs(m.kzet.y + p), zet2 = __ldcs(m.kzet.z + p);
  double dc[3], de[3], dz[3];
  cross_diff(u, p, p + sz, p + sx, p + sz + sx, p - sx, p + sz - sx,
             !kReg && (nv[p + sx] > 0 || nv[p + sz + sx] > 0),
             !kReg && (nv[p - sx] > 0 || nv[p + sz - sx] > 0), dc);
  cross_diff(u, p, p + sz, p + sy, p + sz + sy, p - sy, p + sz - sy,
             !kReg && (nv[p + sy] > 0 || nv[p + sz + sy] > 0),
             !kReg && (nv[p - sy] > 0 || nv[p + sz - sy] > 0), de);
  dz[0] = u.x[p + sz] - u.x[p]; dz[1] = u.y[p + sz] - u.y[p]; dz[2] = u.z[p + sz] - u.z[p];
  const double g11 = csi0 * zet0 + csi1 * zet1 + csi2 * zet2;
  const double g21 = eta0 * zet0 + eta1 * zet1 + eta2 * zet2;
  const double g31 = zet0 * zet0 + zet1 * zet1 + zet2 * zet2;
  const double r11 = dc[0] * csi0 + de[0] * eta0 + dz[0] * zet0;
  const double r21 = dc[1] * csi0 + de[1] * eta0 + dz[1] * zet0;
  const double r31 = dc[2] * csi0 + de[2] * eta0 + dz[2] * zet0;
  const double r12 = dc[0] * csi1 + de[0] * eta1 + dz[0] * zet1;
  const double r22 = dc[1] * csi1 + de[1] * eta1 + dz[1] * zet1;
  const double r32 = dc[2] * csi1 + de[2] * eta1 + dz[2] * zet1;
  const double r13 = dc[0] * csi2 + de[0] * eta2 + dz[0] * zet2;
  const double r23 = dc[1] * csi2 + de[1] * eta2 + dz[1] * zet2;
  const double r33 = dc[2] * csi2 + de[2] * eta2 + dz[2] * zet2;
  int kL = k - 1, kR = k + 2;
  if (!kReg && (k == 0 || k == mz - 2)) {
    if (g.kper) kL = mz - 3, kR = 2;
    else kL = k, kR = k + 1;
  } else if (!kReg && nv[p - sz] + nv[p + 2 * sz] > 0) kL = k, kR = k + 1;
  double ucon = uc.z[p];
  if (!kReg && g.kper && (k == 0 || k == mz - 2)) ucon = uc.z[p + (long long)(mz - 2 - k) * sz];
  if (!kReg && k == mz - 2 && g.bc[5] == 4 && nv[p] == 0) ucon = uc.z[p - sz];
  const double up = -0.5 * (ucon + fabs(ucon));
  const double um = -0.5 * (ucon - fabs(ucon));
  const long long pL = p + (long long)(kL - k) * sz, pR = p + (long long)(kR - k) * sz;
  if (!kReg && g.immersed && k != mz - 2 && nv[p] > 0) {
    d[0] = quick_a(um, up, u.x[p], u.x[p + sz], u.x[p + 2 * sz]);
    d[1] = quick_a(um, up, u.y[p], u.y[p + sz], u.y[p + 2 * sz]);
    d[2] = quick_a(um, up, u.z[p], u.z[p + sz], u.z[p + 2 * sz]);
  } else if (!kReg && g.immersed && k != 0 && nv[p + sz] > 0) {
    d[0] = quick_b(um, up, u.x[p - sz], u.x[p], u.x[p + sz]);
    d[1] = quick_b(um, up, u.y[p - sz], u.y[p], u.y[p + sz]);
    d[2] = quick_b(um, up, u.z[p - sz], u.z[p], u.z[p + sz]);
  } else {
    const double cu = uc.z[p];
    d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + sz] - u.x[pR]);
    d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + sz] - u.y[pR]);
    d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + sz] - u.z[pR]);
  }
  if (!kReg && nv[p] + nv[p + sz] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
  v[0] = 0; v[1] = 0; v[2] = 0;
  if (les) {
    double nut_f;
    if (!kReg && ((k == 0 && !g.kper) || nv[p] > 0)) nut_f = nut[p + sz];
    else if (!kReg && ((k == mz - 2 && !g.kper) || nv[p + sz] > 0)) nut_f = nut[p];
    else nut_f = 0.5 * (nut[p] + nut[p + sz]);
    v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, zet0, zet1, zet2, ajc, nut_f);
    v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, zet0, zet1, zet2, ajc, nut_f);
    v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, zet0, zet1, zet2, ajc, nut_f);
  }
  v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, zet0, zet1, zet2, ajc, nu);
  v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, zet0, zet1, zet2, ajc, nu);
  v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, zet0, zet1, zet2, ajc, nu);
}

// True when every nvert the three face fluxes of point p read is 0 (fluid), so that no
// one-sided, QUICK or masked branch applies.
__device__ __forceinline__ bool regular_faces(const uint8_t *__restrict__ nv, long long p, long long sy, long long sz) {
  const int s = nv[p] + nv[p + 1] + nv[p - 1] + nv[p + 2] + nv[p + sy] + nv[p - sy] + nv[p + 2 * sy] + nv[p + sz] +
                nv[p - sz] + nv[p + 2 * sz] + nv[p + sy + 1] + nv[p - sy + 1] + nv[p + sz + 1] + nv[p - sz + 1] +
                nv[p + sy - 1] + nv[p + sz - 1] + nv[p + sz + sy] + nv[p + sz - sy] + nv[p - sz + sy];
  return s == 0;
}

// One thread per DA point (i,j,k) with i<mx-1, j<my-1, k<mz-1: computes the fluxes of
// its i-face (if j,k >= 1), j-face (if i,k >= 1) and k-face (if i,j >= 1), following
// the three face loops of Formfunction_2 (momentum.c:671-1415).
// Points whose whole stencil is regular fluid interior take a branch-free path with
// constant offsets (regular_faces); the rest run the general form.
// Launch shape: VFS_FF_THREADS threads per block, at least VFS_FF_MINB blocks per SM (the
// register cap that follows from it sets the occupancy of this latency-bound kernel:
// 5 blocks cap it at 96 registers, which at 256 x 192 x 256 runs Formfunction_2 in
// 2.20 ms against 2.50 ms uncapped at 154 registers and 2.45 ms at 64).
#ifndef VFS_FF_THREADS
#define VFS_FF_THREADS 128
#endif
#ifndef VFS_FF_MINB
#define VFS_FF_MINB 5
#endif
__device__ __forceinline__ void face_flux_point(const Grid &g, const Metrics &m, CV3 uc, CV3 u,
                                                const uint8_t *__restrict__ nv, const double *__restrict__ nut,
                                                long long p, const FluxOut &f1, const FluxOut &f2, const FluxOut &f3) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i == mx - 1 || j == my - 1 || k == mz - 1) return;
  double d[3], v[3];
  const long long sy = mx, sz = (long long)mx * my;
  if (i >= 2 && i <= mx - 3 && j >= 2 && j <= my - 3 && k >= 2 && k <= mz - 3 &&
      regular_faces(nv, p, sy, sz)) {
    // Away from walls, periodic images, the outlet plane and solid cells every branch of
    // the three face fluxes takes its interior form: the same arithmetic with constant offsets.
    flux_i<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f1.div[0][p] = d[0]; f1.div[1][p] = d[1]; f1.div[2][p] = d[2];
    f1.visc[0][p] = v[0]; f1.visc[1][p] = v[1]; f1.visc[2][p] = v[2];
    flux_j<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f2.div[0][p] = d[0]; f2.div[1][p] = d[1]; f2.div[2][p] = d[2];
    f2.visc[0][p] = v[0]; f2.visc[1][p] = v[1]; f2.visc[2][p] = v[2];
    flux_k<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f3.div[0][p] = d[0]; f3.div[1][p] = d[1]; f3.div[2][p] = d[2];
    f3.visc[0][p] = v[0]; f3.visc[1][p] = v[1]; f3.visc[2][p] = v[2];
    return;
  }
  if (j != 0 && k != 0) {
    flux_i(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f1.div[0][p] = d[0]; f1.div[1][p] = d[1]; f1.div[2][p] = d[2];
    f1.visc[0][p] = v[0]; f1.visc[1][p] = v[1]; f1.visc[2][p] = v[2];
  }
  if (i != 0 && k != 0) {
    flux_j(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f2.div[0][p] = d[0]; f2.div[1][p] = d[1]; f2.div[2][p] = d[2];
    f2.visc[0][p] = v[0]; f2.visc[1][p] = v[1]; f2.visc[2][p] = v[2];
  }
  if (i != 0 && j != 0) {
    flux_k(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    f3.div[0][p] = d[0]; f3.div[1][p] = d[1]; f3.div[2][p] = d[2];
    f3.visc[0][p] = v[0]; f3.visc[1][p] = v[1]; f3.visc[2][p] = v[2];
  }
}

__global__ void __launch_bounds__(VFS_FF_THREADS, VFS_FF_MINB) k_face_flux(Grid g, Metrics m, CV3 uc, CV3 u,
                                                                           const uint8_t *__restrict__ nv,
                                                                           const double *__restrict__ nut, FluxOut f1,
                                                                           FluxOut f2, FluxOut f3) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  face_flux_point(g, m, uc, u, nv, nut, p, f1, f2, f3);
}

// Fp at interior cells: 4th-order divergence correction 9/8*div - 1/8*wide/denom plus the
// viscous divergence (momentum.c:1508-1640).  Face fluxes on a periodic ghost plane are
// read from their periodic image (momentum.c:1456-1500 copy loop).
struct FluxIn { const double *div[3]; const double *visc[3]; };

// Unwrapped face index u (u = cell + offset) -> the face whose flux the reference reads:
// on a periodic direction the faces 0 and m-1 and beyond are images of interior faces
// (the copy loop of momentum.c:1456-1500); m = number of points in the direction.
__device__ __forceinline__ int face_image(int u, int m, int per) {
  if (per) {
    if (u <= 0) return u + (m - 2);
    if (u >= m - 1) return u - (m - 2);
  }
  return u;
}

// Stencil offsets of the wide (4th-order) difference of Fp along one direction at cell
// index c (1..m-2): faces c+oR and c+oL, divided by den (momentum.c:1508-1640).
__device__ __forceinline__ void fp_offsets(int c, int m, int per, int nvsum, int &oR, int &oL, double &den) {
  oR = 1; oL = -2; den = 3.;
  if (!per && (c == 1 || c == 2 || c == m - 3 || c == m - 2)) { oR = 0; oL = -1; den = 1.; }
  if (nvsum > 0) { oR = 0; oL = -1; den = 1.; }
}

// Fp at interior cell (i,j,k): 9/8 div - 1/8 wide / den plus the viscous divergence.
// F supplies face fluxes by direction, component and offset from the cell:
// F.d(dir, comp, off) (off in -2..1) and F.v(dir, comp, off) (off in -1..0).
template <class F>
__device__ __forceinline__ void fp_cell(const Grid &g, const uint8_t *__restrict__ nv, long long p, int i, int j,
                                        int k, const F &f, double fpv[3]) {
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  int oiR, oiL, ojR, ojL, okR, okL;
  double di, dj, dk;
  fp_offsets(i, g.mx, g.iper, nv[p - 1] + nv[p] + nv[p + 1], oiR, oiL, di);
  fp_offsets(j, g.my, g.jper, nv[p - sy] + nv[p] + nv[p + sy], ojR, ojL, dj);
  fp_offsets(k, g.mz, g.kper, nv[p - sz] + nv[p] + nv[p + sz], okR, okL, dk);
  const double ai = 1. / di, aj_ = 1. / dj, ak = 1. / dk;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double div = (f.d(0, c, 0) - f.d(0, c, -1) + f.d(1, c, 0) - f.d(1, c, -1) + f.d(2, c, 0) - f.d(2, c, -1));
    double acc = 0;
    acc += (f.d(0, c, oiR) - f.d(0, c, oiL)) * ai;
    acc += (f.d(1, c, ojR) - f.d(1, c, ojL)) * aj_;
    acc += (f.d(2, c, okR) - f.d(2, c, okL)) * ak;
    double v = 9. / 8. * div + -1. / 8. * acc;
    v += (f.v(0, c, 0) - f.v(0, c, -1) + f.v(1, c, 0) - f.v(1, c, -1) + f.v(2, c, 0) - f.v(2, c, -1)) / 1.0;
    fpv[c] = v;
  }
}

// Face fluxes from the global face-flux arrays.
struct GlobalFaces {
  const Grid *g;
  FluxIn f1, f2, f3;
  long long rowi, rowj, rowk;
  int i, j, k;
  __device__ __forceinline__ long long at(int dir, int off) const {
    if (dir == 0) return rowi + face_image(i + off, g->mx, g->iper);
    if (dir == 1) return rowj + (long long)face_image(j + off, g->my, g->jper) * g->mx;
    return rowk + (long long)face_image(k + off, g->mz, g->kper) * ((long long)g->mx * g->my);
  }
  __device__ __forceinline__ double d(int dir, int c, int off) const {
    const FluxIn &f = dir == 0 ? f1 : (dir == 1 ? f2 : f3);
    return f.div[c][at(dir, off)];
  }
  __device__ __forceinline__ double v(int dir, int c, int off) const {
    const FluxIn &f = dir == 0 ? f1 : (dir == 1 ? f2 : f3);
    return f.visc[c][at(dir, off)];
  }
};

// Interior cell p away from walls, periodic images and solid cells: every wide difference
// of Fp is the 4th-order one (faces c+1 and c-2 over 3) and every face is its own.
__device__ __forceinline__ bool fp_regular(const Grid &g, const uint8_t *__restrict__ nv, long long p, int i, int j,
                                           int k) {
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  return i >= 3 && i <= g.mx - 4 && j >= 3 && j <= g.my - 4 && k >= 3 && k <= g.mz - 4 &&
         nv[p - 1] + nv[p] + nv[p + 1] + nv[p - sy] + nv[p + sy] + nv[p - sz] + nv[p + sz] == 0;
}

// fp_cell at a regular cell: constant offsets, the same arithmetic in the same order.
__device__ __forceinline__ void fp_cell_regular(const Grid &g, const FluxIn &f1, const FluxIn &f2, const FluxIn &f3,
                                                long long p, double fpv[3]) {
  const long long st[3] = {1, g.mx, (long long)g.mx * g.my};
  const FluxIn *fl[3] = {&f1, &f2, &f3};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    auto D = [&](int dir, int off) { return fl[dir]->div[c][p + off * st[dir]]; };
    auto Vv = [&](int dir, int off) { return fl[dir]->visc[c][p + off * st[dir]]; };
    const double div = (D(0, 0) - D(0, -1) + D(1, 0) - D(1, -1) + D(2, 0) - D(2, -1));
    double acc = 0;
    acc += (D(0, 1) - D(0, -2)) * (1. / 3.);
    acc += (D(1, 1) - D(1, -2)) * (1. / 3.);
    acc += (D(2, 1) - D(2, -2)) * (1. / 3.);
    double v = 9. / 8. * div + -1. / 8. * acc;
    v += (Vv(0, 0) - Vv(0, -1) + Vv(1, 0) - Vv(1, -1) + Vv(2, 0) - Vv(2, -1)) / 1.0;
    fpv[c] = v;
  }
}

// Fp at DA point p (nothing outside the interior cells).
__device__ __forceinline__ void fp_point(const Grid &g, const FluxIn &f1, const FluxIn &f2, const FluxIn &f3,
                                         const uint8_t *__restrict__ nv, long long p, double *fpx, double *fpy,
                                         double *fpz) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) return;
  double fpv[3];
  if (fp_regular(g, nv, p, i, j, k)) {
    fp_cell_regular(g, f1, f2, f3, p, fpv);
  } else {
    GlobalFaces F;
    F.g = &g; F.f1 = f1; F.f2 = f2; F.f3 = f3;
    F.rowi = p - i; F.rowj = p - (long long)j * mx; F.rowk = p - (long long)k * mx * my;
    F.i = i; F.j = j; F.k = k;
    fp_cell(g, nv, p, i, j, k, F, fpv);
  }
  fpx[p] = fpv[0]; fpy[p] = fpv[1]; fpz[p] = fpv[2];
}

// Four resident blocks per SM (64 registers): 0.56 ms at 256 x 192 x 256 against 0.70 ms
// uncapped (116 registers) and slower again at five or six (spills).
#ifndef VFS_FP_MINB
#define VFS_FP_MINB 4
#endif
__global__ void __launch_bounds__(256, VFS_FP_MINB) k_fp(Grid g, FluxIn f1, FluxIn f2, FluxIn f3,
                                                         const uint8_t *__restrict__ nv, double *fpx, double *fpy,
                                                         double *fpz) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  fp_point(g, f1, f2, f3, nv, p, fpx, fpy, fpz);
}

// Contravariant projection of Fp onto the faces, scale, masks and the boundary zeroing
// of the right-hand side (momentum.c:1686-1900).  In RK mode the stage update
// Ucont = pUcont + a*(RHS - dP) (rhs.c:1644-1650) is fused into the epilogue and the
// accumulation starts from a zeroed RHS (VecSet(Rhs,0) at rhs.c:1643).
// Right-hand side at one point from Fp, accessed as F.fp(w, c) with w = 0 the cell and
// w = 1, 2, 3 its +i, +j, +k neighbour (the periodic image on the last interior plane);
// ghost points get zero.  With rk set, the stage update is applied as well.
template <class FPA>
__device__ __forceinline__ void rhs_point(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv,
                                          long long p, int i, int j, int k, bool ghost, const FPA &f, double scale,
                                          V3 rhs, int rk, double a, CV3 dP, CV3 pu, V3 ucont) {
  const int mx = g.mx, my = g.my, mz = g.mz;
  double r[3];
  if (ghost) {
    r[0] = r[1] = r[2] = 0;
  } else {
    const long long sy = mx, sz = (long long)mx * my;
    if (rk) { r[0] = 0; r[1] = 0; r[2] = 0; }
    else { r[0] = rhs.x[p]; r[1] = rhs.y[p]; r[2] = rhs.z[p]; }
    r[0] += scale * (0.5 * (m.csi.x[p] * f.fp(0, 0) + m.csi.y[p] * f.fp(0, 1) + m.csi.z[p] * f.fp(0, 2)) +
                     0.5 * (m.csi.x[p + 1] * f.fp(1, 0) + m.csi.y[p + 1] * f.fp(1, 1) + m.csi.z[p + 1] * f.fp(1, 2))) *
            m.iaj[p];
    r[1] += scale * (0.5 * (m.eta.x[p] * f.fp(0, 0) + m.eta.y[p] * f.fp(0, 1) + m.eta.z[p] * f.fp(0, 2)) +
                     0.5 * (m.eta.x[p + sy] * f.fp(2, 0) + m.eta.y[p + sy] * f.fp(2, 1) + m.eta.z[p + sy] * f.fp(2, 2))) *
            m.jaj[p];
    r[2] += scale * (0.5 * (m.zet.x[p] * f.fp(0, 0) + m.zet.y[p] * f.fp(0, 1) + m.zet.z[p] * f.fp(0, 2)) +
                     0.5 * (m.zet.x[p + sz] * f.fp(3, 0) + m.zet.y[p + sz] * f.fp(3, 1) + m.zet.z[p + sz] * f.fp(3, 2))) *
            m.kaj[p];
    if (nv[p] + nv[p + 1] > 0 || (!g.iper && i == mx - 2)) r[0] = 0;
    if (nv[p] + nv[p + sy] > 0 || (!g.jper && j == my - 2)) r[1] = 0;
    if (nv[p] + nv[p + sz] > 0 || (!g.kper && k == mz - 2)) r[2] = 0;
  }
  if (!rk) {
    rhs.x[p] = r[0]; rhs.y[p] = r[1]; rhs.z[p] = r[2];
  } else {
    r[0] = r[0] + -1 * dP.x[p];
    r[1] = r[1] + -1 * dP.y[p];
    r[2] = r[2] + -1 * dP.z[p];
    rhs.x[p] = r[0]; rhs.y[p] = r[1]; rhs.z[p] = r[2];
    if (ucont.x) {
      ucont.x[p] = a * r[0] + pu.x[p];
      ucont.y[p] = a * r[1] + pu.y[p];
      ucont.z[p] = a * r[2] + pu.z[p];
    }
  }
}

// The stage update Ucont = pUcont + a * RHS (RHS already holding -dP) over every point.
__global__ void k_rk_update(long long n, double a, CV3 rhs, CV3 pu, V3 ucont) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  ucont.x[p] = a * rhs.x[p] + pu.x[p];
  ucont.y[p] = a * rhs.y[p] + pu.y[p];
  ucont.z[p] = a * rhs.z[p] + pu.z[p];
}

struct GlobalFp {
  const double *f[3];
  long long q[4];
  __device__ __forceinline__ double fp(int w, int c) const { return f[c][q[w]]; }
};

// Contravariant projection of Fp onto the faces, scale, masks and the boundary zeroing
// of the right-hand side (momentum.c:1686-1900).  In RK mode the stage update
// Ucont = pUcont + a*(RHS - dP) (rhs.c:1644-1650) is fused into the epilogue and the
// accumulation starts from a zeroed RHS (VecSet(Rhs,0) at rhs.c:1643).
__global__ void k_rhs(Grid g, Metrics m, const uint8_t *__restrict__ nv, const double *__restrict__ fpx,
                      const double *__restrict__ fpy, const double *__restrict__ fpz, double scale,
                      V3 rhs, int rk, double a, CV3 dP, CV3 pu, V3 ucont) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const bool ghost = i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1;
  const long long sy = mx, sz = (long long)mx * my;
  GlobalFp F;
  F.f[0] = fpx; F.f[1] = fpy; F.f[2] = fpz;
  // Fp on the periodic ghost plane is the image of the first interior plane
  F.q[0] = p;
  F.q[1] = (g.iper && i == mx - 2) ? p - i + 1 : p + 1;
  F.q[2] = (g.jper && j == my - 2) ? p - (long long)j * sy + sy : p + sy;
  F.q[3] = (g.kper && k == mz - 2) ? p - (long long)k * sz + sz : p + sz;
  rhs_point(g, m, nv, p, i, j, k, ghost, F, scale, rhs, rk, a, dP, pu, ucont);
}

// ------------------------------------------------------------------ Formfunction_2, one pass
// Image of a cell index (1..m-2 unchanged; m-1 -> 1 on a periodic direction), -1 if none.
__device__ __forceinline__ int cell_image(int u, int m, int per) {
  if (u >= 1 && u <= m - 2) return u;
  if (per && u == m - 1) return 1;
  return -1;
}
// Image of a face index, -1 if the face does not exist.
__device__ __forceinline__ int face_image_or_none(int u, int m, int per) {
  const int f = face_image(u, m, per);
  return (f >= 0 && f <= m - 2) ? f : -1;
}

static FluxOut flux_out(Ctx *c, int d) {
  FluxOut f;
  for (int q = 0; q < 3; q++) { f.div[q] = c->div[d][q]; f.visc[q] = c->visc[d][q]; }
  return f;
}
static FluxIn flux_in(Ctx *c, int d) {
  FluxIn f;
  for (int q = 0; q < 3; q++) { f.div[q] = c->div[d][q]; f.visc[q] = c->visc[d][q]; }
  return f;
}

void launch_fp(Ctx *c);

// The 18 face-flux arrays of Formfunction_2 (one launch for the three face directions;
// one launch per direction measured 30 % slower on the B200).
static int face_fluxes(Ctx *c) {
  const Grid &g = c->g;
  Metrics m = metrics(c);
  CV3 uc = cv(field3(c, VFS_UCONT)), u = cv(field3(c, VFS_UCAT));
  const unsigned nb = nblocks(g.N, VFS_FF_THREADS);
  c->launches++, k_face_flux<<<nb, VFS_FF_THREADS, 0, c->stream>>>(g, m, uc, u, c->nv, c->f[VFS_NU_T][0], flux_out(c, 0),
                                                    flux_out(c, 1), flux_out(c, 2));
  return check_launch(c, "k_face_flux");
}

// Formfunction_2 as three kernels: face fluxes (written to 18 arrays), Fp, right-hand
// side (with the RK stage update in place).  Same results as the one-pass form; kept as
// the reference form for the kernel-level comparison and the diagnostics entry point.
int formfunction2_split(Ctx *c, double scale, bool rk_stage, double rk_coeff) {
  const Grid &g = c->g;
  int rc;
  V3 uc = field3(c, VFS_UCONT);
  if ((rc = periodic_copy3(c, uc))) return rc;
  Metrics m = metrics(c);
  if ((rc = face_fluxes(c))) return rc;
  launch_fp(c);
  if ((rc = check_launch(c, "k_fp"))) return rc;
  V3 pu{c->pucont[0], c->pucont[1], c->pucont[2]};
  c->launches++, k_rhs<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, c->fp[0], c->fp[1], c->fp[2], scale,
                                                 field3(c, VFS_RHS), rk_stage ? 1 : 0, rk_coeff,
                                                 cv(field3(c, VFS_DP)), cv(pu), uc);
  return check_launch(c, "k_rhs");
}

// One-pass Formfunction_2: face fluxes, Fp and the right-hand side (with the RK stage
// update) of a tile of cells in one kernel, with no face-flux array in HBM.
//
// A thread block of NW warps owns a strip of planes kb .. ke-1 of an (i, j) tile: lane l
// of warp w is the column (i0 - 2 + l, j0 + w), and the block marches through the planes
// in k.  Per plane kc every thread computes the fluxes of three faces of its column: the
// i-face and j-face of plane kc and the k-face of plane kc+1 (the reference's three face
// loops, momentum.c:671-1415, through the same flux_i/j/k code as the split form).  Then
//  * the four i-faces Fp needs (offsets -2..1) come from the neighbouring lanes (warp
//    shuffles), so a warp produces Fp for its lanes 2..30 and the right-hand side for
//    lanes 2..29 (28 columns; neighbouring tiles overlap by four lanes);
//  * the j-faces go through shared memory: each warp writes its row's, warps 0-2 also
//    compute rows j0-2, j0-1 and j0+NW, and after one block barrier every row reads the
//    four faces around it; rows j0 .. j0+NW-2 produce the right-hand side, row j0+NW-1
//    only its Fp (the +j neighbour of the row below);
//  * the k-faces stay in registers as a ring over planes kc-2 .. kc+1 (each k-face is
//    computed once per column).
// The contravariant projection of the right-hand side at a cell (momentum.c:1686-1900)
// reads csi.Fp, eta.Fp and zet.Fp of the cell and of its +i, +j and +k neighbours; each
// thread forms the three products once for its own cell (at plane kc, with the metrics of
// its own DA point: on a periodic ghost plane the reference pairs the ghost's metric
// with the Fp of the periodic image) and the right-hand side of plane kc-1 takes them
// from the lane to the right (shuffle), the row above (shared memory, previous plane)
// and its own registers.  Every expression is the split form's, in the same order, so
// the results are identical bit for bit.
//
// In RK mode the stage update Ucont' = pUcont + a (RHS - dP) is written to `out` (not in
// place: neighbouring tiles still read Ucont in their halos); the caller swaps the two
// arrays.  Ghost points of the DA are written by k_ff2_ghosts.
constexpr int kMarchLanes = 32;
constexpr int kMarchOut = 28;  // right-hand-side columns per warp

template <int NW>
struct MarchSmem {
  double jf[2][NW + 3][6][kMarchLanes];      // j-face d(3), v(3) of rows j0-2 .. j0+NW, two planes
  double fi[NW][6][kMarchLanes + 3];         // i-face d(3), v(3) of each row, lanes at +2
  double ay[2][NW][kMarchLanes];             // eta.Fp of rows j0 .. j0+NW-1, two planes
  double kd[4][3][NW * kMarchLanes];         // k-face d of faces f (slot f & 3), per thread
  double kv[4][3][NW * kMarchLanes];         // k-face v of faces f (slot f & 3), per thread
};

// Fluxes of one face; zero where the face does not exist.  reg: the point's whole flux
// stencil is regular fluid interior (regular_faces), so the branch-free form applies.
// True when the three faces of point (i, j, k) take the interior form (face_flux_point's
// test); false for a point that does not exist.
__device__ __forceinline__ bool point_regular(const Grid &g, const uint8_t *__restrict__ nv, int i, int j, int k) {
  if (i < 2 || i > g.mx - 3 || j < 2 || j > g.my - 3 || k < 2 || k > g.mz - 3) return false;
  return regular_faces(nv, lidx(g, i, j, k), g.mx, (long long)g.mx * g.my);
}

template <int D>
__device__ __forceinline__ void march_face(const Grid &g, const Metrics &m, CV3 uc, CV3 u,
                                           const uint8_t *__restrict__ nv, const double *__restrict__ nut, int i,
                                           int j, int k, bool reg, double d[3], double v[3]) {
  d[0] = d[1] = d[2] = 0.0;
  v[0] = v[1] = v[2] = 0.0;
  if (i < 0 || j < 0 || k < 0) return;
  const long long p = lidx(g, i, j, k);
  if (D == 0) {
    if (reg) flux_i<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    else flux_i(g, m, uc, u, nv, nut, p, i, j, k, d, v);
  } else if (D == 1) {
    if (reg) flux_j<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    else flux_j(g, m, uc, u, nv, nut, p, i, j, k, d, v);
  } else {
    if (reg) flux_k<true>(g, m, uc, u, nv, nut, p, i, j, k, d, v);
    else flux_k(g, m, uc, u, nv, nut, p, i, j, k, d, v);
  }
}

// Face values by offset from the cell, for fp_cell (d at offsets -2..1, v at -1..0), all
// from shared memory: the i- and j-faces of the plane, and the thread's own ring of
// k-faces (face f in slot f & 3).
template <int NW>
struct MarchFaces {
  const MarchSmem<NW> *S;
  int b, w, lane, t, kc;
  __device__ __forceinline__ double d(int dir, int c, int off) const {
    if (dir == 0) return S->fi[w][c][lane + 2 + off];
    if (dir == 1) return S->jf[b][w + 2 + off][c][lane];
    return S->kd[(kc + off) & 3][c][t];
  }
  __device__ __forceinline__ double v(int dir, int c, int off) const {
    if (dir == 0) return S->fi[w][3 + c][lane + 2 + off];
    if (dir == 1) return S->jf[b][w + 2 + off][3 + c][lane];
    return S->kv[(kc + off) & 3][c][t];
  }
};

#ifndef VFS_MARCH_NW
#define VFS_MARCH_NW 16
#endif
#ifndef VFS_MARCH_MINB
#define VFS_MARCH_MINB 1
#endif
#ifndef VFS_MARCH_KC
#define VFS_MARCH_KC 32
#endif

template <int NW>
__global__ void __launch_bounds__(kMarchLanes * NW, VFS_MARCH_MINB)
    k_ff2_march(Grid g, Metrics m, CV3 uc, CV3 u, const uint8_t *__restrict__ nv, const double *__restrict__ nut,
                double scale, V3 rhs, int rk, double a, CV3 dP, CV3 pu, V3 out, int kc_per_block) {
  extern __shared__ __align__(16) unsigned char march_raw[];
  MarchSmem<NW> &S = *reinterpret_cast<MarchSmem<NW> *>(march_raw);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sy = mx, sz = (long long)mx * my;
  const int i0 = 1 + blockIdx.x * kMarchOut, j0 = 1 + blockIdx.y * (NW - 1);
  const int kb = 1 + blockIdx.z * kc_per_block;
  // the lanes' i-face slots 0, 1 and 34 (offsets beyond the warp) are read only by lanes
  // whose Fp is not used; clear them once so that nothing uninitialised is read
  if (lane < 3) {
    const int slot = lane < 2 ? lane : kMarchLanes + 2;
    for (int c = 0; c < 6; c++) S.fi[w][c][slot] = 0.0;
  }
  const int ke = min(kb + kc_per_block, mz - 1);  // right-hand side of planes kb .. ke-1
  const int uI = i0 - 2 + lane, vJ = j0 + w;
  const int ii = cell_image(uI, mx, g.iper), jj = cell_image(vJ, my, g.jper);
  const int fi = face_image_or_none(uI, mx, g.iper), fj = face_image_or_none(vJ, my, g.jper);
  // the extra j-face row of warps 0-2
  const int hv = w == 0 ? j0 - 2 : (w == 1 ? j0 - 1 : j0 + NW);
  const int hr = w == 0 ? 0 : (w == 1 ? 1 : NW + 2);
  const int hfj = face_image_or_none(hv, my, g.jper);
  // the DA point of this column (for the metrics of the projection products), if any
  const bool col_da = uI >= 0 && uI <= mx - 1 && vJ <= my - 1;
  const bool out_col = lane >= 2 && lane < 2 + kMarchOut && w <= NW - 2 && uI <= mx - 2 && vJ <= my - 2;

  // k-face ring (shared memory, own slots): warmed up with the faces kb-2 .. kb
  const int t = w * kMarchLanes + lane;
  for (int f = kb - 2; f <= kb; f++) {
    double d[3], v[3];
    const int fk = face_image_or_none(f, mz, g.kper);
    march_face<2>(g, m, uc, u, nv, nut, ii, jj, (ii >= 0 && jj >= 0) ? fk : -1, point_regular(g, nv, ii, jj, fk), d,
                  v);
#pragma unroll
    for (int c = 0; c < 3; c++) { S.kd[f & 3][c][t] = d[c]; S.kv[f & 3][c][t] = v[c]; }
  }
  // regularity of the point (ii, jj, kc), the point of the i- and j-faces of plane kc
  // away from periodic images; the k-face of plane kc computed it one plane earlier
  bool reg_ij = point_regular(g, nv, ii, jj, kb), reg_next = false;
  double ax_prev = 0, ay_prev = 0, az_prev = 0;
  for (int kc = kb; kc <= ke; kc++) {
    const int b = kc & 1;
    const int kimg = cell_image(kc, mz, g.kper);
    // k-face of plane kc+1 into the ring
    {
      double d[3], v[3];
      const int fk = face_image_or_none(kc + 1, mz, g.kper);
      reg_next = point_regular(g, nv, ii, jj, fk);
      march_face<2>(g, m, uc, u, nv, nut, ii, jj, (ii >= 0 && jj >= 0) ? fk : -1, reg_next, d, v);
#pragma unroll
      for (int c = 0; c < 3; c++) { S.kd[(kc + 1) & 3][c][t] = d[c]; S.kv[(kc + 1) & 3][c][t] = v[c]; }
    }
    // i-face and j-face of plane kc
    {
      double d[3], v[3];
      const bool same = fi == ii && fj == jj && kimg == kc;
      march_face<0>(g, m, uc, u, nv, nut, fi, jj, (fi >= 0 && jj >= 0) ? kimg : -1,
                    same ? reg_ij : point_regular(g, nv, fi, jj, kimg), d, v);
      // a row's i-faces are read only by its own warp: the __syncwarp after the
      // previous plane's Fp lets them be overwritten
#pragma unroll
      for (int c = 0; c < 3; c++) { S.fi[w][c][lane + 2] = d[c]; S.fi[w][3 + c][lane + 2] = v[c]; }
      march_face<1>(g, m, uc, u, nv, nut, ii, fj, (ii >= 0 && fj >= 0) ? kimg : -1,
                    same ? reg_ij : point_regular(g, nv, ii, fj, kimg), d, v);
#pragma unroll
      for (int c = 0; c < 3; c++) { S.jf[b][w + 2][c][lane] = d[c]; S.jf[b][w + 2][3 + c][lane] = v[c]; }
      if (w < 3) {
        march_face<1>(g, m, uc, u, nv, nut, ii, hfj, (ii >= 0 && hfj >= 0) ? kimg : -1,
                      point_regular(g, nv, ii, hfj, kimg), d, v);
#pragma unroll
        for (int c = 0; c < 3; c++) { S.jf[b][hr][c][lane] = d[c]; S.jf[b][hr][3 + c][lane] = v[c]; }
      }
    }
    __syncthreads();
    // Fp of (uI, vJ, kc)
    MarchFaces<NW> F;
    F.S = &S; F.b = b; F.w = w; F.lane = lane; F.t = t; F.kc = kc;
    double fpv[3] = {0, 0, 0};
    if (ii >= 0 && jj >= 0 && kimg >= 0) fp_cell(g, nv, lidx(g, ii, jj, kimg), ii, jj, kimg, F, fpv);
    __syncwarp();
    // projection products of this cell at plane kc (metrics of its own DA point)
    double ax = 0, ay = 0, az = 0;
    if (col_da && kc <= mz - 1) {
      const long long q = lidx(g, uI, vJ, kc);
      ax = m.csi.x[q] * fpv[0] + m.csi.y[q] * fpv[1] + m.csi.z[q] * fpv[2];
      ay = m.eta.x[q] * fpv[0] + m.eta.y[q] * fpv[1] + m.eta.z[q] * fpv[2];
      az = m.zet.x[q] * fpv[0] + m.zet.y[q] * fpv[1] + m.zet.z[q] * fpv[2];
    }
    S.ay[b][w][lane] = ay;
    // right-hand side of plane kc-1
    const double ax_right = __shfl_down_sync(0xffffffffu, ax_prev, 1);
    if (kc > kb && out_col && uI >= 1 && vJ >= 1) {
      const int k = kc - 1;
      const long long p = lidx(g, uI, vJ, k);
      const double ay_up = S.ay[b ^ 1][w + 1][lane];
      double r[3];
      if (rk) { r[0] = 0; r[1] = 0; r[2] = 0; }
      else { r[0] = rhs.x[p]; r[1] = rhs.y[p]; r[2] = rhs.z[p]; }
      r[0] += scale * (0.5 * ax_prev + 0.5 * ax_right) * m.iaj[p];
      r[1] += scale * (0.5 * ay_prev + 0.5 * ay_up) * m.jaj[p];
      r[2] += scale * (0.5 * az_prev + 0.5 * az) * m.kaj[p];
      if (nv[p] + nv[p + 1] > 0 || (!g.iper && uI == mx - 2)) r[0] = 0;
      if (nv[p] + nv[p + sy] > 0 || (!g.jper && vJ == my - 2)) r[1] = 0;
      if (nv[p] + nv[p + sz] > 0 || (!g.kper && k == mz - 2)) r[2] = 0;
      if (!rk) {
        rhs.x[p] = r[0]; rhs.y[p] = r[1]; rhs.z[p] = r[2];
      } else {
        r[0] = r[0] + -1 * dP.x[p];
        r[1] = r[1] + -1 * dP.y[p];
        r[2] = r[2] + -1 * dP.z[p];
        out.x[p] = a * r[0] + pu.x[p];
        out.y[p] = a * r[1] + pu.y[p];
        out.z[p] = a * r[2] + pu.z[p];
      }
    }
    ax_prev = ax; ay_prev = ay; az_prev = az;
    reg_ij = reg_next && face_image_or_none(kc + 1, mz, g.kper) == kc + 1;
  }
}

// Ghost points of the DA (an index 0 or m-1 in some direction): zero right-hand side, and
// in RK mode the stage update  out = pUcont + a (0 - dP)  (k_rhs at a ghost point).
__global__ void k_ff2_ghosts(Grid g, V3 rhs, int rk, double a, CV3 dP, CV3 pu, V3 out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ni = 2LL * g.my * g.mz, nj = 2LL * (g.mx - 2) * g.mz, nk = 2LL * (g.mx - 2) * (g.my - 2);
  if (t >= ni + nj + nk) return;
  long long r = t;
  int i, j, k;
  if (r < ni) { i = (r & 1) ? g.mx - 1 : 0; r >>= 1; j = (int)(r % g.my); k = (int)(r / g.my); }
  else if ((r -= ni) < nj) { j = (r & 1) ? g.my - 1 : 0; r >>= 1; i = 1 + (int)(r % (g.mx - 2)); k = (int)(r / (g.mx - 2)); }
  else { r -= nj; k = (r & 1) ? g.mz - 1 : 0; r >>= 1; i = 1 + (int)(r % (g.mx - 2)); j = 1 + (int)(r / (g.mx - 2)); }
  const long long p = lidx(g, i, j, k);
  double v[3] = {0, 0, 0};
  if (!rk) {
    rhs.x[p] = v[0]; rhs.y[p] = v[1]; rhs.z[p] = v[2];
  } else {
    v[0] = v[0] + -1 * dP.x[p];
    v[1] = v[1] + -1 * dP.y[p];
    v[2] = v[2] + -1 * dP.z[p];
    out.x[p] = a * v[0] + pu.x[p];
    out.y[p] = a * v[1] + pu.y[p];
    out.z[p] = a * v[2] + pu.z[p];
  }
}

// Formfunction_2 (momentum.c:456): adds scale * RHS into the context's RHS; in RK mode
// (rk_stage) writes the stage update  pUcont + rk_coeff (RHS - dP)  into the RHS arrays
// and swaps them with Ucont, so Ucont holds the updated fluxes (an RK step swaps four
// times and ends with the original arrays).
int formfunction2_onepass(Ctx *c, double scale, bool rk_stage, double rk_coeff) {
  const Grid &g = c->g;
  int rc;
  V3 uc = field3(c, VFS_UCONT);
  if ((rc = periodic_copy3(c, uc))) return rc;
  Metrics m = metrics(c);
  V3 pu{c->pucont[0], c->pucont[1], c->pucont[2]};
  V3 rhs = field3(c, VFS_RHS);
  constexpr int NW = VFS_MARCH_NW;
  const size_t smem = sizeof(MarchSmem<NW>);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_ff2_march<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  const int kc = VFS_MARCH_KC;
  dim3 grid((g.mx - 2 + kMarchOut - 1) / kMarchOut, (g.my - 2 + NW - 2) / (NW - 1), (g.mz - 2 + kc - 1) / kc);
  c->launches++, k_ff2_march<NW><<<grid, dim3(kMarchLanes, NW), smem, c->stream>>>(
      g, m, cv(uc), cv(field3(c, VFS_UCAT)), c->nv, c->f[VFS_NU_T][0], scale, rhs, rk_stage ? 1 : 0, rk_coeff,
      cv(field3(c, VFS_DP)), cv(pu), rhs, kc);
  if ((rc = check_launch(c, "k_ff2_march"))) return rc;
  const long long ng = 2LL * g.my * g.mz + 2LL * (g.mx - 2) * g.mz + 2LL * (g.mx - 2) * (g.my - 2);
  c->launches++, k_ff2_ghosts<<<nblocks(ng, 256), 256, 0, c->stream>>>(g, rhs, rk_stage ? 1 : 0, rk_coeff,
                                                                      cv(field3(c, VFS_DP)), cv(pu), rhs);
  if ((rc = check_launch(c, "k_ff2_ghosts"))) return rc;
  if (rk_stage) {
    for (int q = 0; q < 3; q++) std::swap(c->f[VFS_UCONT][q], c->f[VFS_RHS][q]);
  }
  return VFS_OK;
}

// The form the step runs.
#ifndef VFS_FF2_ONEPASS
#define VFS_FF2_ONEPASS 0
#endif
int formfunction2(Ctx *c, double scale, bool rk_stage, double rk_coeff) {
  return VFS_FF2_ONEPASS ? formfunction2_onepass(c, scale, rk_stage, rk_coeff)
                         : formfunction2_split(c, scale, rk_stage, rk_coeff);
}

// single-kernel launchers for the diagnostics entry point (vfs_run_kernel)
void launch_face_flux(Ctx *c) { face_fluxes(c); }
void launch_fp(Ctx *c) {
  c->launches++, k_fp<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, flux_in(c, 0), flux_in(c, 1), flux_in(c, 2), c->nv,
                                                   c->fp[0], c->fp[1], c->fp[2]);
}
void launch_rhs(Ctx *c) {
  V3 pu{c->pucont[0], c->pucont[1], c->pucont[2]};
  c->launches++, k_rhs<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), c->nv, c->fp[0], c->fp[1], c->fp[2], 1.0,
                                                    field3(c, VFS_RHS), 0, 0.0, cv(field3(c, VFS_DP)), cv(pu),
                                                    field3(c, VFS_UCONT));
}

// ------------------------------------------------------------------ face-metric products
// The nine products of face metrics that Pressure_Gradient (momentum.c:311-319) and
// Projection (poisson.c:2837-2960) form at every face: on the i-face icsi.icsi, ieta.icsi,
// izet.icsi; on the j-face jcsi.jeta, jeta.jeta, jzet.jeta; on the k-face kcsi.kzet,
// keta.kzet, kzet.kzet, each summed x + y + z in that order.  Stored once per metric upload
// (9 x N doubles, slot q of point p at G[q*N + p]); both kernels read 12 doubles per point
// (these and iaj, jaj, kaj) instead of the 30 face metrics, with the same bits as forming
// them in place.
__global__ void k_gab(Grid g, Metrics m, double *G) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const long long N = g.N;
  G[p] = dot3(m.icsi.x[p], m.icsi.y[p], m.icsi.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  G[N + p] = dot3(m.ieta.x[p], m.ieta.y[p], m.ieta.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  G[2 * N + p] = dot3(m.izet.x[p], m.izet.y[p], m.izet.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  G[3 * N + p] = dot3(m.jcsi.x[p], m.jcsi.y[p], m.jcsi.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  G[4 * N + p] = dot3(m.jeta.x[p], m.jeta.y[p], m.jeta.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  G[5 * N + p] = dot3(m.jzet.x[p], m.jzet.y[p], m.jzet.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  G[6 * N + p] = dot3(m.kcsi.x[p], m.kcsi.y[p], m.kcsi.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
  G[7 * N + p] = dot3(m.keta.x[p], m.keta.y[p], m.keta.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
  G[8 * N + p] = dot3(m.kzet.x[p], m.kzet.y[p], m.kzet.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
}

int ensure_gab(Ctx *c) {
  if (c->gab_valid) return VFS_OK;
  if (c->capturing) return set_err(c, VFS_ERR_STATE, "face-metric products not formed before capture");
  if (!c->gab && cudaMalloc(&c->gab, sizeof(double) * 9 * (size_t)c->g.N) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "face-metric product allocation failed");
  c->launches++, k_gab<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), c->gab);
  int rc = check_launch(c, "k_gab");
  if (rc == VFS_OK) c->gab_valid = true;
  c->setup_epoch++;
  return rc;
}

// ------------------------------------------------------------------ Pressure_Gradient
// momentum.c:197-443 (levelset off): dP on the three faces of each interior cell, with
// one-sided cross differences next to IB nodes (nvert == 1) and non-periodic walls, and
// the mean-pressure-gradient forcing along a periodic k direction.
// Five resident blocks per SM (a small spill) hide the loads of the 30 metric arrays:
// 0.71 ms against 1.14 ms uncapped at 12.6 M cells.
#ifndef VFS_PG_MINB
#define VFS_PG_MINB 5
#endif
__global__ void __launch_bounds__(256, VFS_PG_MINB) k_pressure_gradient(Grid g, const double *__restrict__ G,
                                    const double *__restrict__ iaj, const double *__restrict__ jaj,
                                    const double *__restrict__ kaj, const uint8_t *__restrict__ nv,
                                    const double *__restrict__ P, double kdiff, double kdt,
                                    double karea, int kforce_mode, double mpg, const double *__restrict__ ds,
                                    V3 dp) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) {
    dp.x[p] = 0; dp.y[p] = 0; dp.z[p] = 0;  // VecSet(dP, 0) outside the loop
    return;
  }
  const long long sy = mx, sz = (long long)mx * my, N = g.N;
  const double g11_i = __ldcs(G + p), g12_i = __ldcs(G + N + p), g13_i = __ldcs(G + 2 * N + p);
  const double g21_j = __ldcs(G + 3 * N + p), g22_j = __ldcs(G + 4 * N + p), g23_j = __ldcs(G + 5 * N + p);
  const double g31_k = __ldcs(G + 6 * N + p), g32_k = __ldcs(G + 7 * N + p), g33_k = __ldcs(G + 8 * N + p);
  const double r1 = 1.0, r2 = 1.0, r3 = 1.0;
  auto ib = [&](long long o) { return nv[o] == 1; };  // (int)(nvert+0.5)==1
  double dpdc, dpde, dpdz;
  // x face
  if ((i == 0 || i == mx - 2) && g.iper) dpdc = P[p - i + 1] - P[p];
  else dpdc = P[p + 1] - P[p];
  if (ib(p + sy) || ib(p + sy + 1) || (j == my - 2 && !g.jper))
    dpde = (P[p] - P[p - sy] + P[p + 1] - P[p - sy + 1]) * 0.5;
  else if (ib(p - sy) || ib(p - sy + 1) || (j == 1 && !g.jper))
    dpde = (P[p + sy] - P[p] + P[p + sy + 1] - P[p + 1]) * 0.5;
  else dpde = (P[p + sy] - P[p - sy] + P[p + sy + 1] - P[p - sy + 1]) * 0.25;
  if (ib(p + sz) || ib(p + sz + 1) || (k == mz - 2 && !g.kper))
    dpdz = (P[p] - P[p - sz] + P[p + 1] - P[p - sz + 1]) * 0.5;
  else if (ib(p - sz) || ib(p - sz + 1) || (k == 1 && !g.kper))
    dpdz = (P[p + sz] - P[p] + P[p + sz + 1] - P[p + 1]) * 0.5;
  else dpdz = (P[p + sz] - P[p - sz] + P[p + sz + 1] - P[p - sz + 1]) * 0.25;
  double ox = (dpdc * g11_i + dpde * g12_i + dpdz * g13_i) * iaj[p] / r1;
  // y face
  if (ib(p + 1) || ib(p + sy + 1) || (i == mx - 2 && !g.iper))
    dpdc = (P[p] - P[p - 1] + P[p + sy] - P[p + sy - 1]) * 0.5;
  else if (ib(p - 1) || ib(p + sy - 1) || (i == 1 && !g.iper))
    dpdc = (P[p + 1] - P[p] + P[p + sy + 1] - P[p + sy]) * 0.5;
  else dpdc = (P[p + 1] - P[p - 1] + P[p + sy + 1] - P[p + sy - 1]) * 0.25;
  if ((j == 0 || j == my - 2) && g.jper) dpde = P[p - (long long)j * sy + sy] - P[p];
  else dpde = P[p + sy] - P[p];
  if (ib(p + sz) || ib(p + sz + sy) || (k == mz - 2 && !g.kper))
    dpdz = (P[p] - P[p - sz] + P[p + sy] - P[p - sz + sy]) * 0.5;
  else if (ib(p - sz) || ib(p - sz + sy) || (k == 1 && !g.kper))
    dpdz = (P[p + sz] - P[p] + P[p + sz + sy] - P[p + sy]) * 0.5;
  else dpdz = (P[p + sz] - P[p - sz] + P[p + sz + sy] - P[p - sz + sy]) * 0.25;
  double oy = (dpdc * g21_j + dpde * g22_j + dpdz * g23_j) * jaj[p] / r2;
  // z face
  if (ib(p + 1) || ib(p + sz + 1) || (i == mx - 2 && !g.iper))
    dpdc = (P[p] - P[p - 1] + P[p + sz] - P[p + sz - 1]) * 0.5;
  else if (ib(p - 1) || ib(p + sz - 1) || (i == 1 && !g.iper))
    dpdc = (P[p + 1] - P[p] + P[p + sz + 1] - P[p + sz]) * 0.5;
  else dpdc = (P[p + 1] - P[p - 1] + P[p + sz + 1] - P[p + sz - 1]) * 0.25;
  if (ib(p + sy) || ib(p + sz + sy) || (j == my - 2 && !g.jper))
    dpde = (P[p] - P[p - sy] + P[p + sz] - P[p + sz - sy]) * 0.5;
  else if (ib(p - sy) || ib(p + sz - sy) || (j == 1 && !g.jper))
    dpde = (P[p + sy] - P[p] + P[p + sz + sy] - P[p + sz]) * 0.5;
  else dpde = (P[p + sy] - P[p - sy] + P[p + sz + sy] - P[p + sz - sy]) * 0.25;
  if ((k == 0 || k == mz - 2) && g.kper) dpdz = P[p - (long long)k * sz + sz] - P[p];
  else dpdz = (P[p + sz] - P[p]);
  if (g.kper) {
    const double dz = 1. / kaj[p] / sqrt(g33_k);   // |kzet|^2 is g33
    if (kforce_mode == 1) dpdz += mpg * dz;
    else if (kforce_mode == 2) {
      // ds: the step's device scalars (mean_k_flux - inlet_flux, mean_k_area)
      if (ds) { kdiff = ds[DS_MEAN_K_FLUX] - ds[DS_INLET_FLUX]; karea = ds[DS_MEAN_K_AREA]; }
      dpdz += dz * kdiff / kdt / karea;
    }
  }
  double oz = (dpdc * g31_k + dpde * g32_k + dpdz * g33_k) * kaj[p] / r3;
  if (i == 0 || nv[p] + nv[p + 1] > 0 || (!g.iper && i == mx - 2)) ox = 0;
  if (j == 0 || nv[p] + nv[p + sy] > 0 || (!g.jper && j == my - 2)) oy = 0;
  if (k == 0 || nv[p] + nv[p + sz] > 0 || (!g.kper && k == mz - 2)) oz = 0;
  dp.x[p] = ox; dp.y[p] = oy; dp.z[p] = oz;
}

// k-periodic forcing (momentum.c:379-399): dpdz_set -> mean_pressure_gradient (mode 1),
// else (inletprofile != 17) the flux-deficit term (mean_k_flux - inlet_flux)/dt/mean_k_area
// (mode 2); only a k-periodic grid applies it.
int pressure_forcing_mode(const Ctx *c) {
  if (c->cfg.dpdz_set) return 1;
  if (c->cfg.inletprofile != 17) return 2;
  return 0;
}

// Pressure_Gradient with an explicit forcing mode and flux deficit kdiff (ds null), or
// with the flux deficit of the step's device scalars (ds = c->ds).
static int pressure_gradient_launch(Ctx *c, int mode, double kdiff, const double *ds) {
  int rc;
  if ((rc = ensure_gab(c))) return rc;
  // P's periodic ghosts are refreshed first (momentum.c:241-273)
  if ((rc = periodic_copy1(c, c->f[VFS_P][0]))) return rc;
  c->launches++, k_pressure_gradient<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(
      c->g, c->gab, c->f[VFS_IAJ][0], c->f[VFS_JAJ][0], c->f[VFS_KAJ][0], c->nv, c->f[VFS_P][0], kdiff, c->g.dt,
      c->scal[VFS_S_MEAN_K_AREA], mode, c->cfg.mean_pressure_gradient, ds, field3(c, VFS_DP));
  return check_launch(c, "k_pressure_gradient");
}

int pressure_gradient_mode(Ctx *c, int mode, double kdiff) { return pressure_gradient_launch(c, mode, kdiff, nullptr); }

// The step's Pressure_Gradient: Calc_k_Flux's result and the inlet flux from the device
// scalars (which vfs_set_scalar keeps equal to the host's between steps).
int pressure_gradient(Ctx *c) { return pressure_gradient_launch(c, pressure_forcing_mode(c), 0.0, c->ds); }

// ------------------------------------------------------------------ Calc_k_Flux
// rhs2.c:1562-1646: sum of Ucont.z over k-faces k = 1..mz-2, interior (i,j), whose two
// adjacent cells are fluid; divided by (mz-2).
__global__ void k_kflux_parts(Grid g, const double *__restrict__ uz, const uint8_t *__restrict__ nv,
                              double *parts) {
  __shared__ double sh[256];
  double s = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (k < 1 || k > g.mz - 2 || j < 1 || j > g.my - 2 || i < 1 || i > g.mx - 2) continue;
    const long long sz = (long long)g.mx * g.my;
    if (nv[p - sz] + nv[p] == 0) s += uz[p];
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// ds[dst] = ds[src] / den (one thread).
__global__ void k_ds_div(double *ds, int dst, int src, double den) { ds[dst] = ds[src] / den; }
// ds[dst] = ds[src] (one thread).
__global__ void k_ds_copy(double *ds, int dst, int src) { ds[dst] = ds[src]; }

int calc_k_flux(Ctx *c, double *flux) {
  int rc;
  const int nb = 148 * 4;
  if ((rc = ensure_red(c, nb + 64))) return rc;
  c->launches++, k_kflux_parts<<<nb, 256, 0, c->stream>>>(c->g, c->f[VFS_UCONT][2], c->nv, c->red);
  if ((rc = check_launch(c, "k_kflux_parts"))) return rc;
  if ((rc = reduce_to(c, c->red, nb, c->ds + DS_KFLUX_SUM))) return rc;
  c->launches++, k_ds_div<<<1, 1, 0, c->stream>>>(c->ds, DS_MEAN_K_FLUX, DS_KFLUX_SUM, (double)(c->g.mz - 2));
  if ((rc = check_launch(c, "k_ds_div"))) return rc;
  if (!c->capturing) {
    if ((rc = ds_fetch(c))) return rc;
    if (flux) *flux = c->scal[VFS_S_MEAN_K_FLUX];
  }
  return VFS_OK;
}

// ------------------------------------------------------------------ Calc_Inlet_Area
// bcs.c:216-322: mean over k = 1..mz-2 of the fluid k-face area |zet| of the interior
// (i,j), and the fluid area of the k = 0 plane (inletArea) for an inlet or periodic k.
__global__ void k_area_parts(Grid g, CV3 zet, const uint8_t *__restrict__ nv, double *parts) {
  __shared__ double s1[256], s2[256];
  double a = 0, b = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long sz = (long long)g.mx * g.my;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (j < 1 || j > g.my - 2 || i < 1 || i > g.mx - 2) continue;
    const double area = sqrt(zet.x[p] * zet.x[p] + zet.y[p] * zet.y[p] + zet.z[p] * zet.z[p]);
    if (k >= 1 && k <= g.mz - 2 && nv[p - sz] + nv[p] == 0) a += area;
    if (k == 0 && nv[p + sz] == 0) b += area;
  }
  s1[threadIdx.x] = a; s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { parts[blockIdx.x] = s1[0]; parts[gridDim.x + blockIdx.x] = s2[0]; }
}

int calc_inlet_area(Ctx *c) {
  int rc;
  const int nb = 148 * 2;
  if ((rc = ensure_red(c, 2 * nb + 64))) return rc;
  c->launches++, k_area_parts<<<nb, 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_ZET)), c->nv, c->red);
  if ((rc = check_launch(c, "k_area_parts"))) return rc;
  double a = 0, b = 0;
  if ((rc = reduce_sum(c, c->red, nb, &a))) return rc;
  if ((rc = reduce_sum(c, c->red + nb, nb, &b))) return rc;
  c->scal[VFS_S_MEAN_K_AREA] = a / (double)(c->g.mz - 2);
  if (c->g.bc[4] == 5 || c->g.kper) c->scal[VFS_S_INLET_AREA] = b;
  return ds_upload(c);
}

// ------------------------------------------------------------------ IB_BC (no IB nodes)
// momentum.c:1982-2195 without immersed bodies: normal flux through free-slip faces set
// to zero and the normal flux of periodic ghost planes taken from the image plane.
__global__ void k_ib_bc_faces(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const long long sy = mx, sz = (long long)mx * my;
  const int *bc = g.bc;
  // the reference loops over all points and writes the plane values named below; each
  // thread writes exactly the entries the loop would write at its (i,j,k)
  if (bc[0] == 10 && i == 1) uc.x[p - 1] = 0;
  if (bc[1] == 10 && i == mx - 2) uc.x[p] = 0;
  if (bc[2] == 10 && j == 1) uc.y[p - sy] = 0;
  if (bc[3] == 10 && j == my - 2) uc.y[p] = 0;
  if (bc[4] == 10 && k == 1) uc.z[p - sz] = 0;
  if (bc[5] == 10 && k == mz - 2) uc.z[p] = 0;
}
__global__ void k_periodic_normal(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const long long sy = mx, sz = (long long)mx * my;
  if (g.iper && i == 0) uc.x[p] = uc.x[p + (mx - 2)];
  if (g.iper && i == mx - 1) uc.x[p] = uc.x[p - (mx - 2)];
  if (g.jper && j == 0) uc.y[p] = uc.y[p + (long long)(my - 2) * sy];
  if (g.jper && j == my - 1) uc.y[p] = uc.y[p - (long long)(my - 2) * sy];
  if (g.kper && k == 0) uc.z[p] = uc.z[p + (long long)(mz - 2) * sz];
  if (g.kper && k == mz - 1) uc.z[p] = uc.z[p - (long long)(mz - 2) * sz];
}

int ib_bc(Ctx *c) {
  int rc;
  if (c->g.immersed) {  // momentum.c:2049-2108: periodic Ucat ghosts, then the IB-node faces
    if ((rc = periodic_copy3(c, field3(c, VFS_UCAT)))) return rc;
    if ((rc = ib_faces(c))) return rc;
  }
  c->launches++, k_ib_bc_faces<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
  if ((rc = check_launch(c, "k_ib_bc_faces"))) return rc;
  if (c->g.iper || c->g.jper || c->g.kper) {
    c->launches++, k_periodic_normal<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
    if ((rc = check_launch(c, "k_periodic_normal"))) return rc;
  }
  return VFS_OK;
}

// Transpose of k_periodic_normal: each source face adds the adjoint of the ghost face
// that copies it (i = 0 <- mx-2, mx-1 <- 1, per normal component); the ghosts are cleared.
__global__ void k_periodic_normal_adjoint(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const long long sy = mx, sz = (long long)mx * my;
  if (g.iper) {
    if (i == mx - 2) uc.x[p] += uc.x[p - (mx - 2)];
    if (i == 1) uc.x[p] += uc.x[p + (mx - 2)];
  }
  if (g.jper) {
    if (j == my - 2) uc.y[p] += uc.y[p - (long long)(my - 2) * sy];
    if (j == 1) uc.y[p] += uc.y[p + (long long)(my - 2) * sy];
  }
  if (g.kper) {
    if (k == mz - 2) uc.z[p] += uc.z[p - (long long)(mz - 2) * sz];
    if (k == 1) uc.z[p] += uc.z[p + (long long)(mz - 2) * sz];
  }
}
__global__ void k_periodic_normal_clear(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (g.iper && (i == 0 || i == g.mx - 1)) uc.x[p] = 0;
  if (g.jper && (j == 0 || j == g.my - 1)) uc.y[p] = 0;
  if (g.kper && (k == 0 || k == g.mz - 1)) uc.z[p] = 0;
}

// Transpose of ib_bc without IB nodes: k_periodic_normal, then the 0/1 diagonal
// k_ib_bc_faces (its own transpose).
int ib_bc_adjoint(Ctx *c, V3 luc) {
  int rc;
  if (c->g.immersed) return set_err(c, VFS_ERR_INVALID, "ib_bc_adjoint: IB nodes need the measured operator");
  if (c->g.iper || c->g.jper || c->g.kper) {
    c->launches++, k_periodic_normal_adjoint<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, luc);
    if ((rc = check_launch(c, "k_periodic_normal_adjoint"))) return rc;
    c->launches++, k_periodic_normal_clear<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, luc);
    if ((rc = check_launch(c, "k_periodic_normal_clear"))) return rc;
  }
  c->launches++, k_ib_bc_faces<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, luc);
  return check_launch(c, "k_ib_bc_faces");
}

// ------------------------------------------------------------------ InflowFlux
// bcs.c:329-706 for an inlet on the k = 0 face (bctype[4] = 5), interior (i, j):
//   inletprofile 2     uniform uin = inlet_flux/inletArea (1 when inlet_flux < 0);
//   inletprofile 1     uin = 0: the reference sets the uniform value first, then its
//                      second profile chain (bcs.c:408-466) has no branch for 1 and ends
//                      in uin = 0, which is what the reference runs with;
//   inletprofile 21    laminar Poiseuille 1.5*yc*(2 - yc) at the k = 1 face centre;
//   inletprofile 100   Cartesian velocity plane supplied by the caller (ucont_plane,
//                      read_inflow_section, rhs2.c:701), then the flux rescaled to
//                      inlet_flux over the fluid inlet area.
// A face whose downstream cell is blocked (nvert[1] >= 0.1) gets zero flux.  The ghost
// velocity at k = 0 is -Ucat(k=1) + 2*u(face), u from the face flux by Cramer's rule
// (Contra2Cart_single, rhs.c:34).
__global__ void k_inflow(Grid g, Metrics m, V3 uc, V3 ucat, const uint8_t *__restrict__ nv, int profile,
                         const double *__restrict__ ds, const double *__restrict__ plane,
                         const double *__restrict__ ynode, double *parts) {
  __shared__ double sh[256];
  // uniform inflow of profile 2: the bulk velocity from the target flux (bcs.c:399-412)
  const double inlet_flux = ds[DS_INLET_FLUX], inlet_area = ds[DS_INLET_AREA];
  const double uin_const = (profile == 2) ? ((inlet_flux < 0) ? 1. : inlet_flux / inlet_area) : 0.0;
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = 0;
  if (t < (long long)nx * ny) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
    const long long p = lidx(g, i, j, 0), p1 = p + (long long)g.mx * g.my;
    const double zx = m.zet.x[p], zy = m.zet.y[p], zz = m.zet.z[p];
    const double area = sqrt(zx * zx + zy * zy + zz * zz);
    if (nv[p1] == 0) {
      if (profile == 100) {
        const double *pl = plane + 3 * ((long long)j * g.mx + i);
        const double u = pl[0], v = pl[1], w = pl[2];
        ucat.x[p] = u; ucat.y[p] = v; ucat.z[p] = w;
        uc.z[p] = 0.5 * (u + ucat.x[p1]) * zx + 0.5 * (v + ucat.y[p1]) * zy + 0.5 * (w + ucat.z[p1]) * zz;
      } else {
        double uin = uin_const;
        if (profile == 21) {
          const int IM = g.mx - 1;
          const double yc = (ynode[(long long)j * IM + i] + ynode[(long long)(j - 1) * IM + i] +
                             ynode[(long long)j * IM + i - 1] + ynode[(long long)(j - 1) * IM + i - 1]) * 0.25;
          const double w_bulk = 1.0;
          uin = 1.5 * w_bulk * yc * (2 - yc);
        }
        const double ux = 0, uy = 0, uz = uin * area;
        uc.z[p] = uz; uc.x[p] = ux; uc.y[p] = uy;
        const double cx = m.csi.x[p], cy = m.csi.y[p], cz = m.csi.z[p];
        const double ex = m.eta.x[p], ey = m.eta.y[p], ez = m.eta.z[p];
        const double det = cx * (ey * zz - ez * zy) - cy * (ex * zz - ez * zx) + cz * (ex * zy - ey * zx);
        const double det0 = ux * (ey * zz - ez * zy) - uy * (cy * zz - cz * zy) + uz * (cy * ez - cz * ey);
        const double det1 = -ux * (ex * zz - ez * zx) + uy * (cx * zz - cz * zx) - uz * (cx * ez - cz * ex);
        const double det2 = ux * (ex * zy - ey * zx) - uy * (cx * zy - cy * zx) + uz * (cx * ey - cy * ex);
        const double vx = det0 / det, vy = det1 / det, vz = det2 / det;
        ucat.x[p] = -ucat.x[p1] + 2 * vx;
        ucat.y[p] = -ucat.y[p1] + 2 * vy;
        ucat.z[p] = -ucat.z[p1] + 2 * vz;
      }
    } else {
      ucat.z[p] = 0;
      uc.z[p] = 0;
    }
    s = uc.z[p];
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// Flux rescaling of the inlet plane (bcs.c:579-587): Ucont.z += dflux*|zet|/inletArea on
// faces with a fluid downstream cell, and the partial sums of the new inlet flux.
__global__ void k_inflow_rescale(Grid g, CV3 zet, V3 uc, const uint8_t *__restrict__ nv, const double *__restrict__ ds,
                                 double *parts) {
  // the target flux and the flux of the profile from the device scalars; with no target
  // (inlet_flux <= 0) the plane is left as it is and only summed
  const double inlet_flux = ds[DS_INLET_FLUX], inlet_area = ds[DS_INLET_AREA];
  const bool rescale = inlet_flux > 0;
  const double dflux = inlet_flux - ds[DS_FLUX1];
  __shared__ double sh[256];
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double s = 0;
  if (t < (long long)nx * ny) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
    const long long p = lidx(g, i, j, 0), p1 = p + (long long)g.mx * g.my;
    if (nv[p1] == 0) {
      if (rescale) {
        const double A = sqrt(zet.x[p] * zet.x[p] + zet.y[p] * zet.y[p] + zet.z[p] * zet.z[p]);
        uc.z[p] += dflux * A / inlet_area;
      }
      s = uc.z[p];
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

int inflow_flux(Ctx *c) {
  const Grid &g = c->g;
  if (g.bc[4] != 5) return VFS_OK;  // no k = 0 inlet: FluxInSum keeps its value
  const int prof = c->cfg.inletprofile;
  int rc;
  if (prof == 100 && !c->inflow_plane)
    return set_err(c, VFS_ERR_STATE, "InflowFlux: inletprofile 100 needs vfs_set_inflow_plane first");
  if (prof == 21 && !c->inlet_nodes)
    return set_err(c, VFS_ERR_STATE, "InflowFlux: inletprofile 21 needs the grid nodes (vfs_form_metrics)");
  const long long npl = (long long)(g.mx - 2) * (g.my - 2);
  const int nb = (int)nblocks(npl, 256);
  if ((rc = ensure_red(c, nb + 64))) return rc;
  c->launches++, k_inflow<<<nb, 256, 0, c->stream>>>(g, metrics(c), field3(c, VFS_UCONT), field3(c, VFS_UCAT), c->nv, prof, c->ds,
                                     c->inflow_plane, c->inlet_nodes ? c->inlet_nodes + 1 * (size_t)(g.mx - 1) * (g.my - 1) : nullptr,
                                     c->red);
  if ((rc = check_launch(c, "k_inflow"))) return rc;
  if ((rc = reduce_to(c, c->red, nb, c->ds + DS_FLUX1))) return rc;
  if (prof == 100) {  // bcs.c:572-588 (sumFluxIn0 = inlet_flux), when inlet_flux > 0
    c->launches++, k_inflow_rescale<<<nb, 256, 0, c->stream>>>(g, cv(field3(c, VFS_ZET)), field3(c, VFS_UCONT), c->nv,
                                               c->ds, c->red);
    if ((rc = check_launch(c, "k_inflow_rescale"))) return rc;
    if ((rc = reduce_to(c, c->red, nb, c->ds + DS_FLUX_IN))) return rc;
  } else {
    c->launches++, k_ds_copy<<<1, 1, 0, c->stream>>>(c->ds, DS_FLUX_IN, DS_FLUX1);
    if ((rc = check_launch(c, "k_ds_copy"))) return rc;
  }
  return ds_fetch(c);
}

// ------------------------------------------------------------------ FormBCS subset
// bcs.c:1841-2936 for the codes handled here: Contra2Cart; at an outlet on the k = mz-1
// face (bctype[5] = 4) and with outflow_scale set, the last interior k-face fluxes are
// shifted by (FluxInSum - FluxOut)*|zet|/Area over faces with a fluid upstream cell
// (bcs.c:2285-2417); zero normal flux on no-slip and free-slip walls of the i and j faces
// (interior range); Contra2Cart again; the twelve edges of the box get Ucat = 0.
__global__ void k_outlet_parts(Grid g, CV3 zet, const double *__restrict__ uz, const uint8_t *__restrict__ nv,
                               double *parts) {
  __shared__ double s1[256], s2[256];
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double f = 0, a = 0;
  if (t < (long long)nx * ny) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
    const long long p = lidx(g, i, j, g.mz - 2);
    if (nv[p] == 0) {
      f = uz[p];
      a = sqrt(zet.x[p] * zet.x[p] + zet.y[p] * zet.y[p] + zet.z[p] * zet.z[p]);
    }
  }
  s1[threadIdx.x] = f; s2[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { parts[blockIdx.x] = s1[0]; parts[gridDim.x + blockIdx.x] = s2[0]; }
}

__global__ void k_outlet_scale(Grid g, CV3 zet, double *uz, const uint8_t *__restrict__ nv,
                               const double *__restrict__ ds) {
  const double dflux = ds[DS_FLUX_IN] - ds[DS_FLUX_OUT], area_sum = ds[DS_AREA_OUT];
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny) return;
  const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
  const long long p = lidx(g, i, j, g.mz - 2);
  const double Area = sqrt(zet.x[p] * zet.x[p] + zet.y[p] * zet.y[p] + zet.z[p] * zet.z[p]);
  if (nv[p] == 0) uz[p] += dflux * Area / area_sum;
}

__global__ void k_wall_flux(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int *bc = g.bc;
  bool ik = (k >= 1 && k <= mz - 2);
  if (ik && j >= 1 && j <= my - 2) {
    if ((bc[0] == 1 || bc[0] == 10) && i == 0) uc.x[p] = 0;
    if ((bc[1] == 1 || bc[1] == 10) && i == mx - 2) uc.x[p] = 0;
  }
  if (ik && i >= 1 && i <= mx - 2) {
    if ((bc[2] == 1 || bc[2] == 10) && j == 0) uc.y[p] = 0;
    if ((bc[3] == 1 || bc[3] == 10) && j == my - 2) uc.y[p] = 0;
  }
}
__global__ void k_zero_edges(Grid g, V3 u) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  int bi = (i == 0 || i == mx - 1), bj = (j == 0 || j == my - 1), bk = (k == 0 || k == mz - 1);
  if (bi + bj + bk >= 2) { u.x[p] = 0; u.y[p] = 0; u.z[p] = 0; }
}

// The outlet flux rescaling of FormBCS (outflow_scale set, bctype[5] = 4).
int outlet_rescale(Ctx *c) {
  int rc;
  {
    const Grid &g = c->g;
    const long long npl = (long long)(g.mx - 2) * (g.my - 2);
    const int nb = (int)nblocks(npl, 256);
    if ((rc = ensure_red(c, 2 * nb + 64))) return rc;
    c->launches++, k_outlet_parts<<<nb, 256, 0, c->stream>>>(g, cv(field3(c, VFS_ZET)), c->f[VFS_UCONT][2], c->nv, c->red);
    if ((rc = check_launch(c, "k_outlet_parts"))) return rc;
    if ((rc = reduce_to(c, c->red, nb, c->ds + DS_FLUX_OUT))) return rc;
    if ((rc = reduce_to(c, c->red + nb, nb, c->ds + DS_AREA_OUT))) return rc;
    c->launches++, k_outlet_scale<<<nb, 256, 0, c->stream>>>(g, cv(field3(c, VFS_ZET)), c->f[VFS_UCONT][2], c->nv, c->ds);
    if ((rc = check_launch(c, "k_outlet_scale"))) return rc;
  }
  return ds_fetch(c);
}

// FormBCS after the outlet rescaling: wall fluxes, Contra2Cart, box edges.
int form_bcs_tail(Ctx *c) {
  int rc;
  c->launches++, k_wall_flux<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
  if ((rc = check_launch(c, "k_wall_flux"))) return rc;
  if ((rc = contra2cart(c))) return rc;
  c->launches++, k_zero_edges<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCAT));
  return check_launch(c, "k_zero_edges");
}

// Transpose of form_bcs_tail: k_wall_flux and k_zero_edges zero entries (0/1 diagonals,
// their own transposes) around Contra2Cart.
int form_bcs_tail_adjoint(Ctx *c, V3 luc, V3 lucat, V3 luo, V3 tmp) {
  int rc;
  c->launches++, k_zero_edges<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, lucat);
  if ((rc = check_launch(c, "k_zero_edges"))) return rc;
  if ((rc = contra2cart_adjoint(c, luc, lucat, luo, tmp))) return rc;
  c->launches++, k_wall_flux<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, luc);
  return check_launch(c, "k_wall_flux");
}

int form_bcs(Ctx *c, bool outflow_scale) {
  int rc;
  if ((rc = contra2cart(c))) return rc;
  if (c->g.bc[5] == 4 && outflow_scale && (rc = outlet_rescale(c))) return rc;
  return form_bcs_tail(c);
}

// ------------------------------------------------------------------ RungeKutta
// rhs.c:1578-1700 (implicit=0): InflowFlux, FormBCS without outlet rescaling, the IB-node
// interpolation when immersed, then four stages  Contra2Cart; Rhs = Formfunction_2 - dP; Ucont = pUcont + alfa*dt*st*Rhs;
// Contra2Cart  and finally FormBCS with the outlet rescaling (outflow_scale = 1).
int runge_kutta(Ctx *c) {
  int rc;
  const double alfa[4] = {0.25, 1 / 3., 0.5, 1.};
  if ((rc = inflow_flux(c))) return rc;
  if ((rc = form_bcs(c, false))) return rc;
  if (c->g.immersed && (rc = ibm_interpolation(c))) return rc;  // rhs.c:1610-1614
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(c->pucont[q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  for (int s = 0; s < 4; s++) {
    // the reference converts at the start and at the end of every stage; the start of
    // stage s > 0 sees exactly the Ucont the end of stage s-1 converted, and Contra2Cart
    // of the same Ucont reproduces the same Ucat, so only stage 0 converts first
    if (s == 0 && (rc = contra2cart(c))) return rc;
    if (c->tape && (rc = tape_stage(c, s))) return rc;
    const double a = alfa[s] * c->g.dt * c->g.st;
    if ((rc = formfunction2(c, 1.0, true, a))) return rc;
    if ((rc = contra2cart(c))) return rc;
  }
  // FormBCS with the outlet rescaling (rhs.c:1670).  Its leading Contra2Cart would convert
  // the Ucont the last stage has just converted, which reproduces the same Ucat, so it is
  // skipped here as at the start of stages 2-4.
  if (c->g.bc[5] == 4 && (rc = outlet_rescale(c))) return rc;
  return form_bcs_tail(c);
}


// ------------------------------------------------------------------ tangent / adjoint of a stage
// Linearisation of one RK stage  Ucont' = pUcont + a*(Formfunction_2(Ucont, Ucat) - dP)
// (les = 0) about the recorded stage input (uc, u): the face fluxes are linear in Ucat for
// a fixed Ucont and, through the convecting flux, linear in Ucont (piecewise through the
// upwind weights of the QUICK faces).  The tangent computes the face-flux tangents and
// runs the forward Fp and right-hand-side kernels on them; the adjoint mirrors k_rhs,
// k_fp and the face loops in reverse, scattering with atomics.

// Up to four (index, weight) pairs: one computational-space difference of a face.
struct DiffW { long long idx[4]; double w[4]; int n; };

__device__ __forceinline__ void cross_desc(long long a0, long long a1, long long bp0, long long bp1, long long bm0,
                                           long long bm1, bool ps, bool ms, DiffW &d) {
  d.n = 4;
  if (ps) {
    d.idx[0] = a1; d.idx[1] = a0; d.idx[2] = bm1; d.idx[3] = bm0;
    d.w[0] = 0.5; d.w[1] = 0.5; d.w[2] = -0.5; d.w[3] = -0.5;
  } else if (ms) {
    d.idx[0] = bp1; d.idx[1] = bp0; d.idx[2] = a1; d.idx[3] = a0;
    d.w[0] = 0.5; d.w[1] = 0.5; d.w[2] = -0.5; d.w[3] = -0.5;
  } else {
    d.idx[0] = bp1; d.idx[1] = bp0; d.idx[2] = bm1; d.idx[3] = bm0;
    d.w[0] = 0.25; d.w[1] = 0.25; d.w[2] = -0.25; d.w[3] = -0.25;
  }
}

// Everything the face of direction D at point p (index qd along D) reads, as the face
// loops of flux_i / flux_j / flux_k read it.
struct FaceLin {
  DiffW dw[3];                 // d/dcsi, d/deta, d/dzeta of each velocity component
  double cs[3], et[3], ze[3];  // face metrics
  double nrm[3];               // the face's own metric (csi, eta or zet)
  double g[3];                 // g11, g21, g31 of the face
  double K;                    // ajc * nu
  int mode;                    // 0 central, 1 QUICK A, 2 QUICK B, 3 no convective flux
  long long cidx[4];           // central: pL, p, p+s, pR; QUICK: the three cells
  long long pcu, pucon;        // convecting flux (central) and upwinding flux (QUICK)
};

__device__ __forceinline__ void face_lin(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv, int D,
                                         long long p, int i, int j, int k, FaceLin &F) {
  const long long st[3] = {1, (long long)g.mx, (long long)g.mx * g.my};
  const long long s = st[D];
  const int qd = D == 0 ? i : (D == 1 ? j : k);
  const int mm = D == 0 ? g.mx : (D == 1 ? g.my : g.mz);
  const int per = D == 0 ? g.iper : (D == 1 ? g.jper : g.kper);
  CV3 mc = D == 0 ? m.icsi : (D == 1 ? m.jcsi : m.kcsi);
  CV3 me = D == 0 ? m.ieta : (D == 1 ? m.jeta : m.keta);
  CV3 mz = D == 0 ? m.izet : (D == 1 ? m.jzet : m.kzet);
  const double *aj = D == 0 ? m.iaj : (D == 1 ? m.jaj : m.kaj);
  F.cs[0] = mc.x[p]; F.cs[1] = mc.y[p]; F.cs[2] = mc.z[p];
  F.et[0] = me.x[p]; F.et[1] = me.y[p]; F.et[2] = me.z[p];
  F.ze[0] = mz.x[p]; F.ze[1] = mz.y[p]; F.ze[2] = mz.z[p];
  const double *n = D == 0 ? F.cs : (D == 1 ? F.et : F.ze);
  for (int a = 0; a < 3; a++) F.nrm[a] = n[a];
  F.g[0] = F.cs[0] * n[0] + F.cs[1] * n[1] + F.cs[2] * n[2];
  F.g[1] = F.et[0] * n[0] + F.et[1] * n[1] + F.et[2] * n[2];
  F.g[2] = F.ze[0] * n[0] + F.ze[1] * n[1] + F.ze[2] * n[2];
  F.K = aj[p] * (1. / g.ren);
  for (int E = 0; E < 3; E++) {
    if (E == D) {
      F.dw[E].n = 2;
      F.dw[E].idx[0] = p + s; F.dw[E].w[0] = 1.0;
      F.dw[E].idx[1] = p; F.dw[E].w[1] = -1.0;
    } else {
      const long long t = st[E];
      cross_desc(p, p + s, p + t, p + t + s, p - t, p - t + s, nv[p + t] > 0 || nv[p + t + s] > 0,
                 nv[p - t] > 0 || nv[p - t + s] > 0, F.dw[E]);
    }
  }
  int qL = qd - 1, qR = qd + 2;
  if (qd == 0 || qd == mm - 2) {
    if (per) qL = mm - 3, qR = 2;
    else qL = qd, qR = qd + 1;
  } else if (nv[p - s] + nv[p + 2 * s] > 0) qL = qd, qR = qd + 1;
  F.pucon = p;
  if (per && (qd == 0 || qd == mm - 2)) F.pucon = p + (long long)(mm - 2 - qd) * s;
  if (D == 2 && qd == mm - 2 && g.bc[5] == 4 && nv[p] == 0) F.pucon = p - s;
  F.pcu = p;
  if (g.immersed && qd != mm - 2 && nv[p] > 0) {
    F.mode = 1; F.cidx[0] = p; F.cidx[1] = p + s; F.cidx[2] = p + 2 * s;
  } else if (g.immersed && qd != 0 && nv[p + s] > 0) {
    F.mode = 2; F.cidx[0] = p - s; F.cidx[1] = p; F.cidx[2] = p + s;
  } else {
    F.mode = 0;
    F.cidx[0] = p + (long long)(qL - qd) * s; F.cidx[1] = p; F.cidx[2] = p + s;
    F.cidx[3] = p + (long long)(qR - qd) * s;
  }
  if (nv[p] + nv[p + s] > 0 && !g.immersed) F.mode = 3;
}

__device__ __forceinline__ double comp(CV3 v, int c, long long p) { return c == 0 ? v.x[p] : (c == 1 ? v.y[p] : v.z[p]); }
__device__ __forceinline__ double *compp(V3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// QUICK coefficients: d = um*A + up*B with A, B linear in the three cells (variant A
// cells u0 u1 u2 = p, p+s, p+2s; variant B cells um1 u0 u1 = p-s, p, p+s).
__device__ __forceinline__ void quick_ab(int mode, double x0, double x1, double x2, double &A, double &B,
                                         double dA[3], double dB[3]) {
  if (mode == 1) {
    A = 0.125 * (-x2 - 2. * x1 + 3. * x0) + x1; B = 0.125 * (-x0 - 2. * x0 + 3. * x1) + x0;
    dA[0] = 0.375; dA[1] = 0.75; dA[2] = -0.125;
    dB[0] = 0.625; dB[1] = 0.375; dB[2] = 0.0;
  } else {
    A = 0.125 * (-x2 - 2. * x2 + 3. * x1) + x2; B = 0.125 * (-x0 - 2. * x1 + 3. * x2) + x1;
    dA[0] = 0.0; dA[1] = 0.375; dA[2] = 0.625;
    dB[0] = -0.125; dB[1] = 0.75; dB[2] = 0.375;
  }
}

// Tangent face fluxes of direction D at p: delta d (3) and delta v (3).
__device__ __forceinline__ void face_tangent(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv, int D,
                                             long long p, int i, int j, int k, CV3 uc, CV3 u, CV3 duc, CV3 du,
                                             double dd[3], double dv[3]) {
  FaceLin F;
  face_lin(g, m, nv, D, p, i, j, k, F);
  double dg[3][3];  // [E][component]
  for (int E = 0; E < 3; E++)
    for (int c = 0; c < 3; c++) {
      double s = 0;
      for (int t = 0; t < F.dw[E].n; t++) s += F.dw[E].w[t] * comp(du, c, F.dw[E].idx[t]);
      dg[E][c] = s;
    }
  const double *mt[3] = {F.cs, F.et, F.ze};
  for (int c = 0; c < 3; c++) {
    double v = F.g[0] * dg[0][c] + F.g[1] * dg[1][c] + F.g[2] * dg[2][c];
    for (int a = 0; a < 3; a++) {
      const double r = dg[0][a] * mt[0][c] + dg[1][a] * mt[1][c] + dg[2][a] * mt[2][c];
      v += r * F.nrm[a];
    }
    dv[c] = v * F.K;
  }
  const double *ucD = D == 0 ? uc.x : (D == 1 ? uc.y : uc.z);
  const double *ducD = D == 0 ? duc.x : (D == 1 ? duc.y : duc.z);
  for (int c = 0; c < 3; c++) dd[c] = 0;
  if (F.mode == 0) {
    const double cu = ucD[F.pcu], dcu = ducD[F.pcu];
    for (int c = 0; c < 3; c++) {
      const double S = -comp(u, c, F.cidx[0]) + 9. * comp(u, c, F.cidx[1]) + 9. * comp(u, c, F.cidx[2]) -
                       comp(u, c, F.cidx[3]);
      const double dS = -comp(du, c, F.cidx[0]) + 9. * comp(du, c, F.cidx[1]) + 9. * comp(du, c, F.cidx[2]) -
                        comp(du, c, F.cidx[3]);
      dd[c] = -dcu * 0.0625 * S - cu * 0.0625 * dS;
    }
  } else if (F.mode != 3) {
    const double ucon = ucD[F.pucon], ducon = ducD[F.pucon];
    const double up = -0.5 * (ucon + fabs(ucon)), um = -0.5 * (ucon - fabs(ucon));
    const double sg = ucon > 0 ? 1. : (ucon < 0 ? -1. : 0.);
    const double dum = -0.5 * (1. - sg) * ducon, dup = -0.5 * (1. + sg) * ducon;
    for (int c = 0; c < 3; c++) {
      double A, B, dA[3], dB[3];
      quick_ab(F.mode, comp(u, c, F.cidx[0]), comp(u, c, F.cidx[1]), comp(u, c, F.cidx[2]), A, B, dA, dB);
      double dAv = 0, dBv = 0;
      for (int t = 0; t < 3; t++) {
        const double x = comp(du, c, F.cidx[t]);
        dAv += dA[t] * x; dBv += dB[t] * x;
      }
      dd[c] = dum * A + dup * B + um * dAv + up * dBv;
    }
  }
}

// Adjoint of the face of direction D at p: scatters lambda_d (3) and lambda_v (3) onto
// the Ucont (luc) and Ucat (lu) adjoints.
__device__ __forceinline__ void face_adjoint(const Grid &g, const Metrics &m, const uint8_t *__restrict__ nv, int D,
                                             long long p, int i, int j, int k, CV3 uc, CV3 u, const double ld[3],
                                             const double lv[3], V3 luc, V3 lu) {
  FaceLin F;
  face_lin(g, m, nv, D, p, i, j, k, F);
  double lg[3][3] = {};  // adjoint of the differences [E][component]
  const double *mt[3] = {F.cs, F.et, F.ze};
  for (int c = 0; c < 3; c++) {
    const double t = lv[c] * F.K;
    if (t == 0) continue;
    lg[0][c] += F.g[0] * t; lg[1][c] += F.g[1] * t; lg[2][c] += F.g[2] * t;
    for (int a = 0; a < 3; a++) {
      const double ta = t * F.nrm[a];
      lg[0][a] += mt[0][c] * ta; lg[1][a] += mt[1][c] * ta; lg[2][a] += mt[2][c] * ta;
    }
  }
  for (int E = 0; E < 3; E++)
    for (int c = 0; c < 3; c++) {
      if (lg[E][c] == 0) continue;
      double *dst = compp(lu, c);
      for (int t = 0; t < F.dw[E].n; t++) atomicAdd(dst + F.dw[E].idx[t], F.dw[E].w[t] * lg[E][c]);
    }
  const double *ucD = D == 0 ? uc.x : (D == 1 ? uc.y : uc.z);
  double *lucD = D == 0 ? luc.x : (D == 1 ? luc.y : luc.z);
  if (F.mode == 0) {
    const double cu = ucD[F.pcu];
    double lcu = 0;
    for (int c = 0; c < 3; c++) {
      if (ld[c] == 0) continue;
      const double S = -comp(u, c, F.cidx[0]) + 9. * comp(u, c, F.cidx[1]) + 9. * comp(u, c, F.cidx[2]) -
                       comp(u, c, F.cidx[3]);
      lcu += -0.0625 * S * ld[c];
      const double w = -cu * 0.0625 * ld[c];
      double *dst = compp(lu, c);
      atomicAdd(dst + F.cidx[0], -w);
      atomicAdd(dst + F.cidx[1], 9. * w);
      atomicAdd(dst + F.cidx[2], 9. * w);
      atomicAdd(dst + F.cidx[3], -w);
    }
    if (lcu != 0) atomicAdd(lucD + F.pcu, lcu);
  } else if (F.mode != 3) {
    const double ucon = ucD[F.pucon];
    const double up = -0.5 * (ucon + fabs(ucon)), um = -0.5 * (ucon - fabs(ucon));
    const double sg = ucon > 0 ? 1. : (ucon < 0 ? -1. : 0.);
    double lum = 0, lup = 0;
    for (int c = 0; c < 3; c++) {
      if (ld[c] == 0) continue;
      double A, B, dA[3], dB[3];
      quick_ab(F.mode, comp(u, c, F.cidx[0]), comp(u, c, F.cidx[1]), comp(u, c, F.cidx[2]), A, B, dA, dB);
      lum += A * ld[c]; lup += B * ld[c];
      double *dst = compp(lu, c);
      for (int t = 0; t < 3; t++) {
        const double w = (um * dA[t] + up * dB[t]) * ld[c];
        if (w != 0) atomicAdd(dst + F.cidx[t], w);
      }
    }
    const double lucon = lum * (-0.5 * (1. - sg)) + lup * (-0.5 * (1. + sg));
    if (lucon != 0) atomicAdd(lucD + F.pucon, lucon);
  }
}

struct FaceBank { double *f[3][6]; };

__global__ void k_tan_face(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 uc, CV3 u, CV3 duc, CV3 du,
                           FaceBank out) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i == g.mx - 1 || j == g.my - 1 || k == g.mz - 1) return;
  const bool on[3] = {j != 0 && k != 0, i != 0 && k != 0, i != 0 && j != 0};
  for (int D = 0; D < 3; D++) {
    if (!on[D]) continue;
    double dd[3], dv[3];
    face_tangent(g, m, nv, D, p, i, j, k, uc, u, duc, du, dd, dv);
    for (int c = 0; c < 3; c++) { out.f[D][c][p] = dd[c]; out.f[D][3 + c][p] = dv[c]; }
  }
}

__global__ void k_adj_face(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 uc, CV3 u, FaceBank lf, V3 luc,
                           V3 lu) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i == g.mx - 1 || j == g.my - 1 || k == g.mz - 1) return;
  const bool on[3] = {j != 0 && k != 0, i != 0 && k != 0, i != 0 && j != 0};
  for (int D = 0; D < 3; D++) {
    if (!on[D]) continue;
    double ld[3], lv[3];
    bool any = false;
    for (int c = 0; c < 3; c++) {
      ld[c] = lf.f[D][c][p]; lv[c] = lf.f[D][3 + c][p];
      any |= ld[c] != 0 || lv[c] != 0;
    }
    if (any) face_adjoint(g, m, nv, D, p, i, j, k, uc, u, ld, lv, luc, lu);
  }
}

// Adjoint of fp_cell: lambda_Fp of each interior cell onto the face-flux adjoints it read.
__global__ void k_adj_fp(Grid g, const uint8_t *__restrict__ nv, const double *__restrict__ lfx,
                         const double *__restrict__ lfy, const double *__restrict__ lfz, FaceBank lf) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) return;
  const double l[3] = {lfx[p], lfy[p], lfz[p]};
  if (l[0] == 0 && l[1] == 0 && l[2] == 0) return;
  const long long sy = mx, sz = (long long)mx * my;
  int oR[3], oL[3];
  double den[3];
  fp_offsets(i, mx, g.iper, nv[p - 1] + nv[p] + nv[p + 1], oR[0], oL[0], den[0]);
  fp_offsets(j, my, g.jper, nv[p - sy] + nv[p] + nv[p + sy], oR[1], oL[1], den[1]);
  fp_offsets(k, mz, g.kper, nv[p - sz] + nv[p] + nv[p + sz], oR[2], oL[2], den[2]);
  const long long row[3] = {p - i, p - (long long)j * mx, p - (long long)k * mx * my};
  const int idx[3] = {i, j, k};
  const int ext[3] = {mx, my, mz};
  const int per[3] = {g.iper, g.jper, g.kper};
  const long long str[3] = {1, sy, sz};
  for (int D = 0; D < 3; D++) {
    auto at = [&](int off) { return row[D] + (long long)face_image(idx[D] + off, ext[D], per[D]) * str[D]; };
    const long long f0 = at(0), fm = at(-1), fR = at(oR[D]), fL = at(oL[D]);
    const double wide = -1. / 8. * (1. / den[D]);
    for (int c = 0; c < 3; c++) {
      if (l[c] == 0) continue;
      atomicAdd(lf.f[D][c] + f0, 9. / 8. * l[c]);
      atomicAdd(lf.f[D][c] + fm, -9. / 8. * l[c]);
      atomicAdd(lf.f[D][c] + fR, wide * l[c]);
      atomicAdd(lf.f[D][c] + fL, -wide * l[c]);
      atomicAdd(lf.f[D][3 + c] + f0, l[c]);
      atomicAdd(lf.f[D][3 + c] + fm, -l[c]);
    }
  }
}

// Adjoint of rhs_point in RK mode (scale 1): lambda of the stage output Ucont' onto
// pUcont, dP and Fp.
__global__ void k_adj_rhs(Grid g, Metrics m, const uint8_t *__restrict__ nv, double a, CV3 lU, V3 lpu, V3 ldp,
                          double *lfx, double *lfy, double *lfz) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i, j, k;
  dijk(g, p, i, j, k);
  const double l0 = lU.x[p], l1 = lU.y[p], l2 = lU.z[p];
  lpu.x[p] += l0; lpu.y[p] += l1; lpu.z[p] += l2;
  ldp.x[p] -= a * l0; ldp.y[p] -= a * l1; ldp.z[p] -= a * l2;
  const bool ghost = i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1;
  if (ghost) return;
  const long long sy = mx, sz = (long long)mx * my;
  double r0 = a * l0, r1 = a * l1, r2 = a * l2;
  if (nv[p] + nv[p + 1] > 0 || (!g.iper && i == mx - 2)) r0 = 0;
  if (nv[p] + nv[p + sy] > 0 || (!g.jper && j == my - 2)) r1 = 0;
  if (nv[p] + nv[p + sz] > 0 || (!g.kper && k == mz - 2)) r2 = 0;
  const long long q1 = (g.iper && i == mx - 2) ? p - i + 1 : p + 1;
  const long long q2 = (g.jper && j == my - 2) ? p - (long long)j * sy + sy : p + sy;
  const long long q3 = (g.kper && k == mz - 2) ? p - (long long)k * sz + sz : p + sz;
  double *lf[3] = {lfx, lfy, lfz};
  if (r0 != 0) {
    const double w = 0.5 * m.iaj[p] * r0;
    const double a0[3] = {m.csi.x[p], m.csi.y[p], m.csi.z[p]}, a1[3] = {m.csi.x[p + 1], m.csi.y[p + 1], m.csi.z[p + 1]};
    for (int c = 0; c < 3; c++) { atomicAdd(lf[c] + p, w * a0[c]); atomicAdd(lf[c] + q1, w * a1[c]); }
  }
  if (r1 != 0) {
    const double w = 0.5 * m.jaj[p] * r1;
    const double a0[3] = {m.eta.x[p], m.eta.y[p], m.eta.z[p]};
    const double a1[3] = {m.eta.x[p + sy], m.eta.y[p + sy], m.eta.z[p + sy]};
    for (int c = 0; c < 3; c++) { atomicAdd(lf[c] + p, w * a0[c]); atomicAdd(lf[c] + q2, w * a1[c]); }
  }
  if (r2 != 0) {
    const double w = 0.5 * m.kaj[p] * r2;
    const double a0[3] = {m.zet.x[p], m.zet.y[p], m.zet.z[p]};
    const double a1[3] = {m.zet.x[p + sz], m.zet.y[p + sz], m.zet.z[p + sz]};
    for (int c = 0; c < 3; c++) { atomicAdd(lf[c] + p, w * a0[c]); atomicAdd(lf[c] + q3, w * a1[c]); }
  }
}

// Tangent of one stage: dU (in: tangent of the stage input; out: of the stage output).
int ff2_stage_tangent(Ctx *c, const double *const uc[3], const double *const uk[3], double a, V3 dU, V3 du, V3 ddp,
                      V3 dpu, double *const tf[3][6]) {
  const Grid &g = c->g;
  int rc;
  if ((rc = periodic_copy3(c, dU))) return rc;
  FaceBank fb;
  for (int d = 0; d < 3; d++)
    for (int q = 0; q < 6; q++) fb.f[d][q] = tf[d][q];
  Metrics m = metrics(c);
  CV3 ucb{uc[0], uc[1], uc[2]}, ukb{uk[0], uk[1], uk[2]};
  c->launches++, k_tan_face<<<nblocks(g.N, 128), 128, 0, c->stream>>>(g, m, c->nv, ucb, ukb, cv(dU), cv(du), fb);
  if ((rc = check_launch(c, "k_tan_face"))) return rc;
  FluxIn f[3];
  for (int d = 0; d < 3; d++)
    for (int q = 0; q < 3; q++) { f[d].div[q] = tf[d][q]; f[d].visc[q] = tf[d][3 + q]; }
  c->launches++, k_fp<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, f[0], f[1], f[2], c->nv, c->fp[0], c->fp[1], c->fp[2]);
  if ((rc = check_launch(c, "k_fp"))) return rc;
  c->launches++, k_rhs<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, c->fp[0], c->fp[1], c->fp[2], 1.0, field3(c, VFS_RHS),
                                                 1, a, cv(ddp), cv(dpu), dU);
  return check_launch(c, "k_rhs");
}

// Adjoint of one stage: lU (in: adjoint of the stage output; out: of the stage input),
// lu (Ucat adjoint), ldp and lpu accumulate.
int ff2_stage_adjoint(Ctx *c, const double *const uc[3], const double *const uk[3], double a, V3 lU, V3 lu, V3 ldp,
                      V3 lpu, double *const lf[3][6], double *const lfp[3]) {
  const Grid &g = c->g;
  const size_t bytes = sizeof(double) * g.N;
  int rc;
  for (int d = 0; d < 3; d++) {
    cudaMemsetAsync(lfp[d], 0, bytes, c->stream);
    for (int q = 0; q < 6; q++) cudaMemsetAsync(lf[d][q], 0, bytes, c->stream);
  }
  Metrics m = metrics(c);
  c->launches++, k_adj_rhs<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, a, cv(lU), lpu, ldp, lfp[0], lfp[1], lfp[2]);
  if ((rc = check_launch(c, "k_adj_rhs"))) return rc;
  cudaMemsetAsync(lU.x, 0, bytes, c->stream);
  cudaMemsetAsync(lU.y, 0, bytes, c->stream);
  cudaMemsetAsync(lU.z, 0, bytes, c->stream);
  FaceBank fb;
  for (int d = 0; d < 3; d++)
    for (int q = 0; q < 6; q++) fb.f[d][q] = lf[d][q];
  c->launches++, k_adj_fp<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nv, lfp[0], lfp[1], lfp[2], fb);
  if ((rc = check_launch(c, "k_adj_fp"))) return rc;
  CV3 ucb{uc[0], uc[1], uc[2]}, ukb{uk[0], uk[1], uk[2]};
  c->launches++, k_adj_face<<<nblocks(g.N, 128), 128, 0, c->stream>>>(g, m, c->nv, ucb, ukb, fb, lU, lu);
  if ((rc = check_launch(c, "k_adj_face"))) return rc;
  return periodic_copy3_adjoint(c, lU);
}

}  // namespace vfs
