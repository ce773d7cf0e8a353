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
  k_periodic_copy<<<nblocks(ghost_points(c->g), 256), 256, 0, c->stream>>>(c->g, v.x, v.y, v.z);
  return check_launch(c, "k_periodic_copy");
}
int periodic_copy1(Ctx *c, double *s) {
  if (!(c->g.iper || c->g.jper || c->g.kper)) return VFS_OK;
  k_periodic_copy<<<nblocks(ghost_points(c->g), 256), 256, 0, c->stream>>>(c->g, s, nullptr, nullptr);
  return check_launch(c, "k_periodic_copy");
}

// ------------------------------------------------------------------ Contra2Cart
// Interior Cartesian velocity from averaged face fluxes by Cramer's rule on the centre
// metrics (rhs.c:186-233).  Cells with nvert >= 0.1 keep their value.
__global__ void k_contra2cart_interior(Grid g, CV3 uc, CV3 csi, CV3 eta, CV3 zet,
                                       const uint8_t *__restrict__ nv, V3 ucat) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i = (int)(p % g.mx);
  long long q = p / g.mx;
  int j = (int)(q % g.my);
  int k = (int)(q / g.my);
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

// Slip-wall ghost: mirror the neighbour's old velocity about the wall normal taken from
// the covariant metric column `col` of the neighbour cell (rhs.c:384-478).
__device__ void slip_ghost(long long nb, int col, double sgn, Metrics m, CV3 uo, double *o) {
  double g[3][3], G[3][3];
  g[0][0] = m.csi.x[nb], g[0][1] = m.csi.y[nb], g[0][2] = m.csi.z[nb];
  g[1][0] = m.eta.x[nb], g[1][1] = m.eta.y[nb], g[1][2] = m.eta.z[nb];
  g[2][0] = m.zet.x[nb], g[2][1] = m.zet.y[nb], g[2][2] = m.zet.z[nb];
  covariant(g, G);
  double nx = G[0][col], ny = G[1][col], nz = G[2][col];
  if (sgn < 0) nx = -nx, ny = -ny, nz = -nz;
  double sum = sqrt(nx * nx + ny * ny + nz * nz);
  nx /= sum, ny /= sum, nz /= sum;
  double un = uo.x[nb] * nx + uo.y[nb] * ny + uo.z[nb] * nz;
  o[0] = uo.x[nb] - 2 * un * nx;
  o[1] = uo.y[nb] - 2 * un * ny;
  o[2] = uo.z[nb] - 2 * un * nz;
}

// Boundary part of Contra2Cart_2 (rhs.c:291-675), phase 1: every point the reference's
// boundary loop assigns gets its new value in `out` (reads the pre-loop snapshot `ucat`),
// `flag` marks it.  Phase 2 (k_bc_commit) copies the marked values, which reproduces the
// reference's read-from-lUcat / write-to-Ucat semantics exactly.
__global__ void k_contra2cart_bc(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 lu,
                                 CV3 uo, V3 out, uint8_t *flag) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const int *bc = g.bc;
  bool w = false;
  if (nv[p] == 3) {  // (int)(nvert+0.1)==3 and fixed bodies (rhs.c:296-299)
    out.x[p] = 0; out.y[p] = 0; out.z[p] = 0;
    flag[p] = 1;
    return;
  }
  // every rule below acts on a ghost point or on a cell (1 or mx-2, 1, k)
  if (!(i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1 ||
        (j == 1 && (i == 1 || i == mx - 2))))
    return;
  double v[3] = {lu.x[p], lu.y[p], lu.z[p]};
  int solid_flag = 0;
  if (bc[3] == 13 && j == my - 1) {
    v[0] = lu.x[p - sy]; v[2] = lu.z[p - sy]; v[1] = -lu.y[p - sy]; w = true;
  }
  if (bc[3] == 14 && j == my - 1) {
    v[0] = lu.x[p - sy]; v[1] = lu.y[p - sy]; v[2] = -lu.z[p - sy]; w = true;
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
    v[0] = -1 * lu.x[p + sx]; v[1] = -1 * lu.y[p + sx]; v[2] = -1 * lu.z[p + sx]; w = true; solid_flag = 1;
  }
  if (i == mx - 1 && bc[1] == 1 && (j != 0 && k != 0)) {
    v[0] = -1 * lu.x[p - sx]; v[1] = -1 * lu.y[p - sx]; v[2] = -1 * lu.z[p - sx]; w = true; solid_flag = 1;
  }
  if (j == 0 && bc[2] == 1 && (i != 0 && k != 0)) {
    v[0] = -1 * lu.x[p + sy]; v[1] = -1 * lu.y[p + sy]; v[2] = -1 * lu.z[p + sy]; w = true; solid_flag = 1;
  }
  if (j == my - 1 && bc[3] == 1 && (i != 0 && k != 0)) {
    v[0] = -1 * lu.x[p - sy]; v[1] = -1 * lu.y[p - sy]; v[2] = -1 * lu.z[p - sy]; w = true; solid_flag = 1;
  }
  if (k == 0 && bc[4] == 1 && (i != 0 && j != 0)) {
    v[0] = -1 * lu.x[p + sz]; v[1] = -1 * lu.y[p + sz]; v[2] = -1 * lu.z[p + sz]; w = true; solid_flag = 1;
  }
  if (k == mz - 1 && bc[5] == 1 && (i != 0 && j != 0)) {
    v[0] = -1 * lu.x[p - sz]; v[1] = -1 * lu.y[p - sz]; v[2] = -1 * lu.z[p - sz]; w = true; solid_flag = 1;
  }
  if (j == my - 1 && bc[3] == 2) {
    if (solid_flag) { v[0] = 2.0 - uo.x[p - sy]; v[1] = -uo.y[p - sy]; v[2] = -uo.z[p - sy]; }
    else { v[0] = 2.0 - lu.x[p - sy]; v[1] = -lu.y[p - sy]; v[2] = -lu.z[p - sy]; }
    w = true;
  }
  if (j == 0 && bc[2] == 12) {
    v[0] = -lu.x[p + sy]; v[1] = -lu.y[p + sy]; v[2] = 2.0 - lu.z[p + sy]; w = true;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  if (j == my - 1 && bc[3] == 12) {
    v[0] = -lu.x[p - sy]; v[1] = -lu.y[p - sy]; v[2] = 2.0 - lu.z[p - sy]; w = true;
    if (solid_flag) v[0] = v[1] = v[2] = 0;
  }
  // outflow (rhs.c:573-597)
  if (bc[3] == 4 && j == my - 1 && (i != 0 && i != mx - 1 && k != 0 && k != mz - 1)) {
    v[0] = lu.x[p - sy]; v[1] = lu.y[p - sy]; v[2] = lu.z[p - sy]; w = true;
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
  if (w) {
    out.x[p] = v[0]; out.y[p] = v[1]; out.z[p] = v[2];
    flag[p] = 1;
  }
}

__global__ void k_bc_commit(long long n, CV3 in, uint8_t *flag, V3 dst) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (!flag[p]) return;
  dst.x[p] = in.x[p]; dst.y[p] = in.y[p]; dst.z[p] = in.z[p];
  flag[p] = 0;
}

int contra2cart(Ctx *c) {
  const Grid &g = c->g;
  V3 uc = field3(c, VFS_UCONT), ucat = field3(c, VFS_UCAT);
  int rc;
  if ((rc = periodic_copy3(c, uc))) return rc;
  Metrics m = metrics(c);
  k_contra2cart_interior<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, cv(uc), m.csi, m.eta, m.zet, c->nv, ucat);
  if ((rc = check_launch(c, "k_contra2cart_interior"))) return rc;
  if ((rc = periodic_copy3(c, ucat))) return rc;
  V3 out{c->bcbuf[0], c->bcbuf[1], c->bcbuf[2]};
  uint8_t *fl = c->bcflag;
  k_contra2cart_bc<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, cv(ucat), cv(field3(c, VFS_UCAT_O)), out, fl);
  if ((rc = check_launch(c, "k_contra2cart_bc"))) return rc;
  k_bc_commit<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g.N, cv(out), fl, ucat);
  if ((rc = check_launch(c, "k_bc_commit"))) return rc;
  return periodic_copy3(c, ucat);
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

// One thread per DA point (i,j,k) with i<mx-1, j<my-1, k<mz-1: computes the fluxes of
// its i-face (if j,k >= 1), j-face (if i,k >= 1) and k-face (if i,j >= 1), following
// the three face loops of Formfunction_2 (momentum.c:671-1415).
__global__ void k_face_flux(Grid g, Metrics m, CV3 uc, CV3 u, const uint8_t *__restrict__ nv,
                            const double *__restrict__ nut, FluxOut f1, FluxOut f2, FluxOut f3) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  if (i == mx - 1 || j == my - 1 || k == mz - 1) return;
  const long long sx = 1, sy = mx, sz = (long long)mx * my;
  const double nu = 1. / g.ren;
  const bool les = g.les != 0;

  // ---------------- i direction
  if (j != 0 && k != 0) {
    const double ajc = m.iaj[p];
    const double csi0 = m.icsi.x[p], csi1 = m.icsi.y[p], csi2 = m.icsi.z[p];
    const double eta0 = m.ieta.x[p], eta1 = m.ieta.y[p], eta2 = m.ieta.z[p];
    const double zet0 = m.izet.x[p], zet1 = m.izet.y[p], zet2 = m.izet.z[p];
    double dc[3], de[3], dz[3];
    dc[0] = u.x[p + sx] - u.x[p]; dc[1] = u.y[p + sx] - u.y[p]; dc[2] = u.z[p + sx] - u.z[p];
    cross_diff(u, p, p + sx, p + sy, p + sy + sx, p - sy, p - sy + sx,
               nv[p + sy] > 0 || nv[p + sy + sx] > 0, nv[p - sy] > 0 || nv[p - sy + sx] > 0, de);
    cross_diff(u, p, p + sx, p + sz, p + sz + sx, p - sz, p - sz + sx,
               nv[p + sz] > 0 || nv[p + sz + sx] > 0, nv[p - sz] > 0 || nv[p - sz + sx] > 0, dz);
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
    if (i == 0 || i == mx - 2) {
      if (g.iper) iL = mx - 3, iR = 2;
      else iL = i, iR = i + 1;
    } else if (nv[p - 1] + nv[p + 2] > 0) iL = i, iR = i + 1;
    double ucon = uc.x[p];
    if (g.iper && (i == 0 || i == mx - 2)) ucon = uc.x[p - i + (mx - 2)];
    const double up = -0.5 * (ucon + fabs(ucon));
    const double um = -0.5 * (ucon - fabs(ucon));
    const long long pL = p - i + iL, pR = p - i + iR;
    double d[3];
    if (g.immersed && i != mx - 2 && nv[p] > 0) {
      d[0] = quick_a(um, up, u.x[p], u.x[p + 1], u.x[p + 2]);
      d[1] = quick_a(um, up, u.y[p], u.y[p + 1], u.y[p + 2]);
      d[2] = quick_a(um, up, u.z[p], u.z[p + 1], u.z[p + 2]);
    } else if (g.immersed && i != 0 && nv[p + 1] > 0) {
      d[0] = quick_b(um, up, u.x[p - 1], u.x[p], u.x[p + 1]);
      d[1] = quick_b(um, up, u.y[p - 1], u.y[p], u.y[p + 1]);
      d[2] = quick_b(um, up, u.z[p - 1], u.z[p], u.z[p + 1]);
    } else {
      const double cu = uc.x[p];
      d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + 1] - u.x[pR]);
      d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + 1] - u.y[pR]);
      d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + 1] - u.z[pR]);
    }
    if (nv[p] + nv[p + 1] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
    double v[3] = {0, 0, 0};
    if (les) {
      double nut_f;
      if ((i == 0 && !g.iper) || nv[p] > 0) nut_f = nut[p + 1];
      else if ((i == mx - 2 && !g.iper) || nv[p + 1] > 0) nut_f = nut[p];
      else nut_f = 0.5 * (nut[p] + nut[p + 1]);
      v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, csi0, csi1, csi2, ajc, nut_f);
      v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, csi0, csi1, csi2, ajc, nut_f);
      v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, csi0, csi1, csi2, ajc, nut_f);
    }
    v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, csi0, csi1, csi2, ajc, nu);
    v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, csi0, csi1, csi2, ajc, nu);
    v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, csi0, csi1, csi2, ajc, nu);
    f1.div[0][p] = d[0]; f1.div[1][p] = d[1]; f1.div[2][p] = d[2];
    f1.visc[0][p] = v[0]; f1.visc[1][p] = v[1]; f1.visc[2][p] = v[2];
  }

  // ---------------- j direction
  if (i != 0 && k != 0) {
    const double ajc = m.jaj[p];
    const double csi0 = m.jcsi.x[p], csi1 = m.jcsi.y[p], csi2 = m.jcsi.z[p];
    const double eta0 = m.jeta.x[p], eta1 = m.jeta.y[p], eta2 = m.jeta.z[p];
    const double zet0 = m.jzet.x[p], zet1 = m.jzet.y[p], zet2 = m.jzet.z[p];
    double dc[3], de[3], dz[3];
    cross_diff(u, p, p + sy, p + sx, p + sy + sx, p - sx, p + sy - sx,
               nv[p + sx] > 0 || nv[p + sy + sx] > 0, nv[p - sx] > 0 || nv[p + sy - sx] > 0, dc);
    de[0] = u.x[p + sy] - u.x[p]; de[1] = u.y[p + sy] - u.y[p]; de[2] = u.z[p + sy] - u.z[p];
    cross_diff(u, p, p + sy, p + sz, p + sz + sy, p - sz, p - sz + sy,
               nv[p + sz] > 0 || nv[p + sz + sy] > 0, nv[p - sz] > 0 || nv[p - sz + sy] > 0, dz);
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
    if (j == 0 || j == my - 2) {
      if (g.jper) jL = my - 3, jR = 2;
      else jL = j, jR = j + 1;
    } else if (nv[p - sy] + nv[p + 2 * sy] > 0) jL = j, jR = j + 1;
    double ucon = uc.y[p];
    if (g.jper && (j == 0 || j == my - 2)) ucon = uc.y[p + (long long)(my - 2 - j) * sy];
    const double up = -0.5 * (ucon + fabs(ucon));
    const double um = -0.5 * (ucon - fabs(ucon));
    const long long pL = p + (long long)(jL - j) * sy, pR = p + (long long)(jR - j) * sy;
    double d[3];
    if (g.immersed && j != my - 2 && nv[p] > 0) {
      d[0] = quick_a(um, up, u.x[p], u.x[p + sy], u.x[p + 2 * sy]);
      d[1] = quick_a(um, up, u.y[p], u.y[p + sy], u.y[p + 2 * sy]);
      d[2] = quick_a(um, up, u.z[p], u.z[p + sy], u.z[p + 2 * sy]);
    } else if (g.immersed && j != 0 && nv[p + sy] > 0) {
      d[0] = quick_b(um, up, u.x[p - sy], u.x[p], u.x[p + sy]);
      d[1] = quick_b(um, up, u.y[p - sy], u.y[p], u.y[p + sy]);
      d[2] = quick_b(um, up, u.z[p - sy], u.z[p], u.z[p + sy]);
    } else {
      const double cu = uc.y[p];
      d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + sy] - u.x[pR]);
      d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + sy] - u.y[pR]);
      d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + sy] - u.z[pR]);
    }
    if (nv[p] + nv[p + sy] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
    double v[3] = {0, 0, 0};
    if (les) {
      double nut_f;
      if ((j == 0 && !g.jper) || nv[p] > 0) nut_f = nut[p + sy];
      else if ((j == my - 2 && !g.jper) || nv[p + sy] > 0) nut_f = nut[p];
      else nut_f = 0.5 * (nut[p] + nut[p + sy]);
      v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, eta0, eta1, eta2, ajc, nut_f);
      v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, eta0, eta1, eta2, ajc, nut_f);
      v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, eta0, eta1, eta2, ajc, nut_f);
    }
    v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, eta0, eta1, eta2, ajc, nu);
    v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, eta0, eta1, eta2, ajc, nu);
    v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, eta0, eta1, eta2, ajc, nu);
    f2.div[0][p] = d[0]; f2.div[1][p] = d[1]; f2.div[2][p] = d[2];
    f2.visc[0][p] = v[0]; f2.visc[1][p] = v[1]; f2.visc[2][p] = v[2];
  }

  // ---------------- k direction
  if (i != 0 && j != 0) {
    const double ajc = m.kaj[p];
    const double csi0 = m.kcsi.x[p], csi1 = m.kcsi.y[p], csi2 = m.kcsi.z[p];
    const double eta0 = m.keta.x[p], eta1 = m.keta.y[p], eta2 = m.keta.z[p];
    const double zet0 = m.kzet.x[p], zet1 = m.kzet.y[p], zet2 = m.kzet.z[p];
    double dc[3], de[3], dz[3];
    cross_diff(u, p, p + sz, p + sx, p + sz + sx, p - sx, p + sz - sx,
               nv[p + sx] > 0 || nv[p + sz + sx] > 0, nv[p - sx] > 0 || nv[p + sz - sx] > 0, dc);
    cross_diff(u, p, p + sz, p + sy, p + sz + sy, p - sy, p + sz - sy,
               nv[p + sy] > 0 || nv[p + sz + sy] > 0, nv[p - sy] > 0 || nv[p + sz - sy] > 0, de);
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
    if (k == 0 || k == mz - 2) {
      if (g.kper) kL = mz - 3, kR = 2;
      else kL = k, kR = k + 1;
    } else if (nv[p - sz] + nv[p + 2 * sz] > 0) kL = k, kR = k + 1;
    double ucon = uc.z[p];
    if (g.kper && (k == 0 || k == mz - 2)) ucon = uc.z[p + (long long)(mz - 2 - k) * sz];
    if (k == mz - 2 && g.bc[5] == 4 && nv[p] == 0) ucon = uc.z[p - sz];
    const double up = -0.5 * (ucon + fabs(ucon));
    const double um = -0.5 * (ucon - fabs(ucon));
    const long long pL = p + (long long)(kL - k) * sz, pR = p + (long long)(kR - k) * sz;
    double d[3];
    if (g.immersed && k != mz - 2 && nv[p] > 0) {
      d[0] = quick_a(um, up, u.x[p], u.x[p + sz], u.x[p + 2 * sz]);
      d[1] = quick_a(um, up, u.y[p], u.y[p + sz], u.y[p + 2 * sz]);
      d[2] = quick_a(um, up, u.z[p], u.z[p + sz], u.z[p + 2 * sz]);
    } else if (g.immersed && k != 0 && nv[p + sz] > 0) {
      d[0] = quick_b(um, up, u.x[p - sz], u.x[p], u.x[p + sz]);
      d[1] = quick_b(um, up, u.y[p - sz], u.y[p], u.y[p + sz]);
      d[2] = quick_b(um, up, u.z[p - sz], u.z[p], u.z[p + sz]);
    } else {
      const double cu = uc.z[p];
      d[0] = -cu * 0.0625 * (-u.x[pL] + 9. * u.x[p] + 9. * u.x[p + sz] - u.x[pR]);
      d[1] = -cu * 0.0625 * (-u.y[pL] + 9. * u.y[p] + 9. * u.y[p + sz] - u.y[pR]);
      d[2] = -cu * 0.0625 * (-u.z[pL] + 9. * u.z[p] + 9. * u.z[p + sz] - u.z[pR]);
    }
    if (nv[p] + nv[p + sz] > 0 && !g.immersed) d[0] = d[1] = d[2] = 0;
    double v[3] = {0, 0, 0};
    if (les) {
      double nut_f;
      if ((k == 0 && !g.kper) || nv[p] > 0) nut_f = nut[p + sz];
      else if ((k == mz - 2 && !g.kper) || nv[p + sz] > 0) nut_f = nut[p];
      else nut_f = 0.5 * (nut[p] + nut[p + sz]);
      v[0] = visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, zet0, zet1, zet2, ajc, nut_f);
      v[1] = visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, zet0, zet1, zet2, ajc, nut_f);
      v[2] = visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, zet0, zet1, zet2, ajc, nut_f);
    }
    v[0] += visc_term(g11, g21, g31, dc[0], de[0], dz[0], r11, r21, r31, zet0, zet1, zet2, ajc, nu);
    v[1] += visc_term(g11, g21, g31, dc[1], de[1], dz[1], r12, r22, r32, zet0, zet1, zet2, ajc, nu);
    v[2] += visc_term(g11, g21, g31, dc[2], de[2], dz[2], r13, r23, r33, zet0, zet1, zet2, ajc, nu);
    f3.div[0][p] = d[0]; f3.div[1][p] = d[1]; f3.div[2][p] = d[2];
    f3.visc[0][p] = v[0]; f3.visc[1][p] = v[1]; f3.visc[2][p] = v[2];
  }
}

// Fp at interior cells: 4th-order divergence correction 9/8*div - 1/8*wide/denom plus the
// viscous divergence (momentum.c:1508-1640).  Face fluxes on a periodic ghost plane are
// read from their periodic image (momentum.c:1456-1500 copy loop).
struct FluxIn { const double *div[3]; const double *visc[3]; };

__global__ void k_fp(Grid g, FluxIn f1, FluxIn f2, FluxIn f3, const uint8_t *__restrict__ nv,
                     double *fpx, double *fpy, double *fpz) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) return;
  const long long sy = mx, sz = (long long)mx * my;
  const long long rowi = p - i, rowj = p - (long long)j * sy, rowk = p - (long long)k * sz;
  // periodic images of face indices
  auto fi = [&](int ii) { return rowi + wrapi(g, ii); };
  auto fj = [&](int jj) { return rowj + (long long)wrapj(g, jj) * sy; };
  auto fk = [&](int kk) { return rowk + (long long)wrapk(g, kk) * sz; };
  double div[3], acc[3] = {0, 0, 0}, fpv[3];
  for (int c = 0; c < 3; c++)
    div[c] = (f1.div[c][p] - f1.div[c][fi(i - 1)] + f2.div[c][p] - f2.div[c][fj(j - 1)] +
              f3.div[c][p] - f3.div[c][fk(k - 1)]);
  int iR = i + 1, iL = i - 2, jR = j + 1, jL = j - 2, kR = k + 1, kL = k - 2;
  double di = 3., dj = 3., dk = 3.;
  if (i == 1) { if (g.iper) iL = mx - 3; else iR = i, iL = i - 1, di = 1.; }
  else if (i == 2 || i == mx - 3) { if (!g.iper) iR = i, iL = i - 1, di = 1.; }
  else if (i == mx - 2) { if (g.iper) iR = 1; else iR = i, iL = i - 1, di = 1.; }
  if (j == 1) { if (g.jper) jL = my - 3; else jR = j, jL = j - 1, dj = 1.; }
  else if (j == 2 || j == my - 3) { if (!g.jper) jR = j, jL = j - 1, dj = 1.; }
  else if (j == my - 2) { if (g.jper) jR = 1; else jR = j, jL = j - 1, dj = 1.; }
  if (k == 1) { if (g.kper) kL = mz - 3; else kR = k, kL = k - 1, dk = 1.; }
  else if (k == 2 || k == mz - 3) { if (!g.kper) kR = k, kL = k - 1, dk = 1.; }
  else if (k == mz - 2) { if (g.kper) kR = 1; else kR = k, kL = k - 1, dk = 1.; }
  if (nv[p - 1] + nv[p] + nv[p + 1] > 0) iR = i, iL = i - 1, di = 1.;
  if (nv[p - sy] + nv[p] + nv[p + sy] > 0) jR = j, jL = j - 1, dj = 1.;
  if (nv[p - sz] + nv[p] + nv[p + sz] > 0) kR = k, kL = k - 1, dk = 1.;
  const double ai = 1. / di, aj_ = 1. / dj, ak = 1. / dk;
  for (int c = 0; c < 3; c++) {
    acc[c] += (f1.div[c][fi(iR)] - f1.div[c][fi(iL)]) * ai;
    acc[c] += (f2.div[c][fj(jR)] - f2.div[c][fj(jL)]) * aj_;
    acc[c] += (f3.div[c][fk(kR)] - f3.div[c][fk(kL)]) * ak;
    fpv[c] = 9. / 8. * div[c] + -1. / 8. * acc[c];
    fpv[c] += (f1.visc[c][p] - f1.visc[c][fi(i - 1)] + f2.visc[c][p] - f2.visc[c][fj(j - 1)] +
               f3.visc[c][p] - f3.visc[c][fk(k - 1)]) / 1.0;
  }
  fpx[p] = fpv[0]; fpy[p] = fpv[1]; fpz[p] = fpv[2];
}

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
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  double r[3];
  if (i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1) {
    r[0] = r[1] = r[2] = 0;
  } else {
    const long long sy = mx, sz = (long long)mx * my;
    // Fp on the periodic ghost plane is the image of the first interior plane
    const long long pi1 = (g.iper && i == mx - 2) ? p - i + 1 : p + 1;
    const long long pj1 = (g.jper && j == my - 2) ? p - (long long)j * sy + sy : p + sy;
    const long long pk1 = (g.kper && k == mz - 2) ? p - (long long)k * sz + sz : p + sz;
    if (rk) { r[0] = 0; r[1] = 0; r[2] = 0; }
    else { r[0] = rhs.x[p]; r[1] = rhs.y[p]; r[2] = rhs.z[p]; }
    r[0] += scale * (0.5 * (m.csi.x[p] * fpx[p] + m.csi.y[p] * fpy[p] + m.csi.z[p] * fpz[p]) +
                     0.5 * (m.csi.x[p + 1] * fpx[pi1] + m.csi.y[p + 1] * fpy[pi1] + m.csi.z[p + 1] * fpz[pi1])) *
            m.iaj[p];
    r[1] += scale * (0.5 * (m.eta.x[p] * fpx[p] + m.eta.y[p] * fpy[p] + m.eta.z[p] * fpz[p]) +
                     0.5 * (m.eta.x[p + sy] * fpx[pj1] + m.eta.y[p + sy] * fpy[pj1] + m.eta.z[p + sy] * fpz[pj1])) *
            m.jaj[p];
    r[2] += scale * (0.5 * (m.zet.x[p] * fpx[p] + m.zet.y[p] * fpy[p] + m.zet.z[p] * fpz[p]) +
                     0.5 * (m.zet.x[p + sz] * fpx[pk1] + m.zet.y[p + sz] * fpy[pk1] + m.zet.z[p + sz] * fpz[pk1])) *
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
    ucont.x[p] = a * r[0] + pu.x[p];
    ucont.y[p] = a * r[1] + pu.y[p];
    ucont.z[p] = a * r[2] + pu.z[p];
  }
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

int formfunction2(Ctx *c, double scale, bool rk_stage, double rk_coeff) {
  const Grid &g = c->g;
  int rc;
  V3 uc = field3(c, VFS_UCONT);
  if ((rc = periodic_copy3(c, uc))) return rc;
  Metrics m = metrics(c);
  k_face_flux<<<nblocks(g.N, 128), 128, 0, c->stream>>>(g, m, cv(uc), cv(field3(c, VFS_UCAT)), c->nv,
                                                        c->f[VFS_NU_T][0], flux_out(c, 0), flux_out(c, 1),
                                                        flux_out(c, 2));
  if ((rc = check_launch(c, "k_face_flux"))) return rc;
  k_fp<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, flux_in(c, 0), flux_in(c, 1), flux_in(c, 2), c->nv,
                                                c->fp[0], c->fp[1], c->fp[2]);
  if ((rc = check_launch(c, "k_fp"))) return rc;
  V3 pu{c->pucont[0], c->pucont[1], c->pucont[2]};
  k_rhs<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, m, c->nv, c->fp[0], c->fp[1], c->fp[2], scale,
                                                 field3(c, VFS_RHS), rk_stage ? 1 : 0, rk_coeff,
                                                 cv(field3(c, VFS_DP)), cv(pu), uc);
  return check_launch(c, "k_rhs");
}

// single-kernel launchers for the diagnostics entry point (vfs_run_kernel)
void launch_face_flux(Ctx *c) {
  k_face_flux<<<nblocks(c->g.N, 128), 128, 0, c->stream>>>(c->g, metrics(c), cv(field3(c, VFS_UCONT)),
                                                           cv(field3(c, VFS_UCAT)), c->nv, c->f[VFS_NU_T][0],
                                                           flux_out(c, 0), flux_out(c, 1), flux_out(c, 2));
}
void launch_fp(Ctx *c) {
  k_fp<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, flux_in(c, 0), flux_in(c, 1), flux_in(c, 2), c->nv,
                                                   c->fp[0], c->fp[1], c->fp[2]);
}
void launch_rhs(Ctx *c) {
  V3 pu{c->pucont[0], c->pucont[1], c->pucont[2]};
  k_rhs<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), c->nv, c->fp[0], c->fp[1], c->fp[2], 1.0,
                                                    field3(c, VFS_RHS), 0, 0.0, cv(field3(c, VFS_DP)), cv(pu),
                                                    field3(c, VFS_UCONT));
}

// ------------------------------------------------------------------ Pressure_Gradient
// momentum.c:197-443 (levelset off): dP on the three faces of each interior cell, with
// one-sided cross differences next to IB nodes (nvert == 1) and non-periodic walls, and
// the mean-pressure-gradient forcing along a periodic k direction.
__global__ void k_pressure_gradient(Grid g, Metrics m, const uint8_t *__restrict__ nv,
                                    const double *__restrict__ P, double kdiff, double kdt,
                                    double karea, int kforce_mode, double mpg, V3 dp) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  if (i < 1 || i > mx - 2 || j < 1 || j > my - 2 || k < 1 || k > mz - 2) {
    dp.x[p] = 0; dp.y[p] = 0; dp.z[p] = 0;  // VecSet(dP, 0) outside the loop
    return;
  }
  const long long sy = mx, sz = (long long)mx * my;
  const double g11_i = dot3(m.icsi.x[p], m.icsi.y[p], m.icsi.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  const double g12_i = dot3(m.ieta.x[p], m.ieta.y[p], m.ieta.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  const double g13_i = dot3(m.izet.x[p], m.izet.y[p], m.izet.z[p], m.icsi.x[p], m.icsi.y[p], m.icsi.z[p]);
  const double g21_j = dot3(m.jcsi.x[p], m.jcsi.y[p], m.jcsi.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  const double g22_j = dot3(m.jeta.x[p], m.jeta.y[p], m.jeta.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  const double g23_j = dot3(m.jzet.x[p], m.jzet.y[p], m.jzet.z[p], m.jeta.x[p], m.jeta.y[p], m.jeta.z[p]);
  const double g31_k = dot3(m.kcsi.x[p], m.kcsi.y[p], m.kcsi.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
  const double g32_k = dot3(m.keta.x[p], m.keta.y[p], m.keta.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
  const double g33_k = dot3(m.kzet.x[p], m.kzet.y[p], m.kzet.z[p], m.kzet.x[p], m.kzet.y[p], m.kzet.z[p]);
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
  double ox = (dpdc * g11_i + dpde * g12_i + dpdz * g13_i) * m.iaj[p] / r1;
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
  double oy = (dpdc * g21_j + dpde * g22_j + dpdz * g23_j) * m.jaj[p] / r2;
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
    const double kz2 = m.kzet.x[p] * m.kzet.x[p] + m.kzet.y[p] * m.kzet.y[p] + m.kzet.z[p] * m.kzet.z[p];
    const double dz = 1. / m.kaj[p] / sqrt(kz2);
    if (kforce_mode == 1) dpdz += mpg * dz;
    else if (kforce_mode == 2) dpdz += dz * kdiff / kdt / karea;
  }
  double oz = (dpdc * g31_k + dpde * g32_k + dpdz * g33_k) * m.kaj[p] / r3;
  if (i == 0 || nv[p] + nv[p + 1] > 0 || (!g.iper && i == mx - 2)) ox = 0;
  if (j == 0 || nv[p] + nv[p + sy] > 0 || (!g.jper && j == my - 2)) oy = 0;
  if (k == 0 || nv[p] + nv[p + sz] > 0 || (!g.kper && k == mz - 2)) oz = 0;
  dp.x[p] = ox; dp.y[p] = oy; dp.z[p] = oz;
}

int pressure_gradient(Ctx *c) {
  int rc;
  // P's periodic ghosts are refreshed first (momentum.c:241-273)
  if ((rc = periodic_copy1(c, c->f[VFS_P][0]))) return rc;
  // k-periodic forcing (momentum.c:379-399): dpdz_set -> mean_pressure_gradient, else
  // (inletprofile != 17) the flux-deficit term (mean_k_flux - inlet_flux)/dt/mean_k_area.
  int mode = 0;
  if (c->cfg.dpdz_set) mode = 1;
  else if (c->cfg.inletprofile != 17) mode = 2;
  const double kdiff = c->scal[VFS_S_MEAN_K_FLUX] - c->scal[VFS_S_INLET_FLUX];
  k_pressure_gradient<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(
      c->g, metrics(c), c->nv, c->f[VFS_P][0], kdiff, c->g.dt, c->scal[VFS_S_MEAN_K_AREA], mode,
      c->cfg.mean_pressure_gradient, field3(c, VFS_DP));
  return check_launch(c, "k_pressure_gradient");
}

// ------------------------------------------------------------------ Calc_k_Flux
// rhs2.c:1562-1646: sum of Ucont.z over k-faces k = 1..mz-2, interior (i,j), whose two
// adjacent cells are fluid; divided by (mz-2).
__global__ void k_kflux_parts(Grid g, const double *__restrict__ uz, const uint8_t *__restrict__ nv,
                              double *parts) {
  __shared__ double sh[256];
  double s = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    int i = (int)(p % g.mx);
    long long q = p / g.mx;
    int j = (int)(q % g.my);
    int k = (int)(q / g.my);
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

int calc_k_flux(Ctx *c, double *flux) {
  int rc;
  const int nb = 148 * 4;
  if ((rc = ensure_red(c, nb + 64))) return rc;
  k_kflux_parts<<<nb, 256, 0, c->stream>>>(c->g, c->f[VFS_UCONT][2], c->nv, c->red);
  if ((rc = check_launch(c, "k_kflux_parts"))) return rc;
  double s = 0;
  if ((rc = reduce_sum(c, c->red, nb, &s))) return rc;
  s /= (c->g.mz - 2);
  c->scal[VFS_S_MEAN_K_FLUX] = s;
  if (flux) *flux = s;
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
    int i = (int)(p % g.mx);
    long long q = p / g.mx;
    int j = (int)(q % g.my);
    int k = (int)(q / g.my);
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
  k_area_parts<<<nb, 256, 0, c->stream>>>(c->g, cv(field3(c, VFS_ZET)), c->nv, c->red);
  if ((rc = check_launch(c, "k_area_parts"))) return rc;
  double a = 0, b = 0;
  if ((rc = reduce_sum(c, c->red, nb, &a))) return rc;
  if ((rc = reduce_sum(c, c->red + nb, nb, &b))) return rc;
  c->scal[VFS_S_MEAN_K_AREA] = a / (double)(c->g.mz - 2);
  if (c->g.bc[4] == 5 || c->g.kper) c->scal[VFS_S_INLET_AREA] = b;
  return VFS_OK;
}

// ------------------------------------------------------------------ IB_BC (no IB nodes)
// momentum.c:1982-2195 without immersed bodies: normal flux through free-slip faces set
// to zero and the normal flux of periodic ghost planes taken from the image plane.
__global__ void k_ib_bc_faces(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
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
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
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
  if (c->g.immersed) return set_err(c, VFS_ERR_INVALID, "IB_BC: immersed-boundary reconstruction is not on this path yet");
  k_ib_bc_faces<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
  if ((rc = check_launch(c, "k_ib_bc_faces"))) return rc;
  if (c->g.iper || c->g.jper || c->g.kper) {
    k_periodic_normal<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
    if ((rc = check_launch(c, "k_periodic_normal"))) return rc;
  }
  return VFS_OK;
}

// ------------------------------------------------------------------ FormBCS subset
// bcs.c:1841-2936 for the codes handled here: Contra2Cart, zero normal flux on no-slip
// and free-slip walls of the i and j faces (interior range), Contra2Cart again, then the
// twelve edges of the box get Ucat = 0.
__global__ void k_wall_flux(Grid g, V3 uc) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int mx = g.mx, my = g.my, mz = g.mz;
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
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
  int i = (int)(p % mx);
  long long q = p / mx;
  int j = (int)(q % my);
  int k = (int)(q / my);
  int bi = (i == 0 || i == mx - 1), bj = (j == 0 || j == my - 1), bk = (k == 0 || k == mz - 1);
  if (bi + bj + bk >= 2) { u.x[p] = 0; u.y[p] = 0; u.z[p] = 0; }
}

int form_bcs(Ctx *c) {
  int rc;
  for (int q = 0; q < 6; q++)
    if (c->g.bc[q] == 4 || c->g.bc[q] == 5)
      return set_err(c, VFS_ERR_INVALID, "FormBCS: inlet/outlet faces are not handled by this step driver");
  if ((rc = contra2cart(c))) return rc;
  k_wall_flux<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCONT));
  if ((rc = check_launch(c, "k_wall_flux"))) return rc;
  if ((rc = contra2cart(c))) return rc;
  k_zero_edges<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, field3(c, VFS_UCAT));
  return check_launch(c, "k_zero_edges");
}

// ------------------------------------------------------------------ RungeKutta
// rhs.c:1578-1700 (implicit=0): InflowFlux, FormBCS, then four stages
//   Contra2Cart; Rhs = Formfunction_2 - dP; Ucont = pUcont + alfa*dt*st*Rhs; Contra2Cart
// and finally FormBCS again.
int runge_kutta(Ctx *c) {
  int rc;
  const double alfa[4] = {0.25, 1 / 3., 0.5, 1.};
  if ((rc = form_bcs(c))) return rc;
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(c->pucont[q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  for (int s = 0; s < 4; s++) {
    if ((rc = contra2cart(c))) return rc;
    const double a = alfa[s] * c->g.dt * c->g.st;
    if ((rc = formfunction2(c, 1.0, true, a))) return rc;
    if ((rc = contra2cart(c))) return rc;
  }
  return form_bcs(c);
}

}  // namespace vfs
