// Dynamic Smagorinsky eddy viscosity for sm_100a: Compute_Smagorinsky_Constant_1
// (les.c:67-1133) and Compute_eddy_viscosity_LES (les.c:1135-1252), default options
// (3-D box test filter, testfilter_ik = 0, clark = 0, no homogeneous-direction averaging).
//
// Six kernels, FP64 throughout, each pointwise expression in the reference's order:
//   k_les_prep    every DA point: contravariant centre velocity U,V,W and test-filter
//                 weight of the point itself;
//   k_les_image   every DA point: at the point's periodic image the strain products
//                 S_ab*|S| and the test-filtered velocity (les.c:191-298);
//   k_les_lm      interior cells, 3-D tile with a one-cell halo staged in shared memory:
//                 the Germano identity contractions L_ij M_ij G and M_ij M_ij G
//                 (les.c:300-661);
//   k_les_cs      every DA point: filtered LM/MM, Cs = max(0, LM/(2(MM+eps))), wall floor
//                 and [0, max_cs] clipping, periodic ghosts from their images (les.c:708-1048);
//   k_les_refilter  second test filtering of Cs over fluid cells (les.c:1051-1120);
//   k_les_nut     nu_t = Cs * Delta^2 * |S| and its periodic ghosts (les.c:1174-1243).
// The 3x3x3 test filter is integrate_testfilter (rhs2.c:412-455): eight 2x2x2 sub-cubes,
// each summed in the reference's order, over the same sums of weights.
#include <cmath>

#include "vfs_internal.cuh"

namespace vfs {

constexpr double kLesEps = 1.e-4;  // les_eps, les.c:20
constexpr double kWallCs = 0.001;  // wall_cs, les.c:21

__device__ __forceinline__ bool les_interior(const Grid &g, int i, int j, int k) {
  return i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2;
}

// Compute_du_center (k-omega.c:305-420): centre derivatives of a vector field along the
// three grid directions, one-sided next to cells with nvert > 0.1 and at non-periodic
// boundaries.  d = {du/dc, dv/dc, dw/dc, du/de, dv/de, dw/de, du/dz, dv/dz, dw/dz}.
// The k test uses k == 0 where the i and j tests use 1 (k-omega.c:395), as the reference.
__device__ __forceinline__ void du_center(const Grid &g, CV3 u, const uint8_t *__restrict__ nv, long long p,
                                          int i, int j, int k, double d[9]) {
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  long long a, b;
  double f;
  if (nv[p + 1] > 0 || (!g.iper && i == g.mx - 2)) { a = p; b = p - 1; f = 1.0; }
  else if (nv[p - 1] > 0 || (!g.iper && i == 1)) { a = p + 1; b = p; f = 1.0; }
  else { a = p + 1; b = p - 1; f = 0.5; }
  d[0] = (u.x[a] - u.x[b]) * f; d[1] = (u.y[a] - u.y[b]) * f; d[2] = (u.z[a] - u.z[b]) * f;
  if (nv[p + sy] > 0 || (!g.jper && j == g.my - 2)) { a = p; b = p - sy; f = 1.0; }
  else if (nv[p - sy] > 0 || (!g.jper && j == 1)) { a = p + sy; b = p; f = 1.0; }
  else { a = p + sy; b = p - sy; f = 0.5; }
  d[3] = (u.x[a] - u.x[b]) * f; d[4] = (u.y[a] - u.y[b]) * f; d[5] = (u.z[a] - u.z[b]) * f;
  if (nv[p + sz] > 0 || (!g.kper && k == g.mz - 2)) { a = p; b = p - sz; f = 1.0; }
  else if (nv[p - sz] > 0 || (!g.kper && k == 0)) { a = p + sz; b = p; f = 1.0; }
  else { a = p + sz; b = p - sz; f = 0.5; }
  d[6] = (u.x[a] - u.x[b]) * f; d[7] = (u.y[a] - u.y[b]) * f; d[8] = (u.z[a] - u.z[b]) * f;
}

// Compute_du_dxyz (k-omega.c:597-610): Cartesian gradient by the chain rule.
// o = {du/dx, du/dy, du/dz, dv/dx, dv/dy, dv/dz, dw/dx, dw/dy, dw/dz}.
__device__ __forceinline__ void du_dxyz(const double c[3], const double e[3], const double z[3], double ajc,
                                        const double d[9], double o[9]) {
#pragma unroll
  for (int v = 0; v < 3; v++) {
    o[3 * v + 0] = (d[v] * c[0] + d[3 + v] * e[0] + d[6 + v] * z[0]) * ajc;
    o[3 * v + 1] = (d[v] * c[1] + d[3 + v] * e[1] + d[6 + v] * z[1]) * ajc;
    o[3 * v + 2] = (d[v] * c[2] + d[3 + v] * e[2] + d[6 + v] * z[2]) * ajc;
  }
}

// Strain tensor {Sxx, Sxy, Sxz, Syy, Syz, Szz} and |S| (les.c:209-213).
__device__ __forceinline__ double strain(const double o[9], double s[6]) {
  s[0] = 0.5 * (o[0] + o[0]);
  s[1] = 0.5 * (o[1] + o[3]);
  s[2] = 0.5 * (o[2] + o[6]);
  s[3] = 0.5 * (o[4] + o[4]);
  s[4] = 0.5 * (o[5] + o[7]);
  s[5] = 0.5 * (o[8] + o[8]);
  return sqrt(2.0 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + s[1] * s[1] + s[3] * s[3] + s[4] * s[4] +
                     s[2] * s[2] + s[4] * s[4] + s[5] * s[5]));
}

// Neighbour n = R*9 + Q*3 + P (R, Q, P = k, j, i offsets + 1) of the m-th point of the
// s-th 2x2x2 sub-cube, in the order integrate_testfilter sums them (rhs2.c:433-455).
__host__ __device__ constexpr int tf_base(int s) { return (s & 1) * 9 + ((s >> 2) & 1) * 3 + ((s >> 1) & 1); }
__host__ __device__ constexpr int tf_off(int m) { return (m & 1) * 9 + ((m >> 2) & 1) * 3 + ((m >> 1) & 1); }

// Sum of the sub-cube weight sums (the common denominator w1 + ... + w8).
__device__ __forceinline__ double tf_wsum(const double w[27]) {
  double tot = 0;
#pragma unroll
  for (int s = 0; s < 8; s++) {
    double ws = w[tf_base(s) + tf_off(0)];
#pragma unroll
    for (int m = 1; m < 8; m++) ws += w[tf_base(s) + tf_off(m)];
    tot = (s == 0) ? ws : tot + ws;
  }
  return tot;
}

// integrate_testfilter of one 27-point quantity given as val[n].
__device__ __forceinline__ double tf_apply(const double val[27], const double w[27], double wsum) {
  double tot = 0;
#pragma unroll
  for (int s = 0; s < 8; s++) {
    const int b = tf_base(s);
    double vs = val[b + tf_off(0)] * w[b + tf_off(0)];
#pragma unroll
    for (int m = 1; m < 8; m++) vs += val[b + tf_off(m)] * w[b + tf_off(m)];
    tot = (s == 0) ? vs : tot + vs;
  }
  return tot / wsum;
}

struct LesPrep {
  double *U, *V, *W;   // contravariant centre velocity (own point)
  double *wgt;         // 0 where nvert > 1.1, else 1/aj (own point)
  double *ss[6];       // S_ab*|S| at the periodic image, zero at solid/boundary images
  double *uf[3];       // test-filtered velocity at the periodic image
};

// ------------------------------------------------------------------ k_les_prep
// Own-point quantities of every DA point: U, V, W and the test-filter weight.
__global__ void k_les_prep(Grid g, CV3 u, CV3 csi, CV3 eta, CV3 zet, const double *__restrict__ aj,
                           const uint8_t *__restrict__ nv, LesPrep o) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const double ux = u.x[p], uy = u.y[p], uz = u.z[p];
  o.U[p] = ux * csi.x[p] + uy * csi.y[p] + uz * csi.z[p];
  o.V[p] = ux * eta.x[p] + uy * eta.y[p] + uz * eta.z[p];
  o.W[p] = ux * zet.x[p] + uy * zet.y[p] + uz * zet.z[p];
  o.wgt[p] = (nv[p] > 1) ? 0.0 : 1. / aj[p];  // get_weight, les.c:31-32
}

// Strain products S_ab |S| and the test-filtered velocity at every DA point's periodic
// image (computed at interior fluid cells, les.c:191-238, and copied to periodic ghosts,
// les.c:267-298); zero where the image is solid or a boundary point.
__global__ void k_les_image(Grid g, CV3 u, CV3 csi, CV3 eta, CV3 zet, const double *__restrict__ aj,
                            const uint8_t *__restrict__ nv, LesPrep o) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int a = wrapi(g, i), b = wrapj(g, j), c = wrapk(g, k);
  const long long q = lidx(g, a, b, c);
  double ss[6] = {0, 0, 0, 0, 0, 0}, uf[3] = {0, 0, 0};
  if (les_interior(g, a, b, c) && nv[q] <= 1) {
    double d[9], gr[9], st[6];
    du_center(g, u, nv, q, a, b, c, d);
    const double cc[3] = {csi.x[q], csi.y[q], csi.z[q]};
    const double ee[3] = {eta.x[q], eta.y[q], eta.z[q]};
    const double zz[3] = {zet.x[q], zet.y[q], zet.z[q]};
    du_dxyz(cc, ee, zz, aj[q], d, gr);
    const double sabs = strain(gr, st);
#pragma unroll
    for (int t = 0; t < 6; t++) ss[t] = st[t] * sabs;
    // integrate_testfilter of u, v, w with the get_weight weights (les.c:219-237)
    const long long sy = g.mx, sz = (long long)g.mx * g.my;
    double wt = 0, t0 = 0, t1 = 0, t2 = 0;
#pragma unroll 1
    for (int s = 0; s < 8; s++) {
      double ws = 0, v0 = 0, v1 = 0, v2 = 0;
#pragma unroll
      for (int m = 0; m < 8; m++) {
        const int n = tf_base(s) + tf_off(m);
        const long long qq = q + (n / 9 - 1) * sz + ((n / 3) % 3 - 1) * sy + (n % 3 - 1);
        const double wn = o.wgt[qq];
        if (m == 0) { ws = wn; v0 = u.x[qq] * wn; v1 = u.y[qq] * wn; v2 = u.z[qq] * wn; }
        else { ws += wn; v0 += u.x[qq] * wn; v1 += u.y[qq] * wn; v2 += u.z[qq] * wn; }
      }
      if (s == 0) { wt = ws; t0 = v0; t1 = v1; t2 = v2; }
      else { wt += ws; t0 += v0; t1 += v1; t2 += v2; }
    }
    uf[0] = t0 / wt; uf[1] = t1 / wt; uf[2] = t2 / wt;
  }
#pragma unroll
  for (int t = 0; t < 6; t++) o.ss[t][p] = ss[t];
  o.uf[0][p] = uf[0]; o.uf[1][p] = uf[1]; o.uf[2][p] = uf[2];
}

// ------------------------------------------------------------------ k_les_lm
constexpr int LTX = 32, LTY = 4, LTZ = 2;
constexpr int LHX = LTX + 2, LHY = LTY + 2, LHZ = LTZ + 2, LHN = LHX * LHY * LHZ;
constexpr int kLesLmThreads = LTX * LTY * LTZ;
constexpr int kLesVals = 13;  // u v w U V W weight SS11 SS12 SS13 SS22 SS23 SS33
struct LesLmSmem {
  double v[kLesVals][LHN];
};

struct LesLmIn {
  CV3 u;
  const double *U, *V, *W, *wgt, *ss[6];
  CV3 uf;
};

// Calculate_Covariant_metrics (rhs2.c:538-554): inverse of the centre metric matrix.
__device__ __forceinline__ void covariant(const double a[3][3], double G[3][3]) {
  const double a11 = a[0][0], a12 = a[0][1], a13 = a[0][2];
  const double a21 = a[1][0], a22 = a[1][1], a23 = a[1][2];
  const double a31 = a[2][0], a32 = a[2][1], a33 = a[2][2];
  const double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
  G[0][0] = (a33 * a22 - a32 * a23) / det; G[0][1] = -(a33 * a12 - a32 * a13) / det; G[0][2] = (a23 * a12 - a22 * a13) / det;
  G[1][0] = -(a33 * a21 - a31 * a23) / det; G[1][1] = (a33 * a11 - a31 * a13) / det; G[1][2] = -(a23 * a11 - a21 * a13) / det;
  G[2][0] = (a32 * a21 - a31 * a22) / det; G[2][1] = -(a32 * a11 - a31 * a12) / det; G[2][2] = (a22 * a11 - a21 * a12) / det;
}

// Tile index of neighbour n (R*9 + Q*3 + P) of the cell at tile index c0.
__device__ __forceinline__ int les_nb(int c0, int n) {
  return c0 + (n / 9 - 1) * LHX * LHY + ((n / 3) % 3 - 1) * LHX + (n % 3 - 1);
}

// Quantity q at tile point h: q < 9 the product (U,V,W)[q/3] * (u,v,w)[q%3] (les.c:381-391),
// q >= 9 the strain product S_ab |S| number q-9 (les.c:428-430).
template <int q>
__device__ __forceinline__ double les_quantity(const LesLmSmem &S, int h) {
  if (q < 9) return S.v[3 + q / 3][h] * S.v[q % 3][h];
  return S.v[7 + (q - 9)][h];
}

// integrate_testfilter of quantities Q0 .. Q0+NQ-1 (rhs2.c:412-455) into F[].
template <int Q0, int NQ>
__device__ __forceinline__ void les_filter_pass(const LesLmSmem &S, int c0, double wsum, double *F) {
  double tot[NQ], vs[NQ];
#pragma unroll 1
  for (int s = 0; s < 8; s++) {
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const int h = les_nb(c0, tf_base(s) + tf_off(m));
      const double wn = S.v[6][h];
      double x[NQ];
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        switch (Q0 + q) {
          case 0: x[q] = les_quantity<0>(S, h); break;
          case 1: x[q] = les_quantity<1>(S, h); break;
          case 2: x[q] = les_quantity<2>(S, h); break;
          case 3: x[q] = les_quantity<3>(S, h); break;
          case 4: x[q] = les_quantity<4>(S, h); break;
          case 5: x[q] = les_quantity<5>(S, h); break;
          case 6: x[q] = les_quantity<6>(S, h); break;
          case 7: x[q] = les_quantity<7>(S, h); break;
          case 8: x[q] = les_quantity<8>(S, h); break;
          case 9: x[q] = les_quantity<9>(S, h); break;
          case 10: x[q] = les_quantity<10>(S, h); break;
          case 11: x[q] = les_quantity<11>(S, h); break;
          case 12: x[q] = les_quantity<12>(S, h); break;
          case 13: x[q] = les_quantity<13>(S, h); break;
          default: x[q] = les_quantity<14>(S, h); break;
        }
      }
#pragma unroll
      for (int q = 0; q < NQ; q++) vs[q] = (m == 0) ? x[q] * wn : vs[q] + x[q] * wn;
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) tot[q] = (s == 0) ? vs[q] : tot[q] + vs[q];
  }
#pragma unroll
  for (int q = 0; q < NQ; q++) F[Q0 + q] = tot[q] / wsum;
}

__global__ void __launch_bounds__(kLesLmThreads, 2)
    k_les_lm(Grid g, LesLmIn in, CV3 csi, CV3 eta, CV3 zet, const double *__restrict__ aj,
             const uint8_t *__restrict__ nv, double *LM, double *MM) {
  extern __shared__ __align__(16) unsigned char les_raw[];
  LesLmSmem &S = *reinterpret_cast<LesLmSmem *>(les_raw);
  const int i0 = 1 + blockIdx.x * LTX, j0 = 1 + blockIdx.y * LTY, k0 = 1 + blockIdx.z * LTZ;
  // stage the halo tile: own-point values of the 34 x 6 x 4 points around the tile
  for (int t = threadIdx.x; t < LHN; t += blockDim.x) {
    const int hi = t % LHX, hj = (t / LHX) % LHY, hk = t / (LHX * LHY);
    const int i = i0 - 1 + hi, j = j0 - 1 + hj, k = k0 - 1 + hk;
    if (i < g.mx && j < g.my && k < g.mz) {
      const long long p = lidx(g, i, j, k);
      S.v[0][t] = in.u.x[p]; S.v[1][t] = in.u.y[p]; S.v[2][t] = in.u.z[p];
      S.v[3][t] = in.U[p]; S.v[4][t] = in.V[p]; S.v[5][t] = in.W[p];
      S.v[6][t] = in.wgt[p];
#pragma unroll
      for (int q = 0; q < 6; q++) S.v[7 + q][t] = in.ss[q][p];
    } else {
#pragma unroll
      for (int q = 0; q < kLesVals; q++) S.v[q][t] = 0.0;
    }
  }
  __syncthreads();
  const int ti = threadIdx.x % LTX, tj = (threadIdx.x / LTX) % LTY, tk = threadIdx.x / (LTX * LTY);
  const int i = i0 + ti, j = j0 + tj, k = k0 + tk;
  if (i > g.mx - 2 || j > g.my - 2 || k > g.mz - 2) return;
  const long long p = lidx(g, i, j, k);
  if (nv[p] > 1) { LM[p] = 0; MM[p] = 0; return; }
  const int c0 = (tk + 1) * LHX * LHY + (tj + 1) * LHX + (ti + 1);  // tile index of the cell
  auto nb = [&](int n) { return les_nb(c0, n); };

  // weights stay in shared memory (S.v[6]); w1 + ... + w8 and sum_weight from there
  double wsum = 0;
#pragma unroll
  for (int s = 0; s < 8; s++) {
    double ws = S.v[6][nb(tf_base(s) + tf_off(0))];
#pragma unroll
    for (int m = 1; m < 8; m++) ws += S.v[6][nb(tf_base(s) + tf_off(m))];
    wsum = (s == 0) ? ws : wsum + ws;
  }
  // sum_weight with the (1/2, 1, 1/2)^3 weights, loops p (i) outer, q (j), r (k) inner
  // (les.c:433-452)
  double sum_weight = 0;
#pragma unroll
  for (int pp = 0; pp < 3; pp++)
#pragma unroll
    for (int qq = 0; qq < 3; qq++)
#pragma unroll
      for (int rr = 0; rr < 3; rr++) {
        const double cf = (rr == 1 ? 1.0 : 0.5) * (qq == 1 ? 1.0 : 0.5) * (pp == 1 ? 1.0 : 0.5);
        sum_weight += S.v[6][nb(rr * 9 + qq * 3 + pp)] * cf;
      }

  // 15 test-filtered quantities, three passes of five to keep the accumulators in
  // registers: U u, U v, U w, V u, ..., W w (Lij) and the six S_ab |S|
  double F[15];
  les_filter_pass<0, 5>(S, c0, wsum, F);
  les_filter_pass<5, 5>(S, c0, wsum, F);
  les_filter_pass<10, 5>(S, c0, wsum, F);

  const double cc[3] = {csi.x[p], csi.y[p], csi.z[p]};
  const double ee[3] = {eta.x[p], eta.y[p], eta.z[p]};
  const double zz[3] = {zet.x[p], zet.y[p], zet.z[p]};
  const double ajc = aj[p];
  const double filter = pow(1. / ajc, 1. / 3.);
  const double test_filter = pow(sum_weight, 1. / 3.);
  // filtered velocity at the cell and its contravariant components (les.c:470-475)
  const double fu = in.uf.x[p], fv = in.uf.y[p], fw = in.uf.z[p];
  const double fU = fu * cc[0] + fv * cc[1] + fw * cc[2];
  const double fV = fu * ee[0] + fv * ee[1] + fw * ee[2];
  const double fW = fu * zz[0] + fv * zz[1] + fw * zz[2];
  double d[9], gr[9], sh[6];
  du_center(g, in.uf, nv, p, i, j, k, d);
  du_dxyz(cc, ee, zz, ajc, d, gr);
  const double S_hat = strain(gr, sh);
  const double Sij[3][3] = {{sh[0], sh[1], sh[2]}, {sh[1], sh[3], sh[4]}, {sh[2], sh[4], sh[5]}};
  const double Lij[3][3] = {{F[0] - fU * fu, F[1] - fU * fv, F[2] - fU * fw},
                            {F[3] - fV * fu, F[4] - fV * fv, F[5] - fV * fw},
                            {F[6] - fW * fu, F[7] - fW * fv, F[8] - fW * fw}};
  const double SSij[3][3] = {{F[9], F[10], F[11]}, {F[10], F[12], F[13]}, {F[11], F[13], F[14]}};
  const double gg[3][3] = {{cc[0], cc[1], cc[2]}, {ee[0], ee[1], ee[2]}, {zz[0], zz[1], zz[2]}};
  double ggc[3][3];
  covariant(gg, ggc);
  const double xcsi = ggc[0][0], xeta = ggc[0][1], xzet = ggc[0][2];
  const double ycsi = ggc[1][0], yeta = ggc[1][1], yzet = ggc[1][2];
  const double zcsi = ggc[2][0], zeta = ggc[2][1], zzet = ggc[2][2];
  double G[3][3];
  G[0][0] = xcsi * xcsi + ycsi * ycsi + zcsi * zcsi;
  G[1][1] = xeta * xeta + yeta * yeta + zeta * zeta;
  G[2][2] = xzet * xzet + yzet * yzet + zzet * zzet;
  G[0][1] = G[1][0] = xeta * xcsi + yeta * ycsi + zeta * zcsi;
  G[0][2] = G[2][0] = xzet * xcsi + yzet * ycsi + zzet * zcsi;
  G[1][2] = G[2][1] = xeta * xzet + yeta * yzet + zeta * zzet;
  // Mij (les.c:616-633)
  const double tA = -pow(test_filter, 2.) * S_hat;
  const double fB = pow(filter, 2.);
  double Mc[3][3], M[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) Mc[a][b] = tA * Sij[a][b] + fB * SSij[a][b];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    M[a][0] = Mc[a][0] * cc[0] + Mc[a][1] * cc[1] + Mc[a][2] * cc[2];
    M[a][1] = Mc[a][0] * ee[0] + Mc[a][1] * ee[1] + Mc[a][2] * ee[2];
    M[a][2] = Mc[a][0] * zz[0] + Mc[a][1] * zz[1] + Mc[a][2] * zz[2];
  }
  double num = 0, denom = 0;
#pragma unroll
  for (int q = 0; q < 3; q++)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) num += Lij[b][a] * M[a][q] * G[b][q];
#pragma unroll
  for (int m = 0; m < 3; m++)
#pragma unroll
    for (int n = 0; n < 3; n++)
#pragma unroll
      for (int l = 0; l < 3; l++) denom += M[n][m] * M[n][l] * G[m][l];
  LM[p] = num;
  MM[p] = denom;
}

// Test-filter weights of the Cs averaging and re-filtering loops (les.c:720-762,
// les.c:1069-1110): 1/aj of the neighbour (0 where nvert > 1.1), zero at non-periodic
// boundary neighbours, and the neighbour's value read at its periodic image.  In the j
// direction the reference tests the cell's own j against my-1 (les.c:748, les.c:1097),
// so only J == 0 is zeroed; that test is kept.
__device__ __forceinline__ void wrap_weights(const Grid &g, const double *__restrict__ wgt, int i, int j, int k,
                                             double w[27], long long src[27]) {
#pragma unroll
  for (int n = 0; n < 27; n++) {
    int K = k + n / 9 - 1, J = j + (n / 3) % 3 - 1, I = i + n % 3 - 1;
    double wt = wgt[lidx(g, I, J, K)];  // 1/aj, 0 where nvert > 1.1
    if (g.iper) { if (I == 0) I = g.mx - 2; else if (I == g.mx - 1) I = 1; }
    else if (I == 0 || I == g.mx - 1) wt = 0;
    if (g.jper) { if (J == 0) J = g.my - 2; else if (J == g.my - 1) J = 1; }
    else if (J == 0 || j == g.my - 1) wt = 0;
    if (g.kper) { if (K == 0) K = g.mz - 2; else if (K == g.mz - 1) K = 1; }
    else if (K == 0 || K == g.mz - 1) wt = 0;
    w[n] = wt;
    src[n] = lidx(g, I, J, K);
  }
}

// Clipped Cs of one interior cell (les.c:708-788 with les = 2, then les.c:959-972).
__device__ __forceinline__ double cs_cell(const Grid &g, const double *__restrict__ wgt,
                                          const uint8_t *__restrict__ nv, const double *__restrict__ LM,
                                          const double *__restrict__ MM, int i, int j, int k, double max_cs) {
  const long long p = lidx(g, i, j, k);
  if (nv[p] > 1) return 0.0;
  double w[27], lm[27], mm[27];
  long long src[27];
  wrap_weights(g, wgt, i, j, k, w, src);
#pragma unroll
  for (int n = 0; n < 27; n++) { lm[n] = LM[src[n]]; mm[n] = MM[src[n]]; }
  const double ws = tf_wsum(w);
  const double LM_avg = tf_apply(lm, w, ws);
  const double MM_avg = tf_apply(mm, w, ws);
  const double C = 0.5 * LM_avg / (MM_avg + kLesEps);
  double cs = (C < 0) ? 0 : C;                       // PetscMax(C, 0)
  if (nv[p] == 1) cs = (kWallCs < cs) ? cs : kWallCs;  // PetscMax(wall_cs, Cs) at IB nodes
  cs = (cs < 0) ? 0 : cs;
  cs = (cs < max_cs) ? cs : max_cs;                 // PetscMin(PetscMax(Cs, 0), max_cs)
  return cs;
}

// Every DA point: interior cells their clipped Cs, periodic ghosts the value of their image
// (zero when the image is itself a boundary point), other ghosts zero.
__global__ void k_les_cs(Grid g, const double *__restrict__ wgt, const uint8_t *__restrict__ nv,
                         const double *__restrict__ LM, const double *__restrict__ MM, double max_cs, double *cs) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int a = wrapi(g, i), b = wrapj(g, j), c = wrapk(g, k);
  cs[p] = les_interior(g, a, b, c) ? cs_cell(g, wgt, nv, LM, MM, a, b, c, max_cs) : 0.0;
}

// Second filtering of Cs over fluid cells (nvert < 0.1); every other point keeps its value.
__global__ void k_les_refilter(Grid g, const double *__restrict__ wgt, const uint8_t *__restrict__ nv,
                               const double *__restrict__ cs_tmp, double *cs) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (!les_interior(g, i, j, k) || nv[p] != 0) { cs[p] = cs_tmp[p]; return; }
  double w[27], v[27];
  long long src[27];
  wrap_weights(g, wgt, i, j, k, w, src);
#pragma unroll
  for (int n = 0; n < 27; n++) v[n] = cs_tmp[src[n]];
  cs[p] = tf_apply(v, w, tf_wsum(w));
}

// nu_t of one interior cell (les.c:1177-1198).
__device__ __forceinline__ double nut_cell(const Grid &g, CV3 u, CV3 csi, CV3 eta, CV3 zet,
                                           const double *__restrict__ aj, const uint8_t *__restrict__ nv,
                                           const double *__restrict__ cs, int i, int j, int k) {
  const long long p = lidx(g, i, j, k);
  if (nv[p] > 1) return 0.0;
  double d[9], gr[9], s[6];
  du_center(g, u, nv, p, i, j, k, d);
  const double cc[3] = {csi.x[p], csi.y[p], csi.z[p]};
  const double ee[3] = {eta.x[p], eta.y[p], eta.z[p]};
  const double zz[3] = {zet.x[p], zet.y[p], zet.z[p]};
  du_dxyz(cc, ee, zz, aj[p], d, gr);
  const double sabs = strain(gr, s);
  const double filter = pow(1. / aj[p], 1. / 3.);
  return cs[p] * pow(filter, 2.0) * sabs;
}

// Interior cells and periodic ghosts (value of the image; the old value of the image when
// the image is a non-periodic boundary point); other ghosts keep their value.
__global__ void k_les_nut(Grid g, CV3 u, CV3 csi, CV3 eta, CV3 zet, const double *__restrict__ aj,
                          const uint8_t *__restrict__ nv, const double *__restrict__ cs, double *nut) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int a = wrapi(g, i), b = wrapj(g, j), c = wrapk(g, k);
  if (les_interior(g, a, b, c)) nut[p] = nut_cell(g, u, csi, eta, zet, aj, nv, cs, a, b, c);
  else if (a != i || b != j || c != k) nut[p] = nut[lidx(g, a, b, c)];
}

__global__ void k_fill(long long n, double v, double *a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) a[p] = v;
}

// ------------------------------------------------------------------ host side
// Scratch: the Formfunction_2 face-flux arrays, idle while the eddy viscosity is formed
// (Flow_Solver computes it before the momentum step, solvers.c:648-654).
static LesPrep les_scratch(Ctx *c, double **LM, double **MM, double **cs_tmp) {
  LesPrep o;
  o.U = c->div[0][0]; o.V = c->div[0][1]; o.W = c->div[0][2];
  o.wgt = c->div[1][0];
  o.ss[0] = c->div[1][1]; o.ss[1] = c->div[1][2]; o.ss[2] = c->div[2][0];
  o.ss[3] = c->div[2][1]; o.ss[4] = c->div[2][2]; o.ss[5] = c->visc[0][0];
  o.uf[0] = c->visc[0][1]; o.uf[1] = c->visc[0][2]; o.uf[2] = c->visc[1][0];
  *LM = c->visc[1][1]; *MM = c->visc[1][2]; *cs_tmp = c->visc[2][0];
  return o;
}

int smagorinsky_constant(Ctx *c) {
  const Grid &g = c->g;
  double *cs = c->f[VFS_CS][0];
  int rc;
  if (c->ti < 2 && c->tistart == 0 && !c->rstart) {  // les.c:69-72
    cudaMemsetAsync(cs, 0, sizeof(double) * (size_t)g.N, c->stream);
    return VFS_OK;
  }
  if (g.les == 1) {  // les.c:74-77
    c->launches++, k_fill<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g.N, 0.01, cs);
    return check_launch(c, "k_fill");
  }
  Metrics m = metrics(c);
  double *LM, *MM, *cs_tmp;
  LesPrep o = les_scratch(c, &LM, &MM, &cs_tmp);
  CV3 u = cv(field3(c, VFS_UCAT));
  c->launches++, k_les_prep<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, u, m.csi, m.eta, m.zet, m.aj, c->nv, o);
  if ((rc = check_launch(c, "k_les_prep"))) return rc;
  c->launches++, k_les_image<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, u, m.csi, m.eta, m.zet, m.aj, c->nv, o);
  if ((rc = check_launch(c, "k_les_image"))) return rc;
  cudaMemsetAsync(LM, 0, sizeof(double) * (size_t)g.N, c->stream);
  cudaMemsetAsync(MM, 0, sizeof(double) * (size_t)g.N, c->stream);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_les_lm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LesLmSmem));
    attr = true;
  }
  LesLmIn in;
  in.u = u;
  in.U = o.U; in.V = o.V; in.W = o.W; in.wgt = o.wgt;
  for (int q = 0; q < 6; q++) in.ss[q] = o.ss[q];
  in.uf = CV3{o.uf[0], o.uf[1], o.uf[2]};
  dim3 grid((g.mx - 2 + LTX - 1) / LTX, (g.my - 2 + LTY - 1) / LTY, (g.mz - 2 + LTZ - 1) / LTZ);
  c->launches++, k_les_lm<<<grid, kLesLmThreads, sizeof(LesLmSmem), c->stream>>>(g, in, m.csi, m.eta, m.zet, m.aj, c->nv, LM, MM);
  if ((rc = check_launch(c, "k_les_lm"))) return rc;
  if ((rc = periodic_copy3(c, V3{LM, MM, nullptr}))) return rc;
  c->launches++, k_les_cs<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, o.wgt, c->nv, LM, MM, c->max_cs, cs_tmp);
  if ((rc = check_launch(c, "k_les_cs"))) return rc;
  c->launches++, k_les_refilter<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, o.wgt, c->nv, cs_tmp, cs);
  return check_launch(c, "k_les_refilter");
}

int eddy_viscosity(Ctx *c) {
  const Grid &g = c->g;
  Metrics m = metrics(c);
  c->launches++, k_les_nut<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, cv(field3(c, VFS_UCAT)), m.csi, m.eta, m.zet, m.aj, c->nv,
                                                     c->f[VFS_CS][0], c->f[VFS_NU_T][0]);
  return check_launch(c, "k_les_nut");
}

}  // namespace vfs
