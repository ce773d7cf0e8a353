/*
 * vfs_oracle.c — CPU restatement of the reference's projection-path algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: a plain-C restatement, written here, of
 * the reference functions the B200 library replaces.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg call it, to compare against.  It is pinned bit for bit
 * against the reference's own code (oracle/_ref, the reference sources compiled under a
 * single-rank PETSc shim) by tests/test_oracle_cpu.py.
 *
 * Data layout: the reference's PETSc DA, mx = IM+1 points per direction (init.c:154),
 * linear index ((k*my)+j)*mx+i; vector fields interleaved {x,y,z} (struct Cmpnts,
 * variables.h:45-57); nvert as doubles (0 fluid, 1 IB node, 3 solid).
 *
 * Options covered: i/j/k_periodic (DA non-periodic, ghost copies), immersed 0/1 (QUICK
 * next to IB nodes), les with a given eddy viscosity, no levelset/RANS/skew/weno.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int mx, my, mz;
  int iper, jper, kper;
  int immersed, les;
  int bc[6];
  double ren, dt, st;
} og_grid;

#define IX(g, i, j, k) ((((size_t)(k)) * (g)->my + (j)) * (g)->mx + (i))
#define V(a, g, i, j, k, c) ((a)[3 * IX(g, i, j, k) + (c)])
#define S(a, g, i, j, k) ((a)[IX(g, i, j, k)])

/* periodic image of a ghost index (the copy loops, e.g. momentum.c:641-669) */
static int wrap(int per, int m, int i) {
  if (per) { if (i == 0) return m - 2; if (i == m - 1) return 1; }
  return i;
}

/* Copy all components of every periodic-ghost point from its image (dof 1 or 3). */
void og_periodic_copy(const og_grid *g, double *a, int dof) {
  for (int k = 0; k < g->mz; k++)
    for (int j = 0; j < g->my; j++)
      for (int i = 0; i < g->mx; i++) {
        int a_ = wrap(g->iper, g->mx, i), b_ = wrap(g->jper, g->my, j), c_ = wrap(g->kper, g->mz, k);
        if (a_ == i && b_ == j && c_ == k) continue;
        for (int q = 0; q < dof; q++) a[dof * IX(g, i, j, k) + q] = a[dof * IX(g, a_, b_, c_) + q];
      }
}

/* ------------------------------------------------------------------ FormMetrics
 * metrics.c:4-1347 (NEWMETRIC).  coor: nodes [k][j][i] for i<IM=mx-1 etc (3 doubles).
 * Outputs are the local (ghosted) metric vectors the solver reads. */
void og_form_metrics(const og_grid *g, const double *X, const double *Y, const double *Z,
                     double *cent, double *csi, double *eta, double *zet, double *aj,
                     double *icsi, double *ieta, double *izet, double *iaj,
                     double *jcsi, double *jeta, double *jzet, double *jaj,
                     double *kcsi, double *keta, double *kzet, double *kaj) {
  const int mx = g->mx, my = g->my, mz = g->mz, IM = mx - 1, JM = my - 1;
  const size_t N = (size_t)mx * my * mz;
  memset(cent, 0, 24 * N); memset(csi, 0, 24 * N); memset(eta, 0, 24 * N); memset(zet, 0, 24 * N);
  memset(aj, 0, 8 * N);
#define NODE(a, i, j, k) (a[((size_t)(k) * JM + (j)) * IM + (i)])
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const double *C[3] = {X, Y, Z};
        double c8[3];
        for (int d = 0; d < 3; d++) {
          const double *a = C[d];
          c8[d] = 0.125 * (NODE(a, i, j, k) + NODE(a, i, j - 1, k) + NODE(a, i, j, k - 1) + NODE(a, i, j - 1, k - 1) +
                           NODE(a, i - 1, j, k) + NODE(a, i - 1, j - 1, k) + NODE(a, i - 1, j, k - 1) +
                           NODE(a, i - 1, j - 1, k - 1));
          V(cent, g, i, j, k, d) = c8[d];
        }
        double dc[3], de[3], dz[3];
        for (int d = 0; d < 3; d++) {
          const double *a = C[d];
          dc[d] = 0.25 * (NODE(a, i, j, k) + NODE(a, i, j - 1, k) + NODE(a, i, j, k - 1) + NODE(a, i, j - 1, k - 1) -
                          NODE(a, i - 1, j, k) - NODE(a, i - 1, j - 1, k) - NODE(a, i - 1, j, k - 1) -
                          NODE(a, i - 1, j - 1, k - 1));
          de[d] = 0.25 * (NODE(a, i, j, k) + NODE(a, i - 1, j, k) + NODE(a, i, j, k - 1) + NODE(a, i - 1, j, k - 1) -
                          NODE(a, i, j - 1, k) - NODE(a, i - 1, j - 1, k) - NODE(a, i, j - 1, k - 1) -
                          NODE(a, i - 1, j - 1, k - 1));
          dz[d] = 0.25 * (NODE(a, i, j, k) + NODE(a, i, j - 1, k) + NODE(a, i - 1, j, k) + NODE(a, i - 1, j - 1, k) -
                          NODE(a, i, j, k - 1) - NODE(a, i, j - 1, k - 1) - NODE(a, i - 1, j, k - 1) -
                          NODE(a, i - 1, j - 1, k - 1));
        }
        const double dxdc = dc[0], dydc = dc[1], dzdc = dc[2];
        const double dxde = de[0], dyde = de[1], dzde = de[2];
        const double dxdz = dz[0], dydz = dz[1], dzdz = dz[2];
        double J = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) +
                   dzdc * (dxde * dydz - dyde * dxdz);
        S(aj, g, i, j, k) = 1. / J;
        V(csi, g, i, j, k, 0) = dyde * dzdz - dzde * dydz;
        V(csi, g, i, j, k, 1) = -dxde * dzdz + dzde * dxdz;
        V(csi, g, i, j, k, 2) = dxde * dydz - dyde * dxdz;
        V(eta, g, i, j, k, 0) = dydz * dzdc - dzdz * dydc;
        V(eta, g, i, j, k, 1) = -dxdz * dzdc + dzdz * dxdc;
        V(eta, g, i, j, k, 2) = dxdz * dydc - dydz * dxdc;
        V(zet, g, i, j, k, 0) = dydc * dzde - dzdc * dyde;
        V(zet, g, i, j, k, 1) = -dxdc * dzde + dzdc * dxde;
        V(zet, g, i, j, k, 2) = dxdc * dyde - dydc * dxde;
      }
#undef NODE
  /* ghost planes from their neighbour plane: i, then j, then k (metrics.c:255-335) */
  double *cm[3] = {csi, eta, zet};
  for (int pass = 0; pass < 3; pass++)
    for (int k = 0; k < mz; k++)
      for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) {
          int si = i, sj = j, sk = k;
          if (pass == 0) { if (i == 0) si = 1; else if (i == mx - 1) si = mx - 2; else continue; }
          if (pass == 1) { if (j == 0) sj = 1; else if (j == my - 1) sj = my - 2; else continue; }
          if (pass == 2) { if (k == 0) sk = 1; else if (k == mz - 1) sk = mz - 2; else continue; }
          for (int m = 0; m < 3; m++)
            for (int c = 0; c < 3; c++) V(cm[m], g, i, j, k, c) = V(cm[m], g, si, sj, sk, c);
          S(aj, g, i, j, k) = S(aj, g, si, sj, sk);
        }
  og_periodic_copy(g, csi, 3); og_periodic_copy(g, eta, 3); og_periodic_copy(g, zet, 3);
  og_periodic_copy(g, aj, 1);
  /* face metrics: averages of the two centre metrics, harmonic mean of aj */
  double *fm[3][3] = {{icsi, ieta, izet}, {jcsi, jeta, jzet}, {kcsi, keta, kzet}};
  double *fa[3] = {iaj, jaj, kaj};
  for (int d = 0; d < 3; d++) {
    for (int m = 0; m < 3; m++) memset(fm[d][m], 0, 24 * N);
    memset(fa[d], 0, 8 * N);
  }
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        const int ii = i >= 1 && i <= mx - 2, jj = j >= 1 && j <= my - 2, kk = k >= 1 && k <= mz - 2;
        int ok[3] = {i <= mx - 2 && jj && kk, j <= my - 2 && ii && kk, k <= mz - 2 && ii && jj};
        int e[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
        for (int d = 0; d < 3; d++) {
          if (!ok[d]) continue;
          for (int m = 0; m < 3; m++)
            for (int c = 0; c < 3; c++)
              V(fm[d][m], g, i, j, k, c) = 0.5 * V(cm[m], g, i, j, k, c) + 0.5 * V(cm[m], g, e[d][0], e[d][1], e[d][2], c);
          S(fa[d], g, i, j, k) = 2. / (1. / S(aj, g, i, j, k) + 1. / S(aj, g, e[d][0], e[d][1], e[d][2]));
        }
      }
  for (int d = 0; d < 3; d++) {
    for (int m = 0; m < 3; m++) og_periodic_copy(g, fm[d][m], 3);
    og_periodic_copy(g, fa[d], 1);
  }
}

/* ------------------------------------------------------------------ Contra2Cart
 * rhs.c:57-675 for the boundary codes 1 (no-slip), 10 (free-slip), 4 (outlet), the
 * solid cells (nvert==3) and the periodic copies. */
static void covariant_col(const double *csi, const double *eta, const double *zet, int col, double n[3]) {
  const double a11 = csi[0], a12 = csi[1], a13 = csi[2];
  const double a21 = eta[0], a22 = eta[1], a23 = eta[2];
  const double a31 = zet[0], a32 = zet[1], a33 = zet[2];
  double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
  double G[3][3];
  G[0][0] = (a33 * a22 - a32 * a23) / det, G[0][1] = -(a33 * a12 - a32 * a13) / det, G[0][2] = (a23 * a12 - a22 * a13) / det;
  G[1][0] = -(a33 * a21 - a31 * a23) / det, G[1][1] = (a33 * a11 - a31 * a13) / det, G[1][2] = -(a23 * a11 - a21 * a13) / det;
  G[2][0] = (a32 * a21 - a31 * a22) / det, G[2][1] = -(a32 * a11 - a31 * a12) / det, G[2][2] = (a22 * a11 - a21 * a12) / det;
  n[0] = G[0][col]; n[1] = G[1][col]; n[2] = G[2][col];
}

void og_contra2cart(const og_grid *g, double *ucont, const double *csi, const double *eta, const double *zet,
                    const double *nvert, const double *ucat_old, double *ucat) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  const int *bc = g->bc;
  const size_t N = (size_t)mx * my * mz;
  og_periodic_copy(g, ucont, 3);
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        if (!(S(nvert, g, i, j, k) < 0.1)) continue;
        const double *c = &V(csi, g, i, j, k, 0), *e = &V(eta, g, i, j, k, 0), *z = &V(zet, g, i, j, k, 0);
        double q0 = 0.5 * (V(ucont, g, i - 1, j, k, 0) + V(ucont, g, i, j, k, 0));
        double q1 = 0.5 * (V(ucont, g, i, j - 1, k, 1) + V(ucont, g, i, j, k, 1));
        double q2 = 0.5 * (V(ucont, g, i, j, k - 1, 2) + V(ucont, g, i, j, k, 2));
        double det = c[0] * (e[1] * z[2] - e[2] * z[1]) - c[1] * (e[0] * z[2] - e[2] * z[0]) + c[2] * (e[0] * z[1] - e[1] * z[0]);
        double d0 = q0 * (e[1] * z[2] - e[2] * z[1]) - q1 * (c[1] * z[2] - c[2] * z[1]) + q2 * (c[1] * e[2] - c[2] * e[1]);
        double d1 = -q0 * (e[0] * z[2] - e[2] * z[0]) + q1 * (c[0] * z[2] - c[2] * z[0]) - q2 * (c[0] * e[2] - c[2] * e[0]);
        double d2 = q0 * (e[0] * z[1] - e[1] * z[0]) - q1 * (c[0] * z[1] - c[1] * z[0]) + q2 * (c[0] * e[1] - c[1] * e[0]);
        V(ucat, g, i, j, k, 0) = d0 / det;
        V(ucat, g, i, j, k, 1) = d1 / det;
        V(ucat, g, i, j, k, 2) = d2 / det;
      }
  og_periodic_copy(g, ucat, 3);
  /* boundary loop reads the snapshot lu and writes ucat */
  double *lu = (double *)malloc(24 * N);
  memcpy(lu, ucat, 24 * N);
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        double *o = &V(ucat, g, i, j, k, 0);
        if ((int)(S(nvert, g, i, j, k) + 0.1) == 3) { o[0] = o[1] = o[2] = 0; continue; }
        int solid_flag = 0;
        int slip[4][4] = {{bc[0] == 10 && i == 0 && j != 0 && k != 0, i + 1, 0, -1},
                          {bc[1] == 10 && i == mx - 1 && j != 0 && k != 0, i - 1, 0, 1},
                          {bc[2] == 10 && j == 0 && i != 0 && k != 0, j + 1, 1, -1},
                          {(bc[3] == 10 || bc[3] == -10) && j == my - 1 && i != 0 && k != 0, j - 1, 1, 1}};
        for (int s = 0; s < 4; s++) {
          if (!slip[s][0]) continue;
          int ni = s < 2 ? slip[s][1] : i, nj = s < 2 ? j : slip[s][1];
          double n[3];
          covariant_col(&V(csi, g, ni, nj, k, 0), &V(eta, g, ni, nj, k, 0), &V(zet, g, ni, nj, k, 0), slip[s][2], n);
          if (slip[s][3] < 0) n[0] = -n[0], n[1] = -n[1], n[2] = -n[2];
          double sum = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
          n[0] /= sum, n[1] /= sum, n[2] /= sum;
          const double *uo = &V(ucat_old, g, ni, nj, k, 0);
          double un = uo[0] * n[0] + uo[1] * n[1] + uo[2] * n[2];
          for (int c = 0; c < 3; c++) o[c] = uo[c] - 2 * un * n[c];
          if (S(nvert, g, ni, nj, k) > 0.1) o[0] = o[1] = o[2] = 0;
          if (solid_flag) o[0] = o[1] = o[2] = 0;
        }
        int ns[6][4] = {{i == 0 && bc[0] == 1 && j != 0 && k != 0, 1, 0, 0},
                        {i == mx - 1 && bc[1] == 1 && j != 0 && k != 0, -1, 0, 0},
                        {j == 0 && bc[2] == 1 && i != 0 && k != 0, 0, 1, 0},
                        {j == my - 1 && bc[3] == 1 && i != 0 && k != 0, 0, -1, 0},
                        {k == 0 && bc[4] == 1 && i != 0 && j != 0, 0, 0, 1},
                        {k == mz - 1 && bc[5] == 1 && i != 0 && j != 0, 0, 0, -1}};
        for (int s = 0; s < 6; s++) {
          if (!ns[s][0]) continue;
          const double *src = &lu[3 * IX(g, i + ns[s][1], j + ns[s][2], k + ns[s][3])];
          for (int c = 0; c < 3; c++) o[c] = -1 * src[c];
          solid_flag = 1;
        }
        if (bc[3] == 4 && j == my - 1 && i != 0 && i != mx - 1 && k != 0 && k != mz - 1)
          for (int c = 0; c < 3; c++) o[c] = lu[3 * IX(g, i, j - 1, k) + c];
        if (bc[5] == 4 && k == mz - 1 && i != 0 && i != mx - 1 && j != 0 && j != my - 1) {
          if (S(nvert, g, i, j, k - 1) > 0.1) o[0] = o[1] = o[2] = 0;
          if (solid_flag) o[0] = o[1] = o[2] = 0;
        }
        if (i != 0 && i != mx - 1 && j != 0 && j != my - 2 && k != 0 && k != mz - 2) {
          if (bc[0] <= 1 && bc[2] <= 1 && i == 1 && j == 1) o[0] = o[1] = o[2] = 0;
          if (bc[1] <= 1 && bc[2] <= 1 && i == mx - 2 && j == 1) o[0] = o[1] = o[2] = 0;
        }
      }
  free(lu);
  og_periodic_copy(g, ucat, 3);
}

/* ------------------------------------------------------------------ Formfunction_2
 * momentum.c:456-1980.  rhs is accumulated (scale * RHS added at interior faces, masked
 * faces set to 0, boundary points set to 0). */
typedef struct {
  const double *icsi, *ieta, *izet, *iaj, *jcsi, *jeta, *jzet, *jaj, *kcsi, *keta, *kzet, *kaj;
  const double *csi, *eta, *zet;
} og_metrics;

/* face gradient of ucat along the face normal d, cross derivatives one-sided next to
 * nvert > 0.1 (Compute_du_i/j/k, k-omega.c:48-300). du[a][c]: a = derivative direction
 * (csi, eta, zeta), c = velocity component. */
static void face_grad(const og_grid *g, const double *u, const double *nv, int i, int j, int k, int d,
                      double du[3][3]) {
  int o[3] = {0, 0, 0};
  o[d] = 1;
  for (int a = 0; a < 3; a++) {
    if (a == d) {
      for (int c = 0; c < 3; c++)
        du[a][c] = V(u, g, i + o[0], j + o[1], k + o[2], c) - V(u, g, i, j, k, c);
      continue;
    }
    int e[3] = {0, 0, 0};
    e[a] = 1;
    int pl = S(nv, g, i + e[0], j + e[1], k + e[2]) > 0.1 ||
             S(nv, g, i + e[0] + o[0], j + e[1] + o[1], k + e[2] + o[2]) > 0.1;
    int mi = S(nv, g, i - e[0], j - e[1], k - e[2]) > 0.1 ||
             S(nv, g, i - e[0] + o[0], j - e[1] + o[1], k - e[2] + o[2]) > 0.1;
    for (int c = 0; c < 3; c++) {
      const double a0 = V(u, g, i, j, k, c), a1 = V(u, g, i + o[0], j + o[1], k + o[2], c);
      const double p0 = V(u, g, i + e[0], j + e[1], k + e[2], c), p1 = V(u, g, i + e[0] + o[0], j + e[1] + o[1], k + e[2] + o[2], c);
      const double m0 = V(u, g, i - e[0], j - e[1], k - e[2], c), m1 = V(u, g, i - e[0] + o[0], j - e[1] + o[1], k - e[2] + o[2], c);
      if (pl) du[a][c] = (a1 + a0 - m1 - m0) * 0.5;
      else if (mi) du[a][c] = (p1 + p0 - a1 - a0) * 0.5;
      else du[a][c] = (p1 + p0 - m1 - m0) * 0.25;
    }
  }
}

static void face_flux(const og_grid *g, const og_metrics *M, const double *ucont, const double *u,
                      const double *nv, const double *nut, int i, int j, int k, int d, double div[3],
                      double visc[3]) {
  const int m[3] = {g->mx, g->my, g->mz};
  const int per[3] = {g->iper, g->jper, g->kper};
  const int idx[3] = {i, j, k};
  const int x = idx[d];
  int o[3] = {0, 0, 0};
  o[d] = 1;
  const double *fc[3][4] = {{M->icsi, M->ieta, M->izet, M->iaj}, {M->jcsi, M->jeta, M->jzet, M->jaj},
                            {M->kcsi, M->keta, M->kzet, M->kaj}};
  const double ajc = S(fc[d][3], g, i, j, k);
  const double *c_ = &V(fc[d][0], g, i, j, k, 0), *e_ = &V(fc[d][1], g, i, j, k, 0), *z_ = &V(fc[d][2], g, i, j, k, 0);
  const double csi0 = c_[0], csi1 = c_[1], csi2 = c_[2], eta0 = e_[0], eta1 = e_[1], eta2 = e_[2];
  const double zet0 = z_[0], zet1 = z_[1], zet2 = z_[2];
  double du[3][3];
  face_grad(g, u, nv, i, j, k, d, du);
  /* metric products along the face normal (g11, g21, g31 of the face) */
  const double *nrm = d == 0 ? c_ : (d == 1 ? e_ : z_);
  const double g11 = csi0 * nrm[0] + csi1 * nrm[1] + csi2 * nrm[2];
  const double g21 = eta0 * nrm[0] + eta1 * nrm[1] + eta2 * nrm[2];
  const double g31 = zet0 * nrm[0] + zet1 * nrm[1] + zet2 * nrm[2];
  /* in the reference, g11 = csi.csi is written csi0*csi0+..., g21 = eta.csi as
     eta0*csi0+...; the products commute bit-exactly */
  double r[3][3];
  for (int c = 0; c < 3; c++) {
    r[0][c] = du[0][c] * csi0 + du[1][c] * eta0 + du[2][c] * zet0;
    r[1][c] = du[0][c] * csi1 + du[1][c] * eta1 + du[2][c] * zet1;
    r[2][c] = du[0][c] * csi2 + du[1][c] * eta2 + du[2][c] * zet2;
  }
  int xL = x - 1, xR = x + 2;
  int pL[3] = {i, j, k}, pR[3] = {i, j, k};
  if (x == 0 || x == m[d] - 2) {
    if (per[d]) xL = m[d] - 3, xR = 2;
    else xL = x, xR = x + 1;
  } else {
    int a[3] = {i, j, k}, b[3] = {i, j, k};
    a[d] = x - 1; b[d] = x + 2;
    if (S(nv, g, a[0], a[1], a[2]) + S(nv, g, b[0], b[1], b[2]) > 0.1) xL = x, xR = x + 1;
  }
  pL[d] = xL; pR[d] = xR;
  double ucon = V(ucont, g, i, j, k, d);
  if (per[d] && (x == 0 || x == m[d] - 2)) {
    int s[3] = {i, j, k};
    s[d] = m[d] - 2;
    ucon = V(ucont, g, s[0], s[1], s[2], d);
  }
  if (d == 2 && k == g->mz - 2 && g->bc[5] == 4 && (int)S(nv, g, i, j, k) == 0) ucon = V(ucont, g, i, j, k - 1, 2);
  const double up = -0.5 * (ucon + fabs(ucon));
  const double um = -0.5 * (ucon - fabs(ucon));
  for (int c = 0; c < 3; c++) {
    const double u0 = V(u, g, i, j, k, c), u1 = V(u, g, i + o[0], j + o[1], k + o[2], c);
    if (g->immersed && x != m[d] - 2 && S(nv, g, i, j, k) > 0.1) {
      const double u2 = V(u, g, i + 2 * o[0], j + 2 * o[1], k + 2 * o[2], c);
      div[c] = um * (0.125 * (-u2 - 2. * u1 + 3. * u0) + u1) + up * (0.125 * (-u0 - 2. * u0 + 3. * u1) + u0);
    } else if (g->immersed && x != 0 && S(nv, g, i + o[0], j + o[1], k + o[2]) > 0.1) {
      const double um1 = V(u, g, i - o[0], j - o[1], k - o[2], c);
      div[c] = um * (0.125 * (-u1 - 2. * u1 + 3. * u0) + u1) + up * (0.125 * (-um1 - 2. * u0 + 3. * u1) + u0);
    } else {
      div[c] = -V(ucont, g, i, j, k, d) * 0.0625 *
               (-V(u, g, pL[0], pL[1], pL[2], c) + 9. * u0 + 9. * u1 - V(u, g, pR[0], pR[1], pR[2], c));
    }
  }
  if (S(nv, g, i, j, k) + S(nv, g, i + o[0], j + o[1], k + o[2]) > 0.1 && !g->immersed) div[0] = div[1] = div[2] = 0;
  const double nu = 1. / g->ren;
  double nut_f = 0;
  if (g->les) {
    if ((x == 0 && !per[d]) || S(nv, g, i, j, k) > 0.1) nut_f = S(nut, g, i + o[0], j + o[1], k + o[2]);
    else if ((x == m[d] - 2 && !per[d]) || S(nv, g, i + o[0], j + o[1], k + o[2]) > 0.1) nut_f = S(nut, g, i, j, k);
    else nut_f = 0.5 * (S(nut, g, i, j, k) + S(nut, g, i + o[0], j + o[1], k + o[2]));
  }
  for (int c = 0; c < 3; c++) {
    const double t = g11 * du[0][c] + g21 * du[1][c] + g31 * du[2][c] + r[c][0] * nrm[0] + r[c][1] * nrm[1] +
                     r[c][2] * nrm[2];
    double v = 0;
    if (g->les) v = t * ajc * (nut_f);
    v += t * ajc * (nu);
    visc[c] = v;
  }
}

void og_formfunction2(const og_grid *g, const og_metrics *M, double *ucont, const double *ucat,
                      const double *nvert, const double *nut, double scale, double *rhs) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  const size_t N = (size_t)mx * my * mz;
  og_periodic_copy(g, ucont, 3);
  double *div[3], *visc[3];
  for (int d = 0; d < 3; d++) {
    div[d] = (double *)calloc(3 * N, sizeof(double));
    visc[d] = (double *)calloc(3 * N, sizeof(double));
  }
  double *fp = (double *)calloc(3 * N, sizeof(double));
  for (int k = 0; k < mz - 1; k++)
    for (int j = 0; j < my - 1; j++)
      for (int i = 0; i < mx - 1; i++) {
        if (j != 0 && k != 0) face_flux(g, M, ucont, ucat, nvert, nut, i, j, k, 0, &V(div[0], g, i, j, k, 0), &V(visc[0], g, i, j, k, 0));
        if (i != 0 && k != 0) face_flux(g, M, ucont, ucat, nvert, nut, i, j, k, 1, &V(div[1], g, i, j, k, 0), &V(visc[1], g, i, j, k, 0));
        if (i != 0 && j != 0) face_flux(g, M, ucont, ucat, nvert, nut, i, j, k, 2, &V(div[2], g, i, j, k, 0), &V(visc[2], g, i, j, k, 0));
      }
  for (int d = 0; d < 3; d++) { og_periodic_copy(g, div[d], 3); og_periodic_copy(g, visc[d], 3); }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        int R[3] = {i + 1, j + 1, k + 1}, L[3] = {i - 2, j - 2, k - 2};
        double den[3] = {3., 3., 3.};
        const int x[3] = {i, j, k}, m[3] = {mx, my, mz}, per[3] = {g->iper, g->jper, g->kper};
        for (int d = 0; d < 3; d++) {
          if (x[d] == 1) { if (per[d]) L[d] = m[d] - 3; else R[d] = x[d], L[d] = x[d] - 1, den[d] = 1.; }
          else if (x[d] == 2 || x[d] == m[d] - 3) { if (!per[d]) R[d] = x[d], L[d] = x[d] - 1, den[d] = 1.; }
          else if (x[d] == m[d] - 2) { if (per[d]) R[d] = 1; else R[d] = x[d], L[d] = x[d] - 1, den[d] = 1.; }
        }
        if (S(nvert, g, i - 1, j, k) + S(nvert, g, i, j, k) + S(nvert, g, i + 1, j, k) > 0.1) R[0] = i, L[0] = i - 1, den[0] = 1.;
        if (S(nvert, g, i, j - 1, k) + S(nvert, g, i, j, k) + S(nvert, g, i, j + 1, k) > 0.1) R[1] = j, L[1] = j - 1, den[1] = 1.;
        if (S(nvert, g, i, j, k - 1) + S(nvert, g, i, j, k) + S(nvert, g, i, j, k + 1) > 0.1) R[2] = k, L[2] = k - 1, den[2] = 1.;
        for (int c = 0; c < 3; c++) {
          double dv = (V(div[0], g, i, j, k, c) - V(div[0], g, i - 1, j, k, c) + V(div[1], g, i, j, k, c) -
                       V(div[1], g, i, j - 1, k, c) + V(div[2], g, i, j, k, c) - V(div[2], g, i, j, k - 1, c));
          double d4 = 0;
          d4 += (V(div[0], g, R[0], j, k, c) - V(div[0], g, L[0], j, k, c)) * (1. / den[0]);
          d4 += (V(div[1], g, i, R[1], k, c) - V(div[1], g, i, L[1], k, c)) * (1. / den[1]);
          d4 += (V(div[2], g, i, j, R[2], c) - V(div[2], g, i, j, L[2], c)) * (1. / den[2]);
          double f = 9. / 8. * dv + -1. / 8. * d4;
          f += (V(visc[0], g, i, j, k, c) - V(visc[0], g, i - 1, j, k, c) + V(visc[1], g, i, j, k, c) -
                V(visc[1], g, i, j - 1, k, c) + V(visc[2], g, i, j, k, c) - V(visc[2], g, i, j, k - 1, c)) / 1.0;
          V(fp, g, i, j, k, c) = f;
        }
      }
  og_periodic_copy(g, fp, 3);
  const double *cm[3] = {M->csi, M->eta, M->zet};
  const double *fa[3] = {M->iaj, M->jaj, M->kaj};
  const int per[3] = {g->iper, g->jper, g->kper}, m[3] = {mx, my, mz};
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        double *r = &V(rhs, g, i, j, k, 0);
        if (i == 0 || i == mx - 1 || j == 0 || j == my - 1 || k == 0 || k == mz - 1) {
          r[0] = r[1] = r[2] = 0;
          continue;
        }
        const int x[3] = {i, j, k};
        for (int d = 0; d < 3; d++) {
          int e[3] = {i, j, k};
          e[d] += 1;
          const double *a = &V(cm[d], g, i, j, k, 0), *b = &V(cm[d], g, e[0], e[1], e[2], 0);
          const double *fa0 = &V(fp, g, i, j, k, 0), *fb = &V(fp, g, e[0], e[1], e[2], 0);
          r[d] += scale * (0.5 * (a[0] * fa0[0] + a[1] * fa0[1] + a[2] * fa0[2]) + 0.5 * (b[0] * fb[0] + b[1] * fb[1] + b[2] * fb[2])) *
                  S(fa[d], g, i, j, k);
          if (S(nvert, g, i, j, k) + S(nvert, g, e[0], e[1], e[2]) > 0.1 || (!per[d] && x[d] == m[d] - 2)) r[d] = 0;
        }
      }
  for (int d = 0; d < 3; d++) { free(div[d]); free(visc[d]); }
  free(fp);
}

/* ------------------------------------------------------------------ Pressure_Gradient
 * momentum.c:197-443 (levelset off).  kforce: 0 none, 1 mean_pressure_gradient (mpg),
 * 2 flux-deficit forcing (kdiff = mean_k_flux - inlet_flux, divided by dt and karea). */
void og_pressure_gradient(const og_grid *g, const og_metrics *M, const double *nvert, double *p,
                          int kforce, double mpg, double kdiff, double karea, double *dp) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  og_periodic_copy(g, p, 1);
  memset(dp, 0, 24 * (size_t)mx * my * mz);
#define P_(i, j, k) S(p, g, i, j, k)
#define IB(i, j, k) ((int)(S(nvert, g, i, j, k) + 0.5) == 1)
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const double *ic = &V(M->icsi, g, i, j, k, 0), *ie = &V(M->ieta, g, i, j, k, 0), *iz = &V(M->izet, g, i, j, k, 0);
        const double *jc = &V(M->jcsi, g, i, j, k, 0), *je = &V(M->jeta, g, i, j, k, 0), *jz = &V(M->jzet, g, i, j, k, 0);
        const double *kc = &V(M->kcsi, g, i, j, k, 0), *ke = &V(M->keta, g, i, j, k, 0), *kz = &V(M->kzet, g, i, j, k, 0);
        const double g11 = ic[0] * ic[0] + ic[1] * ic[1] + ic[2] * ic[2];
        const double g12 = ie[0] * ic[0] + ie[1] * ic[1] + ie[2] * ic[2];
        const double g13 = iz[0] * ic[0] + iz[1] * ic[1] + iz[2] * ic[2];
        const double g21 = jc[0] * je[0] + jc[1] * je[1] + jc[2] * je[2];
        const double g22 = je[0] * je[0] + je[1] * je[1] + je[2] * je[2];
        const double g23 = jz[0] * je[0] + jz[1] * je[1] + jz[2] * je[2];
        const double g31 = kc[0] * kz[0] + kc[1] * kz[1] + kc[2] * kz[2];
        const double g32 = ke[0] * kz[0] + ke[1] * kz[1] + ke[2] * kz[2];
        const double g33 = kz[0] * kz[0] + kz[1] * kz[1] + kz[2] * kz[2];
        double dpdc, dpde, dpdz;
        /* x face */
        dpdc = (i == mx - 2 && g->iper) ? P_(1, j, k) - P_(i, j, k) : P_(i + 1, j, k) - P_(i, j, k);
        if (IB(i, j + 1, k) || IB(i + 1, j + 1, k) || (j == my - 2 && !g->jper)) dpde = (P_(i, j, k) - P_(i, j - 1, k) + P_(i + 1, j, k) - P_(i + 1, j - 1, k)) * 0.5;
        else if (IB(i, j - 1, k) || IB(i + 1, j - 1, k) || (j == 1 && !g->jper)) dpde = (P_(i, j + 1, k) - P_(i, j, k) + P_(i + 1, j + 1, k) - P_(i + 1, j, k)) * 0.5;
        else dpde = (P_(i, j + 1, k) - P_(i, j - 1, k) + P_(i + 1, j + 1, k) - P_(i + 1, j - 1, k)) * 0.25;
        if (IB(i, j, k + 1) || IB(i + 1, j, k + 1) || (k == mz - 2 && !g->kper)) dpdz = (P_(i, j, k) - P_(i, j, k - 1) + P_(i + 1, j, k) - P_(i + 1, j, k - 1)) * 0.5;
        else if (IB(i, j, k - 1) || IB(i + 1, j, k - 1) || (k == 1 && !g->kper)) dpdz = (P_(i, j, k + 1) - P_(i, j, k) + P_(i + 1, j, k + 1) - P_(i + 1, j, k)) * 0.5;
        else dpdz = (P_(i, j, k + 1) - P_(i, j, k - 1) + P_(i + 1, j, k + 1) - P_(i + 1, j, k - 1)) * 0.25;
        double ox = (dpdc * g11 + dpde * g12 + dpdz * g13) * S(M->iaj, g, i, j, k) / 1.0;
        /* y face */
        if (IB(i + 1, j, k) || IB(i + 1, j + 1, k) || (i == mx - 2 && !g->iper)) dpdc = (P_(i, j, k) - P_(i - 1, j, k) + P_(i, j + 1, k) - P_(i - 1, j + 1, k)) * 0.5;
        else if (IB(i - 1, j, k) || IB(i - 1, j + 1, k) || (i == 1 && !g->iper)) dpdc = (P_(i + 1, j, k) - P_(i, j, k) + P_(i + 1, j + 1, k) - P_(i, j + 1, k)) * 0.5;
        else dpdc = (P_(i + 1, j, k) - P_(i - 1, j, k) + P_(i + 1, j + 1, k) - P_(i - 1, j + 1, k)) * 0.25;
        dpde = (j == my - 2 && g->jper) ? P_(i, 1, k) - P_(i, j, k) : P_(i, j + 1, k) - P_(i, j, k);
        if (IB(i, j, k + 1) || IB(i, j + 1, k + 1) || (k == mz - 2 && !g->kper)) dpdz = (P_(i, j, k) - P_(i, j, k - 1) + P_(i, j + 1, k) - P_(i, j + 1, k - 1)) * 0.5;
        else if (IB(i, j, k - 1) || IB(i, j + 1, k - 1) || (k == 1 && !g->kper)) dpdz = (P_(i, j, k + 1) - P_(i, j, k) + P_(i, j + 1, k + 1) - P_(i, j + 1, k)) * 0.5;
        else dpdz = (P_(i, j, k + 1) - P_(i, j, k - 1) + P_(i, j + 1, k + 1) - P_(i, j + 1, k - 1)) * 0.25;
        double oy = (dpdc * g21 + dpde * g22 + dpdz * g23) * S(M->jaj, g, i, j, k) / 1.0;
        /* z face */
        if (IB(i + 1, j, k) || IB(i + 1, j, k + 1) || (i == mx - 2 && !g->iper)) dpdc = (P_(i, j, k) - P_(i - 1, j, k) + P_(i, j, k + 1) - P_(i - 1, j, k + 1)) * 0.5;
        else if (IB(i - 1, j, k) || IB(i - 1, j, k + 1) || (i == 1 && !g->iper)) dpdc = (P_(i + 1, j, k) - P_(i, j, k) + P_(i + 1, j, k + 1) - P_(i, j, k + 1)) * 0.5;
        else dpdc = (P_(i + 1, j, k) - P_(i - 1, j, k) + P_(i + 1, j, k + 1) - P_(i - 1, j, k + 1)) * 0.25;
        if (IB(i, j + 1, k) || IB(i, j + 1, k + 1) || (j == my - 2 && !g->jper)) dpde = (P_(i, j, k) - P_(i, j - 1, k) + P_(i, j, k + 1) - P_(i, j - 1, k + 1)) * 0.5;
        else if (IB(i, j - 1, k) || IB(i, j - 1, k + 1) || (j == 1 && !g->jper)) dpde = (P_(i, j + 1, k) - P_(i, j, k) + P_(i, j + 1, k + 1) - P_(i, j, k + 1)) * 0.5;
        else dpde = (P_(i, j + 1, k) - P_(i, j - 1, k) + P_(i, j + 1, k + 1) - P_(i, j - 1, k + 1)) * 0.25;
        dpdz = (k == mz - 2 && g->kper) ? P_(i, j, 1) - P_(i, j, k) : (P_(i, j, k + 1) - P_(i, j, k));
        if (g->kper) {
          const double dz = 1. / S(M->kaj, g, i, j, k) / sqrt(kz[0] * kz[0] + kz[1] * kz[1] + kz[2] * kz[2]);
          if (kforce == 1) dpdz += mpg * dz;
          else if (kforce == 2) dpdz += dz * kdiff / g->dt / karea;
        }
        double oz = (dpdc * g31 + dpde * g32 + dpdz * g33) * S(M->kaj, g, i, j, k) / 1.0;
        if (S(nvert, g, i, j, k) + S(nvert, g, i + 1, j, k) > 0.1 || (!g->iper && i == mx - 2)) ox = 0;
        if (S(nvert, g, i, j, k) + S(nvert, g, i, j + 1, k) > 0.1 || (!g->jper && j == my - 2)) oy = 0;
        if (S(nvert, g, i, j, k) + S(nvert, g, i, j, k + 1) > 0.1 || (!g->kper && k == mz - 2)) oz = 0;
        V(dp, g, i, j, k, 0) = ox; V(dp, g, i, j, k, 1) = oy; V(dp, g, i, j, k, 2) = oz;
      }
#undef P_
#undef IB
}

/* ------------------------------------------------------------------ Poisson operator
 * PoissonLHSNew (poisson.c:971-1683): the matrix row of every fluid cell, stored on the
 * grid as 19 coefficients per cell in the slot order CP EP WP NP SP TP BP NE SE NW SW TN
 * BN TS BS TE BE TW BW, after the MatSetValues filter (|v| > 1e-10 with a valid column,
 * or the diagonal; INSERT: a later slot naming the same column wins). */
static const int OFF[19][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                               {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {0, 1, 1}, {0, 1, -1},
                               {0, -1, 1}, {0, -1, -1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1}, {-1, 0, -1}};
static int slot(int a, int b, int c) {
  for (int s = 0; s < 19; s++) if (OFF[s][0] == a && OFF[s][1] == b && OFF[s][2] == c) return s;
  return -1;
}

static void gab(const og_grid *g, const og_metrics *M, int i, int j, int k, double G[9]) {
  i = wrap(g->iper, g->mx, i); j = wrap(g->jper, g->my, j); k = wrap(g->kper, g->mz, k);
  const double *ic = &V(M->icsi, g, i, j, k, 0), *ie = &V(M->ieta, g, i, j, k, 0), *iz = &V(M->izet, g, i, j, k, 0);
  const double *jc = &V(M->jcsi, g, i, j, k, 0), *je = &V(M->jeta, g, i, j, k, 0), *jz = &V(M->jzet, g, i, j, k, 0);
  const double *kc = &V(M->kcsi, g, i, j, k, 0), *ke = &V(M->keta, g, i, j, k, 0), *kz = &V(M->kzet, g, i, j, k, 0);
  const double ia = S(M->iaj, g, i, j, k), ja = S(M->jaj, g, i, j, k), ka = S(M->kaj, g, i, j, k);
  G[0] = (ic[0] * ic[0] + ic[1] * ic[1] + ic[2] * ic[2]) * ia;
  G[1] = (ie[0] * ic[0] + ie[1] * ic[1] + ie[2] * ic[2]) * ia;
  G[2] = (iz[0] * ic[0] + iz[1] * ic[1] + iz[2] * ic[2]) * ia;
  G[3] = (jc[0] * je[0] + jc[1] * je[1] + jc[2] * je[2]) * ja;
  G[4] = (je[0] * je[0] + je[1] * je[1] + je[2] * je[2]) * ja;
  G[5] = (jz[0] * je[0] + jz[1] * je[1] + jz[2] * je[2]) * ja;
  G[6] = (kc[0] * kz[0] + kc[1] * kz[1] + kc[2] * kz[2]) * ka;
  G[7] = (ke[0] * kz[0] + ke[1] * kz[1] + ke[2] * kz[2]) * ka;
  G[8] = (kz[0] * kz[0] + kz[1] * kz[1] + kz[2] * kz[2]) * ka;
}

/* column (linear index) of the unknown at (i,j,k) after periodic wrap, or -1 */
static long col_at(const og_grid *g, const double *nv, int i, int j, int k) {
  i = wrap(g->iper, g->mx, i); j = wrap(g->jper, g->my, j); k = wrap(g->kper, g->mz, k);
  if (i < 1 || i > g->mx - 2 || j < 1 || j > g->my - 2 || k < 1 || k > g->mz - 2) return -1;
  if ((int)S(nv, g, i, j, k) > 0.1) return -1;
  return (long)IX(g, i, j, k);
}

/* one face's cross term: face to neighbour d, cross direction e with coordinate x along
 * m points, sign s (+1 for "x+1 - x", -1 for "x - x-1") */
static void cross(const og_grid *g, const double *nv, int i, int j, int k, const int d[3], const int e[3], int x, int m,
                  int per, double G, double s, double vol[19]) {
  double np_ = S(nv, g, i + e[0], j + e[1], k + e[2]) + S(nv, g, i + d[0] + e[0], j + d[1] + e[1], k + d[2] + e[2]);
  double nm_ = S(nv, g, i - e[0], j - e[1], k - e[2]) + S(nv, g, i + d[0] - e[0], j + d[1] - e[1], k + d[2] - e[2]);
  if ((x == m - 2 && !per) || np_ > 0.1) {
    if (nm_ < 0.1 && x != 1) {
      vol[0] += s * (G * 0.5); vol[slot(d[0], d[1], d[2])] += s * (G * 0.5);
      vol[slot(-e[0], -e[1], -e[2])] -= s * (G * 0.5);
      vol[slot(d[0] - e[0], d[1] - e[1], d[2] - e[2])] -= s * (G * 0.5);
    }
  } else if ((x == 1 && !per) || nm_ > 0.1) {
    if (np_ < 0.1) {
      vol[slot(e[0], e[1], e[2])] += s * (G * 0.5);
      vol[slot(d[0] + e[0], d[1] + e[1], d[2] + e[2])] += s * (G * 0.5);
      vol[0] -= s * (G * 0.5); vol[slot(d[0], d[1], d[2])] -= s * (G * 0.5);
    }
  } else {
    vol[slot(e[0], e[1], e[2])] += s * (G * 0.25);
    vol[slot(d[0] + e[0], d[1] + e[1], d[2] + e[2])] += s * (G * 0.25);
    vol[slot(-e[0], -e[1], -e[2])] -= s * (G * 0.25);
    vol[slot(d[0] - e[0], d[1] - e[1], d[2] - e[2])] -= s * (G * 0.25);
  }
}

void og_poisson_lhs(const og_grid *g, const og_metrics *M, const double *nv, double *coef) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  const size_t N = (size_t)mx * my * mz;
  memset(coef, 0, 19 * 8 * N);
  const int X1[3] = {1, 0, 0}, Xm[3] = {-1, 0, 0}, Y1[3] = {0, 1, 0}, Ym[3] = {0, -1, 0}, Z1[3] = {0, 0, 1}, Zm[3] = {0, 0, -1};
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        if (S(nv, g, i, j, k) > 0.1) continue;
        double vol[19] = {0}, G[9], Gm[9];
        gab(g, M, i, j, k, G);
        if (S(nv, g, i + 1, j, k) < 0.1 && (i != mx - 2 || g->iper)) {
          vol[0] -= G[0]; vol[1] += G[0];
          cross(g, nv, i, j, k, X1, Y1, j, my, g->jper, G[1], 1, vol);
          cross(g, nv, i, j, k, X1, Z1, k, mz, g->kper, G[2], 1, vol);
        }
        if (S(nv, g, i - 1, j, k) < 0.1 && (i != 1 || g->iper)) {
          gab(g, M, i - 1, j, k, Gm);
          vol[0] -= Gm[0]; vol[2] += Gm[0];
          cross(g, nv, i, j, k, Xm, Y1, j, my, g->jper, Gm[1], -1, vol);
          cross(g, nv, i, j, k, Xm, Z1, k, mz, g->kper, Gm[2], -1, vol);
        }
        if (S(nv, g, i, j + 1, k) < 0.1 && (j != my - 2 || g->jper)) {
          cross(g, nv, i, j, k, Y1, X1, i, mx, g->iper, G[3], 1, vol);
          vol[0] -= G[4]; vol[3] += G[4];
          cross(g, nv, i, j, k, Y1, Z1, k, mz, g->kper, G[5], 1, vol);
        }
        if (S(nv, g, i, j - 1, k) < 0.1 && (j != 1 || g->jper)) {
          gab(g, M, i, j - 1, k, Gm);
          cross(g, nv, i, j, k, Ym, X1, i, mx, g->iper, Gm[3], -1, vol);
          vol[0] -= Gm[4]; vol[4] += Gm[4];
          cross(g, nv, i, j, k, Ym, Z1, k, mz, g->kper, Gm[5], -1, vol);
        }
        if (S(nv, g, i, j, k + 1) < 0.1 && (k != mz - 2 || g->kper)) {
          cross(g, nv, i, j, k, Z1, X1, i, mx, g->iper, G[6], 1, vol);
          cross(g, nv, i, j, k, Z1, Y1, j, my, g->jper, G[7], 1, vol);
          vol[0] -= G[8]; vol[5] += G[8];
        }
        if (S(nv, g, i, j, k - 1) < 0.1 && (k != 1 || g->kper)) {
          gab(g, M, i, j, k - 1, Gm);
          cross(g, nv, i, j, k, Zm, X1, i, mx, g->iper, Gm[6], -1, vol);
          cross(g, nv, i, j, k, Zm, Y1, j, my, g->jper, Gm[7], -1, vol);
          vol[0] -= Gm[8]; vol[6] += Gm[8];
        }
        long col[19];
        int set[19];
        for (int s = 0; s < 19; s++) {
          col[s] = col_at(g, nv, i + OFF[s][0], j + OFF[s][1], k + OFF[s][2]);
          set[s] = (fabs(vol[s]) > 1.e-10 && col[s] >= 0) || s == 0;
        }
        for (int s = 0; s < 19; s++)
          for (int t = s + 1; t < 19 && set[s]; t++)
            if (set[t] && col[t] == col[s]) set[s] = 0;
        for (int s = 0; s < 19; s++) coef[s * N + IX(g, i, j, k)] = set[s] ? vol[s] : 0.0;
      }
}

/* y = A x on the grid layout (rows of fluid cells, columns through the periodic wrap) */
void og_poisson_apply(const og_grid *g, const double *coef, const double *nv, const double *x, double *y) {
  const size_t N = (size_t)g->mx * g->my * g->mz;
  memset(y, 0, 8 * N);
  for (int k = 1; k < g->mz - 1; k++)
    for (int j = 1; j < g->my - 1; j++)
      for (int i = 1; i < g->mx - 1; i++) {
        if (S(nv, g, i, j, k) > 0.1) continue;
        double s = 0;
        for (int t = 0; t < 19; t++) {
          const double c = coef[t * N + IX(g, i, j, k)];
          if (c == 0.0) continue;
          s += c * x[col_at(g, nv, i + OFF[t][0], j + OFF[t][1], k + OFF[t][2])];
        }
        y[IX(g, i, j, k)] = s;
      }
}

/* ------------------------------------------------------------------ Poisson RHS
 * PoissonRHS2_hypre (poisson_hypre.c:330-360) + Remove_Nullspace_Scale (:110). */
void og_poisson_rhs(const og_grid *g, const double *ucont, const double *nv, const double *aj, double *b) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  memset(b, 0, 8 * (size_t)mx * my * mz);
  double sum = 0, sum_aj = 0;
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        if (S(nv, g, i, j, k) >= 0.1) continue;
        double val = 0;
        val -= V(ucont, g, i, j, k, 0);
        val += (i == 1 && g->iper) ? V(ucont, g, mx - 2, j, k, 0) : V(ucont, g, i - 1, j, k, 0);
        val -= V(ucont, g, i, j, k, 1);
        val += (j == 1 && g->jper) ? V(ucont, g, i, my - 2, k, 1) : V(ucont, g, i, j - 1, k, 1);
        val -= V(ucont, g, i, j, k, 2);
        val += (k == 1 && g->kper) ? V(ucont, g, i, j, mz - 2, 2) : V(ucont, g, i, j, k - 1, 2);
        val *= -1.0 / g->dt * g->st * 1.0;
        S(b, g, i, j, k) = val;
        sum += val;
        sum_aj += S(aj, g, i, j, k);
      }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++)
        if (S(nv, g, i, j, k) < 0.1) S(b, g, i, j, k) += -sum * S(aj, g, i, j, k) / sum_aj;
}

/* ------------------------------------------------------------------ UpdatePressure,
 * Projection, Divergence (poisson.c:3144-3305, 2707-3065; main.c:1047-1177) */
void og_update_pressure(const og_grid *g, const double *nv, double *phi, double *p) {
  for (int k = 1; k < g->mz - 1; k++)
    for (int j = 1; j < g->my - 1; j++)
      for (int i = 1; i < g->mx - 1; i++) {
        if (S(nv, g, i, j, k) < 0.1) S(p, g, i, j, k) += S(phi, g, i, j, k);
        if (S(nv, g, i, j, k) > 1.1) S(p, g, i, j, k) = 0;
      }
  og_periodic_copy(g, p, 1);
  og_periodic_copy(g, phi, 1);
}

static double cross_phi(const og_grid *g, const double *phi, const double *nv, int i, int j, int k, const int d[3],
                        const int e[3], int x, int m, int per) {
  const double np_ = S(nv, g, i + e[0], j + e[1], k + e[2]) + S(nv, g, i + d[0] + e[0], j + d[1] + e[1], k + d[2] + e[2]);
  const double nm_ = S(nv, g, i - e[0], j - e[1], k - e[2]) + S(nv, g, i + d[0] - e[0], j + d[1] - e[1], k + d[2] - e[2]);
#define PH(a, b, c) S(phi, g, a, b, c)
  const double a0 = PH(i, j, k), a1 = PH(i + d[0], j + d[1], k + d[2]);
  const double p0 = PH(i + e[0], j + e[1], k + e[2]), p1 = PH(i + d[0] + e[0], j + d[1] + e[1], k + d[2] + e[2]);
  const double m0 = PH(i - e[0], j - e[1], k - e[2]), m1 = PH(i + d[0] - e[0], j + d[1] - e[1], k + d[2] - e[2]);
#undef PH
  if ((x == m - 2 && !per) || np_ > 0.1) {
    if (nm_ < 0.1 && x != 1) return (a0 + a1 - m0 - m1) * 0.5;
    return 0.;
  } else if ((x == 1 && !per) || nm_ > 0.1) {
    if (np_ < 0.1) return (p0 + p1 - a0 - a1) * 0.5;
    return 0.;
  }
  return (p0 + p1 - m0 - m1) * 0.25;
}

void og_projection(const og_grid *g, const og_metrics *M, const double *nv, const double *phi, double *ucont) {
  const int mx = g->mx, my = g->my, mz = g->mz;
  const int X1[3] = {1, 0, 0}, Y1[3] = {0, 1, 0}, Z1[3] = {0, 0, 1};
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        if (i < mx - 2 || (g->iper && i == mx - 2)) {
          double dpdc = S(phi, g, i + 1, j, k) - S(phi, g, i, j, k);
          if (i == mx - 2 && g->iper) dpdc = S(phi, g, 1, j, k) - S(phi, g, i, j, k);
          double dpde = cross_phi(g, phi, nv, i, j, k, X1, Y1, j, my, g->jper);
          double dpdz = cross_phi(g, phi, nv, i, j, k, X1, Z1, k, mz, g->kper);
          if (S(nv, g, i, j, k) + S(nv, g, i + 1, j, k) < 0.1) {
            const double *c = &V(M->icsi, g, i, j, k, 0), *e = &V(M->ieta, g, i, j, k, 0), *z = &V(M->izet, g, i, j, k, 0);
            const double a = S(M->iaj, g, i, j, k);
            V(ucont, g, i, j, k, 0) -= (dpdc * (c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) * a +
                                        dpde * (e[0] * c[0] + e[1] * c[1] + e[2] * c[2]) * a +
                                        dpdz * (z[0] * c[0] + z[1] * c[1] + z[2] * c[2]) * a) * g->dt * g->st / 1.0 / 1.0;
          }
        }
        if (j < my - 2 || (g->jper && j == my - 2)) {
          double dpdc = cross_phi(g, phi, nv, i, j, k, Y1, X1, i, mx, g->iper);
          double dpde = (j == my - 2 && g->jper) ? S(phi, g, i, 1, k) - S(phi, g, i, j, k) : S(phi, g, i, j + 1, k) - S(phi, g, i, j, k);
          double dpdz = cross_phi(g, phi, nv, i, j, k, Y1, Z1, k, mz, g->kper);
          const double s2 = S(nv, g, i, j, k) + S(nv, g, i, j + 1, k);
          if (s2 < 0.1 || (int)s2 == 5) {
            const double *c = &V(M->jcsi, g, i, j, k, 0), *e = &V(M->jeta, g, i, j, k, 0), *z = &V(M->jzet, g, i, j, k, 0);
            const double a = S(M->jaj, g, i, j, k);
            V(ucont, g, i, j, k, 1) -= (dpdc * (c[0] * e[0] + c[1] * e[1] + c[2] * e[2]) * a +
                                        dpde * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) * a +
                                        dpdz * (z[0] * e[0] + z[1] * e[1] + z[2] * e[2]) * a) * g->dt * g->st / 1.0 / 1.0;
          }
        }
        if (k < mz - 2 || (g->kper && k == mz - 2)) {
          double dpdc = cross_phi(g, phi, nv, i, j, k, Z1, X1, i, mx, g->iper);
          double dpde = cross_phi(g, phi, nv, i, j, k, Z1, Y1, j, my, g->jper);
          double dpdz = (k == mz - 2 && g->kper) ? S(phi, g, i, j, 1) - S(phi, g, i, j, k) : S(phi, g, i, j, k + 1) - S(phi, g, i, j, k);
          if (S(nv, g, i, j, k) + S(nv, g, i, j, k + 1) < 0.1) {
            const double *c = &V(M->kcsi, g, i, j, k, 0), *e = &V(M->keta, g, i, j, k, 0), *z = &V(M->kzet, g, i, j, k, 0);
            const double a = S(M->kaj, g, i, j, k);
            V(ucont, g, i, j, k, 2) -= (dpdc * (c[0] * z[0] + c[1] * z[1] + c[2] * z[2]) * a +
                                        dpde * (e[0] * z[0] + e[1] * z[1] + e[2] * z[2]) * a +
                                        dpdz * (z[0] * z[0] + z[1] * z[1] + z[2] * z[2]) * a) * g->dt * g->st / 1.0 / 1.0;
          }
        }
      }
  /* component-wise periodic copy (poisson.c:3013-3046) */
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        int a = wrap(g->iper, mx, i), b = wrap(g->jper, my, j), c = wrap(g->kper, mz, k);
        if (a != i) V(ucont, g, i, j, k, 0) = V(ucont, g, a, b, c, 0);
        if (b != j) V(ucont, g, i, j, k, 1) = V(ucont, g, a, b, c, 1);
        if (c != k) V(ucont, g, i, j, k, 2) = V(ucont, g, a, b, c, 2);
      }
}

double og_divergence(const og_grid *g, const double *ucont, const double *aj, const double *nv) {
  double mx_ = 0;
  for (int k = 1; k < g->mz - 1; k++)
    for (int j = 1; j < g->my - 1; j++)
      for (int i = 1; i < g->mx - 1; i++) {
        double d = fabs((V(ucont, g, i, j, k, 0) - V(ucont, g, i - 1, j, k, 0) + V(ucont, g, i, j, k, 1) -
                         V(ucont, g, i, j - 1, k, 1) + V(ucont, g, i, j, k, 2) - V(ucont, g, i, j, k - 1, 2)) *
                        S(aj, g, i, j, k));
        if (S(nv, g, i, j, k) + S(nv, g, i, j, k + 1) + S(nv, g, i, j, k - 1) + S(nv, g, i, j + 1, k) +
                S(nv, g, i, j - 1, k) + S(nv, g, i + 1, j, k) + S(nv, g, i - 1, j, k) > 0.1)
          d = 0.;
        if (d > mx_) mx_ = d;
      }
  return mx_;
}

/* ------------------------------------------------------------------ dynamic Smagorinsky
 * Compute_Smagorinsky_Constant_1 (les.c:67-1133) with testfilter_ik = 0, clark = 0 and no
 * homogeneous-direction averaging, then Compute_eddy_viscosity_LES (les.c:1135-1252).
 * ucat: the Contra2Cart output with its ghost values; cs and nut are updated in place
 * (nut keeps its values on non-periodic ghost points, as lNu_t does). */
static void les_du_center(const og_grid *g, const double *u, const double *nv, int i, int j, int k, double d[9]) {
  /* Compute_du_center, k-omega.c:305-420 (note k == 0 in the lower k test, k-omega.c:395) */
  int a0[3], b0[3];
  double f;
  for (int c = 0; c < 3; c++) {
    int ia = i, ib = i, ja = j, jb = j, ka = k, kb = k;
    if (c == 0) {
      if (S(nv, g, i + 1, j, k) > 0.1 || (!g->iper && i == g->mx - 2)) { ib = i - 1; f = 1; }
      else if (S(nv, g, i - 1, j, k) > 0.1 || (!g->iper && i == 1)) { ia = i + 1; f = 1; }
      else { ia = i + 1; ib = i - 1; f = 0.5; }
    } else if (c == 1) {
      if (S(nv, g, i, j + 1, k) > 0.1 || (!g->jper && j == g->my - 2)) { jb = j - 1; f = 1; }
      else if (S(nv, g, i, j - 1, k) > 0.1 || (!g->jper && j == 1)) { ja = j + 1; f = 1; }
      else { ja = j + 1; jb = j - 1; f = 0.5; }
    } else {
      if (S(nv, g, i, j, k + 1) > 0.1 || (!g->kper && k == g->mz - 2)) { kb = k - 1; f = 1; }
      else if (S(nv, g, i, j, k - 1) > 0.1 || (!g->kper && k == 0)) { ka = k + 1; f = 1; }
      else { ka = k + 1; kb = k - 1; f = 0.5; }
    }
    for (int v = 0; v < 3; v++) {
      double diff = V(u, g, ia, ja, ka, v) - V(u, g, ib, jb, kb, v);
      d[3 * c + v] = (f == 1) ? diff : diff * 0.5;
    }
    (void)a0; (void)b0;
  }
}

static void les_grad(const double *c, const double *e, const double *z, double ajc, const double d[9], double o[9]) {
  /* Compute_du_dxyz, k-omega.c:597-610; o = du/dx du/dy du/dz dv/dx ... dw/dz */
  for (int v = 0; v < 3; v++)
    for (int x = 0; x < 3; x++) o[3 * v + x] = (d[v] * c[x] + d[3 + v] * e[x] + d[6 + v] * z[x]) * ajc;
}

static double les_strain(const double o[9], double s[3][3]) {
  s[0][0] = 0.5 * (o[0] + o[0]); s[0][1] = 0.5 * (o[1] + o[3]); s[0][2] = 0.5 * (o[2] + o[6]);
  s[1][0] = s[0][1]; s[1][1] = 0.5 * (o[4] + o[4]); s[1][2] = 0.5 * (o[5] + o[7]);
  s[2][0] = s[0][2]; s[2][1] = s[1][2]; s[2][2] = 0.5 * (o[8] + o[8]);
  return sqrt(2.0 * (s[0][0] * s[0][0] + s[0][1] * s[0][1] + s[0][2] * s[0][2] + s[1][0] * s[1][0] +
                     s[1][1] * s[1][1] + s[1][2] * s[1][2] + s[2][0] * s[2][0] + s[2][1] * s[2][1] +
                     s[2][2] * s[2][2]));
}

/* integrate_testfilter (rhs2.c:412-455), val/w indexed [R][Q][P] = [k][j][i] offsets + 1 */
static double les_filter(double val[3][3][3], double w[3][3][3]) {
  double vt = 0, wt = 0;
  for (int s = 0; s < 8; s++) {
    const int R0 = s & 1, P0 = (s >> 1) & 1, Q0 = (s >> 2) & 1;
    double vs = 0, ws = 0;
    for (int m = 0; m < 8; m++) {
      const int R = R0 + (m & 1), P = P0 + ((m >> 1) & 1), Q = Q0 + ((m >> 2) & 1);
      vs = m ? vs + val[R][Q][P] * w[R][Q][P] : val[R][Q][P] * w[R][Q][P];
      ws = m ? ws + w[R][Q][P] : w[R][Q][P];
    }
    vt = s ? vt + vs : vs;
    wt = s ? wt + ws : ws;
  }
  return vt / wt;
}

static void les_inverse(const double a[3][3], double G[3][3]) {
  /* Calculate_Covariant_metrics, rhs2.c:538-554 */
  const double a11 = a[0][0], a12 = a[0][1], a13 = a[0][2], a21 = a[1][0], a22 = a[1][1], a23 = a[1][2];
  const double a31 = a[2][0], a32 = a[2][1], a33 = a[2][2];
  const double det = a11 * (a33 * a22 - a32 * a23) - a21 * (a33 * a12 - a32 * a13) + a31 * (a23 * a12 - a22 * a13);
  G[0][0] = (a33 * a22 - a32 * a23) / det; G[0][1] = -(a33 * a12 - a32 * a13) / det; G[0][2] = (a23 * a12 - a22 * a13) / det;
  G[1][0] = -(a33 * a21 - a31 * a23) / det; G[1][1] = (a33 * a11 - a31 * a13) / det; G[1][2] = -(a23 * a11 - a21 * a13) / det;
  G[2][0] = (a32 * a21 - a31 * a22) / det; G[2][1] = -(a32 * a11 - a31 * a12) / det; G[2][2] = (a22 * a11 - a21 * a12) / det;
}

/* weights of the LM/MM averaging and of the Cs re-filter (les.c:720-762, 1069-1110) */
static void les_wrap_weights(const og_grid *g, const double *aj, const double *nv, int i, int j, int k,
                             double w[3][3][3], int src[3][3][3]) {
  for (int a = -1; a <= 1; a++)
    for (int b = -1; b <= 1; b++)
      for (int c = -1; c <= 1; c++) {
        int I = i + a, J = j + b, K = k + c;
        double wt = 1. / S(aj, g, I, J, K);
        if (S(nv, g, I, J, K) > 1.1) wt = 0;
        if (g->iper) { if (I == 0) I = g->mx - 2; else if (I == g->mx - 1) I = 1; }
        else if (I == 0 || I == g->mx - 1) wt = 0;
        if (g->jper) { if (J == 0) J = g->my - 2; else if (J == g->my - 1) J = 1; }
        else if (J == 0 || j == g->my - 1) wt = 0;
        if (g->kper) { if (K == 0) K = g->mz - 2; else if (K == g->mz - 1) K = 1; }
        else if (K == 0 || K == g->mz - 1) wt = 0;
        w[c + 1][b + 1][a + 1] = wt;
        src[c + 1][b + 1][a + 1] = (int)IX(g, I, J, K);
      }
}

void og_les(const og_grid *g, const double *ucat, const double *csi, const double *eta, const double *zet,
            const double *aj, const double *nv, int ti, int tistart, int rstart, double max_cs, double *cs,
            double *nut) {
  const size_t N = (size_t)g->mx * g->my * g->mz;
  const int mx = g->mx, my = g->my, mz = g->mz;
  if (ti < 2 && tistart == 0 && !rstart) {
    memset(cs, 0, 8 * N);
  } else if (g->les == 1) {
    for (size_t p = 0; p < N; p++) cs[p] = 0.01;
  } else {
    double *A = calloc(9 * N, 8), *Sa = calloc(N, 8), *uf = calloc(3 * N, 8), *LM = calloc(N, 8), *MM = calloc(N, 8);
    double *tmp = calloc(N, 8);
    /* les.c:191-238 */
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          if (S(nv, g, i, j, k) > 1.1) continue;
          const size_t p = IX(g, i, j, k);
          double d[9], o[9], s[3][3];
          les_du_center(g, ucat, nv, i, j, k, d);
          les_grad(csi + 3 * p, eta + 3 * p, zet + 3 * p, aj[p], d, o);
          Sa[p] = les_strain(o, s);
          for (int q = 0; q < 9; q++) A[9 * p + q] = o[q];
          double w[3][3][3], u[3][3][3][3];
          for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++)
              for (int c = -1; c <= 1; c++) {
                const size_t q = IX(g, i + a, j + b, k + c);
                w[c + 1][b + 1][a + 1] = nv[q] > 1.1 ? 0 : 1. / aj[q];
                for (int v = 0; v < 3; v++) u[v][c + 1][b + 1][a + 1] = ucat[3 * q + v];
              }
          for (int v = 0; v < 3; v++) uf[3 * p + v] = les_filter(u[v], w);
        }
    og_periodic_copy(g, A, 9); og_periodic_copy(g, Sa, 1); og_periodic_copy(g, uf, 3);
    /* les.c:300-661 */
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          const size_t p = IX(g, i, j, k);
          if (nv[p] > 1.1) { LM[p] = MM[p] = 0; continue; }
          double w[3][3][3], L[9][3][3][3], SS[3][3][3][3][3];
          for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++)
              for (int c = -1; c <= 1; c++) {
                const size_t q = IX(g, i + a, j + b, k + c);
                const int R = c + 1, Q = b + 1, P = a + 1;
                w[R][Q][P] = nv[q] > 1.1 ? 0 : 1. / aj[q];
                const double *u3 = ucat + 3 * q;
                double UVW[3];
                const double *mt[3] = {csi + 3 * q, eta + 3 * q, zet + 3 * q};
                for (int x = 0; x < 3; x++) UVW[x] = u3[0] * mt[x][0] + u3[1] * mt[x][1] + u3[2] * mt[x][2];
                for (int x = 0; x < 3; x++)
                  for (int y = 0; y < 3; y++) L[3 * x + y][R][Q][P] = UVW[x] * u3[y];
                double s[3][3];
                les_strain(A + 9 * q, s);
                for (int x = 0; x < 3; x++)
                  for (int y = 0; y < 3; y++) SS[x][y][R][Q][P] = s[x][y] * Sa[q];
              }
          double sum_weight = 0;
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              for (int c = 0; c < 3; c++)
                sum_weight += w[c][b][a] * ((c == 1 ? 1.0 : 0.5) * (b == 1 ? 1.0 : 0.5) * (a == 1 ? 1.0 : 0.5));
          const double filter = pow(1. / aj[p], 1. / 3.), test_filter = pow(sum_weight, 1. / 3.);
          const double *c0 = csi + 3 * p, *e0 = eta + 3 * p, *z0 = zet + 3 * p;
          const double *f = uf + 3 * p;
          const double fU[3] = {f[0] * c0[0] + f[1] * c0[1] + f[2] * c0[2], f[0] * e0[0] + f[1] * e0[1] + f[2] * e0[2],
                                f[0] * z0[0] + f[1] * z0[1] + f[2] * z0[2]};
          double d[9], o[9], Sh[3][3];
          les_du_center(g, uf, nv, i, j, k, d);
          les_grad(c0, e0, z0, aj[p], d, o);
          const double S_hat = les_strain(o, Sh);
          double Lij[3][3], SSh[3][3], Mc[3][3], M[3][3], gg[3][3], ggc[3][3], G[3][3];
          for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++) {
              Lij[x][y] = les_filter(L[3 * x + y], w) - fU[x] * f[y];
              SSh[x][y] = les_filter(SS[x][y], w);
            }
          for (int x = 0; x < 3; x++) { gg[0][x] = c0[x]; gg[1][x] = e0[x]; gg[2][x] = z0[x]; }
          les_inverse(gg, ggc);
          for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++)
              G[x][y] = ggc[0][x] * ggc[0][y] + ggc[1][x] * ggc[1][y] + ggc[2][x] * ggc[2][y];
          /* les.c:612-614 form the off-diagonal entries with the second index first */
          G[0][1] = G[1][0] = ggc[0][1] * ggc[0][0] + ggc[1][1] * ggc[1][0] + ggc[2][1] * ggc[2][0];
          G[0][2] = G[2][0] = ggc[0][2] * ggc[0][0] + ggc[1][2] * ggc[1][0] + ggc[2][2] * ggc[2][0];
          G[1][2] = G[2][1] = ggc[0][1] * ggc[0][2] + ggc[1][1] * ggc[1][2] + ggc[2][1] * ggc[2][2];
          for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++)
              Mc[x][y] = -pow(test_filter, 2.) * S_hat * Sh[x][y] + pow(filter, 2.) * SSh[x][y];
          for (int x = 0; x < 3; x++) {
            M[x][0] = Mc[x][0] * c0[0] + Mc[x][1] * c0[1] + Mc[x][2] * c0[2];
            M[x][1] = Mc[x][0] * e0[0] + Mc[x][1] * e0[1] + Mc[x][2] * e0[2];
            M[x][2] = Mc[x][0] * z0[0] + Mc[x][1] * z0[1] + Mc[x][2] * z0[2];
          }
          double num = 0, den = 0;
          for (int q = 0; q < 3; q++)
            for (int a = 0; a < 3; a++)
              for (int b = 0; b < 3; b++) num += Lij[b][a] * M[a][q] * G[b][q];
          for (int m = 0; m < 3; m++)
            for (int n = 0; n < 3; n++)
              for (int l = 0; l < 3; l++) den += M[n][m] * M[n][l] * G[m][l];
          LM[p] = num;
          MM[p] = den;
        }
    og_periodic_copy(g, LM, 1); og_periodic_copy(g, MM, 1);
    /* les.c:708-788 */
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          const size_t p = IX(g, i, j, k);
          if (nv[p] > 1.1) { cs[p] = 0; continue; }
          double w[3][3][3], l0[3][3][3], m0[3][3][3];
          int src[3][3][3];
          les_wrap_weights(g, aj, nv, i, j, k, w, src);
          for (int R = 0; R < 3; R++)
            for (int Q = 0; Q < 3; Q++)
              for (int P = 0; P < 3; P++) { l0[R][Q][P] = LM[src[R][Q][P]]; m0[R][Q][P] = MM[src[R][Q][P]]; }
          const double C = 0.5 * les_filter(l0, w) / (les_filter(m0, w) + 1.e-4);
          cs[p] = C < 0 ? 0 : C;
        }
    /* les.c:959-972, then the periodic copy of les.c:1022-1048 */
    for (int k = 0; k < mz; k++)
      for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) {
          const size_t p = IX(g, i, j, k);
          if (nv[p] > 1.1 || k == 0 || k == mz - 1 || j == 0 || j == my - 1 || i == 0 || i == mx - 1) { cs[p] = 0; continue; }
          if (nv[p] > 0.1 && nv[p] < 1.1) cs[p] = 0.001 < cs[p] ? cs[p] : 0.001;
          double v = cs[p] < 0 ? 0 : cs[p];
          cs[p] = v < max_cs ? v : max_cs;
        }
    og_periodic_copy(g, cs, 1);
    /* les.c:1051-1120 */
    memcpy(tmp, cs, 8 * N);
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          const size_t p = IX(g, i, j, k);
          if (!(nv[p] < 0.1)) continue;
          double w[3][3][3], c0[3][3][3];
          int src[3][3][3];
          les_wrap_weights(g, aj, nv, i, j, k, w, src);
          for (int R = 0; R < 3; R++)
            for (int Q = 0; Q < 3; Q++)
              for (int P = 0; P < 3; P++) c0[R][Q][P] = tmp[src[R][Q][P]];
          cs[p] = les_filter(c0, w);
        }
    free(A); free(Sa); free(uf); free(LM); free(MM); free(tmp);
  }
  /* Compute_eddy_viscosity_LES, les.c:1174-1243 */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const size_t p = IX(g, i, j, k);
        if (nv[p] > 1.1) { nut[p] = 0; continue; }
        double d[9], o[9], s[3][3];
        les_du_center(g, ucat, nv, i, j, k, d);
        les_grad(csi + 3 * p, eta + 3 * p, zet + 3 * p, aj[p], d, o);
        const double Sabs = les_strain(o, s);
        const double filter = pow(1. / aj[p], 1. / 3.);
        nut[p] = cs[p] * pow(filter, 2.0) * Sabs;
      }
  og_periodic_copy(g, nut, 1);
}
