// Hand-written transposes of the cell-to-face and face-to-cell stencils of the projection
// step: Pressure_Gradient (momentum.c:197-443, without its flux forcing), the local Poisson
// right-hand side (poisson_hypre.c PoissonRHS2_hypre, the divergence part), UpdatePressure
// (poisson.c:3144-3305), Projection (poisson.c:2780-3046) and the periodic ghost copies
// they run.  Each is a gather: a thread owns one output point and sums, over the faces (or
// cells) whose forward stencil reads that point, the forward coefficient times the adjoint
// of the face (or cell).  No atomics, so the result does not depend on thread scheduling;
// the coefficients are the forward kernels' own branch for branch (nvert-aware one-sided
// cross differences, the periodic wrap of the main difference, the masked faces).
#include "vfs_internal.cuh"

namespace vfs {

namespace {

struct Box {
  int m[3];
  int per[3];
  long long s[3];
};

__device__ __forceinline__ Box box_of(const Grid &g) {
  Box b;
  b.m[0] = g.mx; b.m[1] = g.my; b.m[2] = g.mz;
  b.per[0] = g.iper; b.per[1] = g.jper; b.per[2] = g.kper;
  b.s[0] = 1; b.s[1] = g.mx; b.s[2] = (long long)g.mx * g.my;
  return b;
}

__device__ __forceinline__ bool interior(const Box &b, const int x[3]) {
  return x[0] >= 1 && x[0] <= b.m[0] - 2 && x[1] >= 1 && x[1] <= b.m[1] - 2 && x[2] >= 1 && x[2] <= b.m[2] - 2;
}

// Face (direction d, lower cell f) carries a value in the forward kernel.
// Pressure_Gradient: both cells nvert 0 and the face not on a non-periodic far wall.
// Projection: the face inside the loop bounds (i < mx-2, or the periodic wrap face) and
// nvert(f) + nvert(f+d) == 0, or == 5 on j-faces (poisson.c:2890).
template <int V>
__device__ __forceinline__ bool face_active(const Box &b, const uint8_t *__restrict__ nv, int d, long long f,
                                            const int x[3]) {
  if (!interior(b, x)) return false;
  const int s = nv[f] + nv[f + b.s[d]];
  if (V == 0) return s == 0 && (b.per[d] || x[d] < b.m[d] - 2);
  if (!(x[d] < b.m[d] - 2 || (b.per[d] && x[d] == b.m[d] - 2))) return false;
  return d == 1 ? (s == 0 || s == 5) : s == 0;
}

// Which form the cross difference along t of face (d, f) takes: 0 one-sided towards the
// minus side (cells f, f+d and their t-1 neighbours), 1 one-sided towards the plus side,
// 2 central, 3 none (Projection's zero when both sides are blocked).
template <int V>
__device__ __forceinline__ int cross_form(const Box &b, const uint8_t *__restrict__ nv, int d, int t, long long f,
                                          const int x[3]) {
  const long long pp0 = f + b.s[t], pp1 = f + b.s[t] + b.s[d];
  const long long pm0 = f - b.s[t], pm1 = f - b.s[t] + b.s[d];
  const int e = x[t], em = b.m[t], eper = b.per[t];
  if (V == 0) {  // IB nodes (nvert == 1) and non-periodic walls block a side
    if (nv[pp0] == 1 || nv[pp1] == 1 || (e == em - 2 && !eper)) return 0;
    if (nv[pm0] == 1 || nv[pm1] == 1 || (e == 1 && !eper)) return 1;
    return 2;
  }
  const int nplus = nv[pp0] + nv[pp1], nminus = nv[pm0] + nv[pm1];
  if ((e == em - 2 && !eper) || nplus > 0) return (nminus == 0 && e != 1) ? 0 : 3;
  if ((e == 1 && !eper) || nminus > 0) return nplus == 0 ? 1 : 3;
  return 2;
}

// Coefficient of the cell at cross offset o (-1, 0, +1) in a cross difference of form f;
// the two cells of the face (offsets 0 and +1 along d) share it.
__device__ __forceinline__ double cross_w(int form, int o) {
  switch (form) {
    case 0: return o == 0 ? 0.5 : (o == -1 ? -0.5 : 0.0);
    case 1: return o == 1 ? 0.5 : (o == 0 ? -0.5 : 0.0);
    case 2: return o == 1 ? 0.25 : (o == -1 ? -0.25 : 0.0);
    default: return 0.0;
  }
}

// lc[c] += scale * sum over faces (d, f) and derivative directions t of
// coefficient(f, t, c) * G[3d+t][f] * aj_d[f] * lf_d[f]: the transpose of
// out_d[f] = aj_d[f] * sum_t G[3d+t][f] * D_t(c)[f] at the active faces.
template <int V>
__global__ void __launch_bounds__(256) k_face_grad_adjoint(Grid g, const double *__restrict__ G,
                                                           const double *__restrict__ iaj,
                                                           const double *__restrict__ jaj,
                                                           const double *__restrict__ kaj,
                                                           const uint8_t *__restrict__ nv, CV3 lf, double scale,
                                                           double *lc) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const Box b = box_of(g);
  int c[3];
  dijk(g, p, c[0], c[1], c[2]);
  const long long N = g.N;
  double acc = 0;
#pragma unroll 1
  for (int d = 0; d < 3; d++) {
    const double *aj = d == 0 ? iaj : (d == 1 ? jaj : kaj);
    const double *l = d == 0 ? lf.x : (d == 1 ? lf.y : lf.z);
    auto term = [&](long long f, int t) { return G[(long long)(3 * d + t) * N + f] * aj[f] * l[f]; };
    // main difference c(f+d) - c(f), or c(1) - c(f) on the periodic wrap face f = m-2
    if (face_active<V>(b, nv, d, p, c)) acc -= term(p, d);
    {
      int x[3] = {c[0], c[1], c[2]};
      x[d] -= 1;
      const bool wrap_face = b.per[d] && x[d] == b.m[d] - 2;
      if (x[d] >= 1 && !wrap_face && face_active<V>(b, nv, d, p - b.s[d], x)) acc += term(p - b.s[d], d);
    }
    if (b.per[d] && c[d] == 1) {
      int x[3] = {c[0], c[1], c[2]};
      x[d] = b.m[d] - 2;
      const long long f = p + (long long)(b.m[d] - 3) * b.s[d];
      if (face_active<V>(b, nv, d, f, x)) acc += term(f, d);
    }
    // cross differences along t: faces f = c - a e_d - o e_t, a in {0, 1}, o in {-1, 0, 1}
#pragma unroll 1
    for (int t = 0; t < 3; t++) {
      if (t == d) continue;
#pragma unroll 1
      for (int a = 0; a < 2; a++) {
#pragma unroll 1
        for (int o = -1; o <= 1; o++) {
          int x[3] = {c[0], c[1], c[2]};
          x[d] -= a;
          x[t] -= o;
          const long long f = p - a * b.s[d] - o * b.s[t];
          if (!face_active<V>(b, nv, d, f, x)) continue;
          const double w = cross_w(cross_form<V>(b, nv, d, t, f, x), o);
          if (w != 0.0) acc += w * term(f, t);
        }
      }
    }
  }
  lc[p] += scale * acc;
}

// Periodic images of coordinate v: itself, then the ghost that copies it (0 <- m-2,
// m-1 <- 1) in a periodic direction.
__device__ __forceinline__ int images(int v, int m, int per, int *o) {
  int n = 0;
  o[n++] = v;
  if (per) {
    if (v == m - 2) o[n++] = 0;
    if (v == 1) o[n++] = m - 1;
  }
  return n;
}

__device__ __forceinline__ bool pghost(int v, int m, int per) { return per && (v == 0 || v == m - 1); }

// Transpose of the periodic copy (k_periodic_copy: every point with a periodic ghost
// coordinate takes the value at its image wrapped in all three directions): each point
// with no periodic ghost coordinate adds the adjoints of the ghosts that copy it.
// comp < 0: the ghosts of any periodic direction (the scalar and 3-component copies, for
// each of a[0..na-1]); comp = 3: component q of a 3-component field copies only across
// direction q (k_periodic_copy_comp).  The ghosts are cleared by k_pcopy_clear afterwards.
struct Arrays3 { double *a[3]; };

__global__ void k_pcopy_gather(Grid g, int comp, int na, Arrays3 a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const Box b = box_of(g);
  int c[3];
  dijk(g, p, c[0], c[1], c[2]);
  if (pghost(c[0], b.m[0], b.per[0]) || pghost(c[1], b.m[1], b.per[1]) || pghost(c[2], b.m[2], b.per[2])) return;
  int oi[3], oj[3], ok[3];
  const int ni = images(c[0], b.m[0], b.per[0], oi), nj = images(c[1], b.m[1], b.per[1], oj),
            nk = images(c[2], b.m[2], b.per[2], ok);
  if (ni == 1 && nj == 1 && nk == 1) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int zk = 0; zk < nk; zk++)
    for (int yj = 0; yj < nj; yj++)
      for (int xi = 0; xi < ni; xi++) {
        if (xi == 0 && yj == 0 && zk == 0) continue;
        const long long q = lidx(g, oi[xi], oj[yj], ok[zk]);
        for (int t = 0; t < na; t++) {
          // component t of a component-wise copy moves only across direction t
          if (comp == 3 && (t == 0 ? xi : (t == 1 ? yj : zk)) == 0) continue;
          acc[t] += a.a[t][q];
        }
      }
  for (int t = 0; t < na; t++)
    if (acc[t] != 0.0) a.a[t][p] += acc[t];
}

__global__ void k_pcopy_clear(Grid g, int comp, int na, Arrays3 a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int c[3];
  dijk(g, p, c[0], c[1], c[2]);
  const bool t3[3] = {pghost(c[0], g.mx, g.iper), pghost(c[1], g.my, g.jper), pghost(c[2], g.mz, g.kper)};
  const bool any = t3[0] || t3[1] || t3[2];
  for (int t = 0; t < na; t++)
    if (comp == 3 ? t3[t] : any) a.a[t][p] = 0.0;
}

// UpdatePressure's transpose: P += Phi on interior fluid cells, P = 0 on interior cells
// with nvert >= 2.
__global__ void k_update_pressure_adjoint(Grid g, const uint8_t *__restrict__ nv, double *lP, double *lphi) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  if (nv[p] == 0) lphi[p] += lP[p];
  if (nv[p] >= 2) lP[p] = 0;
}

// Transpose of b[c] = s * (-u_d[c] + u_d[c - d]) summed over d on the fluid cells (the
// periodic wrap reads u_d at m-2 for c = 1): each face adds s times the adjoints of the
// cells whose divergence reads it.
__global__ void k_poisson_rhs_adjoint(Grid g, const uint8_t *__restrict__ fluid, const double *__restrict__ lb,
                                      double s, V3 lu) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const Box b = box_of(g);
  int c[3];
  dijk(g, p, c[0], c[1], c[2]);
#pragma unroll 1
  for (int d = 0; d < 3; d++) {
    double acc = fluid[p] ? -lb[p] : 0.0;
    if (c[d] + 1 <= b.m[d] - 1) {
      const long long q = p + b.s[d];
      if (fluid[q] && !(b.per[d] && c[d] + 1 == 1)) acc += lb[q];
    }
    if (b.per[d] && c[d] == b.m[d] - 2) {
      const long long q = p - (long long)(b.m[d] - 3) * b.s[d];  // the cell at coordinate 1
      if (fluid[q]) acc += lb[q];
    }
    double *u = d == 0 ? lu.x : (d == 1 ? lu.y : lu.z);
    if (acc != 0.0) u[p] += s * acc;
  }
}

}  // namespace

static bool any_periodic(const Grid &g) { return g.iper || g.jper || g.kper; }

// In place: the transpose of the periodic copy of na arrays (comp -1) or of the
// component-wise copy of a 3-component field (comp 3).
static int pcopy_adjoint(Ctx *c, int comp, int na, Arrays3 a) {
  int rc;
  const Grid &g = c->g;
  if (!any_periodic(g)) return VFS_OK;
  c->launches++, k_pcopy_gather<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, comp, na, a);
  if ((rc = check_launch(c, "k_pcopy_gather"))) return rc;
  c->launches++, k_pcopy_clear<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, comp, na, a);
  return check_launch(c, "k_pcopy_clear");
}

int periodic_copy1_adjoint(Ctx *c, double *a) { return pcopy_adjoint(c, -1, 1, Arrays3{{a, nullptr, nullptr}}); }

int periodic_copy3_adjoint(Ctx *c, V3 a) { return pcopy_adjoint(c, -1, 3, Arrays3{{a.x, a.y, a.z}}); }

// Pressure_Gradient (no forcing term), slots (P, dP) -> (P', dP'), P' = C P, dP' = S P':
// lP <- C^T (lP + S^T ldP), ldP <- 0.
int pressure_gradient_adjoint(Ctx *c, double *lP, V3 ldp) {
  int rc;
  const Grid &g = c->g;
  if ((rc = ensure_gab(c))) return rc;
  c->launches++, k_face_grad_adjoint<0><<<nblocks(g.N, 256), 256, 0, c->stream>>>(
      g, c->gab, c->f[VFS_IAJ][0], c->f[VFS_JAJ][0], c->f[VFS_KAJ][0], c->nv, cv(ldp), 1.0, lP);
  if ((rc = check_launch(c, "k_face_grad_adjoint"))) return rc;
  const size_t bytes = sizeof(double) * g.N;
  cudaMemsetAsync(ldp.x, 0, bytes, c->stream);
  cudaMemsetAsync(ldp.y, 0, bytes, c->stream);
  cudaMemsetAsync(ldp.z, 0, bytes, c->stream);
  return periodic_copy1_adjoint(c, lP);
}

// Projection's face update and its component-wise periodic copy, slots (Phi, Ucont):
// Ucont' = Cq (Ucont - dt st S Phi): lUcont <- Cq^T lUcont, lPhi -= dt st S^T lUcont.
// (Projection's closing Contra2Cart is transposed by the caller.)
int projection_adjoint(Ctx *c, double *lphi, V3 luc) {
  int rc;
  const Grid &g = c->g;
  if ((rc = ensure_gab(c))) return rc;
  if ((rc = pcopy_adjoint(c, 3, 3, Arrays3{{luc.x, luc.y, luc.z}}))) return rc;
  c->launches++, k_face_grad_adjoint<1><<<nblocks(g.N, 256), 256, 0, c->stream>>>(
      g, c->gab, c->f[VFS_IAJ][0], c->f[VFS_JAJ][0], c->f[VFS_KAJ][0], c->nv, cv(luc), -(g.dt * g.st), lphi);
  return check_launch(c, "k_face_grad_adjoint");
}

// UpdatePressure, slots (Phi, P): P' = C U(P, Phi), Phi' = C Phi.
int update_pressure_adjoint(Ctx *c, double *lP, double *lphi) {
  int rc;
  if ((rc = periodic_copy1_adjoint(c, lphi))) return rc;
  if ((rc = periodic_copy1_adjoint(c, lP))) return rc;
  c->launches++, k_update_pressure_adjoint<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, c->nv, lP, lphi);
  return check_launch(c, "k_update_pressure_adjoint");
}

// The local Poisson right-hand side, slots (Ucont, b): Ucont' = C Ucont, b' = D Ucont':
// lUcont <- C^T (lUcont + D^T lb), lb <- 0.
int poisson_rhs_local_adjoint(Ctx *c, V3 luc, double *lb) {
  int rc;
  const Grid &g = c->g;
  if (!c->ps.built) return set_err(c, VFS_ERR_STATE, "poisson_rhs_local_adjoint: Poisson operator not set up");
  const double s = -1.0 / g.dt * g.st;
  c->launches++, k_poisson_rhs_adjoint<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->ps.fluid, lb, s, luc);
  if ((rc = check_launch(c, "k_poisson_rhs_adjoint"))) return rc;
  cudaMemsetAsync(lb, 0, sizeof(double) * g.N, c->stream);
  return periodic_copy3_adjoint(c, luc);
}

}  // namespace vfs
