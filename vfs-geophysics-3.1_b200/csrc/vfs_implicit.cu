// Implicit momentum solve (implicit = 4, solvers.c:1282-1289): the step forms RHS_o =
// Formfunction_2 of its initial state, then Implicit_MatrixFree (implicitsolver.c:4196-4420)
// solves the Crank-Nicolson momentum equations F(Ucont) = 0 of FormFunction_SNES
// (momentum.c:2197-2300) for the new Ucont.
//
// The residual is the reference's: the same boundary faces forced to zero normal flux, the
// same Contra2Cart and IB_BC, the same vector updates in the same order around this
// library's Formfunction_2 (bit-identical to the reference's).  The reference hands F to
// PETSc's SNES (trust region, matrix-free Jacobian, unpreconditioned GMRES with
// Eisenstat-Walker forcing); here the nonlinear solve is Newton's method with the same
// kind of matrix-free Jacobian products, unpreconditioned GMRES(30) to a forcing term of
// 0.1 and a backtracking line search on |F|, driven from the host with every vector
// operation on the device.  Its iterates are not PETSc's; the solution satisfies the same
// equations to the same relative tolerance |F| <= imp_tol |F0|.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "vfs_internal.cuh"

namespace vfs {

namespace {

constexpr int kImpRestart = 30;     // GMRES restart length
constexpr int kImpCycles = 20;      // GMRES restart cycles per Newton iteration
constexpr int kImpNewton = 50;      // Newton iterations (SNESSetTolerances maxit, implicitsolver.c)
constexpr int kImpLineSearch = 10;  // halvings of the Newton step
constexpr double kImpForcing = 0.1; // GMRES relative tolerance inside a Newton iteration
constexpr int kDotBlocks = 592;     // 4 x 148

// The wall faces FormFunction_SNES gives zero normal flux before it evaluates F
// (momentum.c:2225-2243): codes 1 on every face, 2 on j+, 12 on j- and j+, 10 on the
// faces away from the edges; a point on the upper ghost plane writes the face below it.
__global__ void k_snes_bc(Grid g, V3 uc) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sy = mx, sz = (long long)mx * my;
  const int *bc = g.bc;
  if (i == 0 && bc[0] == 1) uc.x[p] = 0;
  if (i == mx - 1 && bc[1] == 1) uc.x[p - 1] = 0;
  if (j == 0 && bc[2] == 1) uc.y[p] = 0;
  if (j == my - 1 && bc[3] == 1) uc.y[p - sy] = 0;
  if (k == 0 && bc[4] == 1) uc.z[p] = 0;
  if (k == mz - 1 && bc[5] == 1) uc.z[p - sz] = 0;
  if (j == my - 1 && bc[3] == 2) uc.y[p - sy] = 0;
  if (j == 0 && bc[2] == 12) uc.y[p] = 0;
  if (j == my - 1 && bc[3] == 12) uc.y[p - sy] = 0;
  const bool jk_in = j != 0 && j != my - 1 && k != 0 && k != mz - 1;
  const bool ik_in = i != 0 && i != mx - 1 && k != 0 && k != mz - 1;
  if (bc[0] == 10 && i == 0 && jk_in) uc.x[p] = 0;
  if (bc[1] == 10 && i == mx - 1 && jk_in) uc.x[p - 1] = 0;
  if (bc[2] == 10 && j == 0 && ik_in) uc.y[p] = 0;
  if (abs(bc[3]) == 10 && j == my - 1 && ik_in) uc.y[p - sy] = 0;
}

// F = 0 + (-1/dt) Ucont, then F = F + (1/dt) Ucont_o (the two VecAXPY of momentum.c:2263-2266).
__global__ void k_time_terms(long long n, double a, double b, CV3 uc, CV3 uo, V3 F) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  F.x[p] = 0.0 + a * uc.x[p]; F.x[p] = F.x[p] + b * uo.x[p];
  F.y[p] = 0.0 + a * uc.y[p]; F.y[p] = F.y[p] + b * uo.y[p];
  F.z[p] = 0.0 + a * uc.z[p]; F.z[p] = F.z[p] + b * uo.z[p];
}

// F = F + 0.5 RHS_o, then F = F + (-1) dP (momentum.c:2280-2283).
__global__ void k_old_and_dp(long long n, CV3 ro, CV3 dp, V3 F) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  F.x[p] = F.x[p] + 0.5 * ro.x[p]; F.x[p] = F.x[p] + -1 * dp.x[p];
  F.y[p] = F.y[p] + 0.5 * ro.y[p]; F.y[p] = F.y[p] + -1 * dp.y[p];
  F.z[p] = F.z[p] + 0.5 * ro.z[p]; F.z[p] = F.z[p] + -1 * dp.z[p];
}

// The fix-ups Implicit_MatrixFree applies to the solution (implicitsolver.c:4291-4370):
// zero normal flux on the faces of codes 1 and 10 (and 2 on j+), and on an outlet (4) the
// ghost Ucat copied from the last cell and the face flux taken from the average of the
// two, set to zero (with the velocity) when it flows back in.
__global__ void k_imp_post(Grid g, Metrics m, V3 uc, V3 ucat) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int mx = g.mx, my = g.my, mz = g.mz;
  const long long sy = mx, sz = (long long)mx * my;
  const int *bc = g.bc;
  auto wall = [](int b) { return b == 1 || b == -1 || b == -2 || b == 10; };
  if (wall(bc[0]) && i == 0) uc.x[p] = 0;
  if (wall(bc[1]) && i == mx - 2) uc.x[p] = 0;
  if (wall(bc[2]) && j == 0) uc.y[p] = 0;
  if ((wall(bc[3]) || bc[3] == 2) && j == my - 2) uc.y[p] = 0;
  if (wall(bc[4]) && k == 0) uc.z[p] = 0;
  if (wall(bc[5]) && k == mz - 2) uc.z[p] = 0;
  if ((bc[0] == -1 || bc[0] == -2) && i == 1) uc.x[p] = 0;
  if ((bc[1] == -1 || bc[1] == -2) && i == mx - 3) uc.x[p] = 0;
  if ((bc[2] == -1 || bc[2] == -2) && j == 1) uc.y[p] = 0;
  if ((bc[3] == -1 || bc[3] == -2) && j == my - 3) uc.y[p] = 0;
  if ((bc[4] == -1 || bc[4] == -2) && k == 1) uc.z[p] = 0;
  if ((bc[5] == -1 || bc[5] == -2) && k == mz - 3) uc.z[p] = 0;
  if (bc[3] == 4 && j == my - 2) {
    const long long q = p + sy;
    ucat.x[q] = ucat.x[p]; ucat.y[q] = ucat.y[p]; ucat.z[q] = ucat.z[p];
    uc.y[p] = 0.5 * (ucat.x[p] + ucat.x[q]) * m.eta.x[p] + 0.5 * (ucat.y[p] + ucat.y[q]) * m.eta.y[p] +
              0.5 * (ucat.z[p] + ucat.z[q]) * m.eta.z[p];
  }
  if (bc[5] == 4 && k == mz - 2) {
    const long long q = p + sz;
    ucat.x[q] = ucat.x[p]; ucat.y[q] = ucat.y[p]; ucat.z[q] = ucat.z[p];
    uc.z[p] = 0.5 * (ucat.x[p] + ucat.x[q]) * m.zet.x[p] + 0.5 * (ucat.y[p] + ucat.y[q]) * m.zet.y[p] +
              0.5 * (ucat.z[p] + ucat.z[q]) * m.zet.z[p];
    if (uc.z[p] < 0) {
      uc.z[p] = 0;
      ucat.x[p] = ucat.y[p] = ucat.z[p] = 0;
      ucat.x[q] = ucat.y[q] = ucat.z[q] = 0;
    }
  }
}

// z = a x + b y over n entries.
__global__ void k_lincomb(long long n, double a, const double *x, double b, const double *y,
                          double *z) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) z[p] = a * x[p] + b * y[p];
}

// Block partial sums of x.y (grid-stride, fixed order: the same bits on every run).
__global__ void __launch_bounds__(256) k_dot_parts(long long n, const double *__restrict__ x,
                                                   const double *__restrict__ y, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
    s += x[p] * y[p];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// The workspace: vectors of 3N doubles (the three components one after the other).
struct Work {
  long long n3;
  double *U, *F, *D, *UT, *FT, *W, *V;  // V: kImpRestart + 1 basis vectors
  double *vec(double *base, int q) const { return base + (size_t)q * n3; }
};

Work work(Ctx *c) {
  Work w;
  w.n3 = 3 * c->g.N;
  double *b = c->imp;
  w.U = b; w.F = b + w.n3; w.D = b + 2 * w.n3; w.UT = b + 3 * w.n3; w.FT = b + 4 * w.n3; w.W = b + 5 * w.n3;
  w.V = b + 6 * w.n3;
  return w;
}

int ensure_work(Ctx *c) {
  if (c->imp) return VFS_OK;
  const size_t n = (size_t)(6 + kImpRestart + 1) * 3 * (size_t)c->g.N;
  if (cudaMalloc(&c->imp, sizeof(double) * n) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "implicit momentum: workspace allocation failed");
  c->imp_m = kImpRestart;
  return VFS_OK;
}

void to_vec(Ctx *c, int field, double *v) {
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(v + (size_t)q * c->g.N, c->f[field][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
}
void from_vec(Ctx *c, int field, const double *v) {
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(c->f[field][q], v + (size_t)q * c->g.N, bytes, cudaMemcpyDeviceToDevice, c->stream);
}

int lincomb(Ctx *c, long long n, double a, const double *x, double b, const double *y, double *z) {
  c->launches++, k_lincomb<<<nblocks(n, 256), 256, 0, c->stream>>>(n, a, x, b, y, z);
  return check_launch(c, "k_lincomb");
}

int vdot(Ctx *c, long long n, const double *x, const double *y, double *out) {
  int rc;
  if ((rc = ensure_red(c, kDotBlocks + 64))) return rc;
  c->launches++, k_dot_parts<<<kDotBlocks, 256, 0, c->stream>>>(n, x, y, c->red);
  if ((rc = check_launch(c, "k_dot_parts"))) return rc;
  return reduce_sum(c, c->red, kDotBlocks, out);
}

int vnorm(Ctx *c, long long n, const double *x, double *out) {
  double s = 0;
  int rc = vdot(c, n, x, x, &s);
  *out = sqrt(s);
  return rc;
}

// F(U): U into Ucont, FormFunction_SNES, RHS out to F.
int residual_at(Ctx *c, const double *U, double *F) {
  int rc;
  from_vec(c, VFS_UCONT, U);
  if ((rc = implicit_residual(c))) return rc;
  to_vec(c, VFS_RHS, F);
  return VFS_OK;
}

// GMRES(m) for J d = -F with J v = (F(U + h v) - F(U)) / h, d from 0, to |J d + F| <=
// eta |F| (or the cycle cap).  h follows Walker and Pernice: sqrt(machine eps)
// * sqrt(1 + |U|) / |v|, with |v| = 1 for the basis vectors.
int newton_direction(Ctx *c, const Work &w, double fnorm, double unorm, double eta, int *kits) {
  int rc;
  const long long n3 = w.n3;
  const int m = kImpRestart;
  const double h = 1.4901161193847656e-08 * sqrt(1.0 + unorm);
  cudaMemsetAsync(w.D, 0, sizeof(double) * n3, c->stream);
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1), y(m);
  double beta = fnorm;
  const double target = eta * fnorm;
  for (int cycle = 0; cycle < kImpCycles; cycle++) {
    // r = -F - J d (J d only after the first cycle)
    if (cycle == 0) {
      if ((rc = lincomb(c, n3, -1.0 / beta, w.F, 0.0, w.F, w.vec(w.V, 0)))) return rc;
    } else {
      double dn = 0;
      if ((rc = vnorm(c, n3, w.D, &dn))) return rc;
      const double hd = 1.4901161193847656e-08 * sqrt(1.0 + unorm) / dn;
      if ((rc = lincomb(c, n3, 1.0, w.U, hd, w.D, w.UT))) return rc;
      if ((rc = residual_at(c, w.UT, w.FT))) return rc;
      if ((rc = lincomb(c, n3, 1.0 / hd, w.FT, -1.0 / hd, w.F, w.W))) return rc;   // J d
      if ((rc = lincomb(c, n3, -1.0, w.F, -1.0, w.W, w.W))) return rc;            // r
      if ((rc = vnorm(c, n3, w.W, &beta))) return rc;
      if (beta <= target) return VFS_OK;
      if ((rc = lincomb(c, n3, 1.0 / beta, w.W, 0.0, w.W, w.vec(w.V, 0)))) return rc;
    }
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int j = 0;
    bool done = false;
    for (; j < m; j++) {
      double *vj = w.vec(w.V, j), *vn = w.vec(w.V, j + 1);
      // w = J v_j
      if ((rc = lincomb(c, n3, 1.0, w.U, h, vj, w.UT))) return rc;
      if ((rc = residual_at(c, w.UT, w.FT))) return rc;
      if ((rc = lincomb(c, n3, 1.0 / h, w.FT, -1.0 / h, w.F, vn))) return rc;
      (*kits)++;
      // modified Gram-Schmidt, twice
      for (int pass = 0; pass < 2; pass++)
        for (int i = 0; i <= j; i++) {
          double hij = 0;
          if ((rc = vdot(c, n3, vn, w.vec(w.V, i), &hij))) return rc;
          H[(size_t)i * m + j] += hij;
          if ((rc = lincomb(c, n3, 1.0, vn, -hij, w.vec(w.V, i), vn))) return rc;
        }
      double hn = 0;
      if ((rc = vnorm(c, n3, vn, &hn))) return rc;
      H[(size_t)(j + 1) * m + j] = hn;
      if (hn > 0 && (rc = lincomb(c, n3, 1.0 / hn, vn, 0.0, vn, vn))) return rc;
      for (int i = 0; i < j; i++) {  // earlier rotations
        const double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
      }
      const double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
      const double r = sqrt(a * a + b * b);
      cs[j] = r > 0 ? a / r : 1.0;
      sn[j] = r > 0 ? b / r : 0.0;
      H[(size_t)j * m + j] = r;
      H[(size_t)(j + 1) * m + j] = 0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      if (fabs(gv[j + 1]) <= target || hn == 0) { j++; done = true; break; }
    }
    // d += V y, H y = g (upper triangular, j columns)
    for (int i = j - 1; i >= 0; i--) {
      double s = gv[i];
      for (int q = i + 1; q < j; q++) s -= H[(size_t)i * m + q] * y[q];
      y[i] = s / H[(size_t)i * m + i];
    }
    for (int i = 0; i < j; i++)
      if ((rc = lincomb(c, n3, 1.0, w.D, y[i], w.vec(w.V, i), w.D))) return rc;
    if (done) return VFS_OK;
  }
  return VFS_OK;
}

}  // namespace

// FormFunction_SNES (momentum.c:2197-2300) at the current Ucont into RHS.
int implicit_residual(Ctx *c) {
  const Grid &g = c->g;
  int rc;
  V3 uc = field3(c, VFS_UCONT), F = field3(c, VFS_RHS);
  c->launches++, k_snes_bc<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, uc);
  if ((rc = check_launch(c, "k_snes_bc"))) return rc;
  if ((rc = contra2cart(c))) return rc;   // Contra2Cart_2
  if ((rc = ib_bc(c))) return rc;
  c->launches++, k_time_terms<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g.N, -1. / g.dt, 1. / g.dt, cv(uc),
                                                                          cv(field3(c, VFS_UCONT_O)), F);
  if ((rc = check_launch(c, "k_time_terms"))) return rc;
  if ((rc = formfunction2(c, 0.5, false, 0.0))) return rc;
  c->launches++, k_old_and_dp<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g.N, cv(field3(c, VFS_RHS_O)),
                                                                          cv(field3(c, VFS_DP)), F);
  return check_launch(c, "k_old_and_dp");
}

// RHS_o = Formfunction_2 of the current state (VecSet(RHS_o, 0) and
// Formfunction_2(user, RHS_o, 1.0), solvers.c:1284-1286).
int implicit_rhs_o(Ctx *c) {
  int rc;
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  for (int q = 0; q < 3; q++) cudaMemsetAsync(c->f[VFS_RHS][q], 0, bytes, c->stream);
  if ((rc = formfunction2(c, 1.0, false, 0.0))) return rc;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(c->f[VFS_RHS_O][q], c->f[VFS_RHS][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  return VFS_OK;
}

// Implicit_MatrixFree (implicitsolver.c:4196-4420).
int implicit_momentum(Ctx *c, vfs_newton_stats *st) {
  int rc;
  if ((rc = ensure_work(c))) return rc;
  Work w = work(c);
  const long long n3 = w.n3;
  const double tol = c->cfg.imp_tol > 0 ? c->cfg.imp_tol : 1e-4;
  if ((rc = inflow_flux(c))) return rc;
  if ((rc = form_bcs(c, false))) return rc;   // outflow_scale = 0
  to_vec(c, VFS_UCONT, w.U);
  if ((rc = residual_at(c, w.U, w.F))) return rc;
  double f0 = 0, f = 0;
  if ((rc = vnorm(c, n3, w.F, &f0))) return rc;
  if (!std::isfinite(f0)) return set_err(c, VFS_ERR_INVALID, "implicit momentum: the residual of the initial state is not finite");
  f = f0;
  int its = 0, kits = 0;
  bool converged = f <= tol * f0 || f == 0;
  while (!converged && its < kImpNewton) {
    double unorm = 0;
    if ((rc = vnorm(c, n3, w.U, &unorm))) return rc;
    if ((rc = newton_direction(c, w, f, unorm, kImpForcing, &kits))) return rc;
    // backtracking on |F|: the first step length that decreases it sufficiently
    double lambda = 1.0, ft = 0;
    for (int ls = 0; ls < kImpLineSearch; ls++, lambda *= 0.5) {
      if ((rc = lincomb(c, n3, 1.0, w.U, lambda, w.D, w.UT))) return rc;
      if ((rc = residual_at(c, w.UT, w.FT))) return rc;
      if ((rc = vnorm(c, n3, w.FT, &ft))) return rc;
      if (ft <= (1.0 - 1e-4 * lambda) * f) break;
    }
    std::swap(w.U, w.UT);   // the accepted trial becomes the iterate
    std::swap(w.F, w.FT);
    f = ft;
    its++;
    converged = f <= tol * f0;
  }
  // the last residual evaluated was at the solution: Ucat and the fixed faces of Ucont
  // belong to it.  Ucont takes the solution itself (VecCopy(U, user->Ucont)), then the
  // reference's fix-ups, FormBCS with the outlet rescaling, the IB-node reconstruction.
  from_vec(c, VFS_UCONT, w.U);
  c->launches++, k_imp_post<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), field3(c, VFS_UCONT),
                                                                           field3(c, VFS_UCAT));
  if ((rc = check_launch(c, "k_imp_post"))) return rc;
  if ((rc = form_bcs(c, true))) return rc;
  if (c->g.immersed && c->ti > 0 && (rc = ibm_interpolation(c))) return rc;
  if (st) {
    memset(st, 0, sizeof(*st));
    st->newton_iterations = its;
    st->krylov_iterations = kits;
    st->converged = converged ? 1 : 0;
    st->f0 = f0;
    st->ffinal = f;
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "implicit momentum failed");
  return converged ? VFS_OK : set_err(c, VFS_ERR_NOT_CONVERGED, "implicit momentum: Newton iteration cap reached");
}

}  // namespace vfs

extern "C" {

int vfs_implicit_residual(vfs_ctx *ctx) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c) return VFS_ERR_INVALID;
  cudaSetDevice(c->device);
  if (!c->metrics_set || !c->nvert_set) return vfs::set_err(c, VFS_ERR_STATE, "vfs_implicit_residual: set-up incomplete");
  int rc = vfs::implicit_residual(c);
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess)
    rc = vfs::set_err(c, VFS_ERR_CUDA, "vfs_implicit_residual failed");
  return rc;
}

int vfs_implicit_momentum(vfs_ctx *ctx, vfs_newton_stats *stats) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c) return VFS_ERR_INVALID;
  cudaSetDevice(c->device);
  if (!c->metrics_set || !c->nvert_set) return vfs::set_err(c, VFS_ERR_STATE, "vfs_implicit_momentum: set-up incomplete");
  return vfs::implicit_momentum(c, stats);
}

}  // extern "C"
