// Internal definitions shared by the sm_100a kernels and the C-ABI layer.
//
// Device data layout (one structured block, one GPU):
//   * Every field covers the reference's whole DA extent, mx*my*mz points with
//     mx = IM+1 (init.c:154), in the reference's linear order ((k*my)+j)*mx+i, so a
//     host array in the reference layout maps 1:1 onto a device index.
//   * Vector fields are stored as three separate component arrays (SoA) so that a warp
//     reading consecutive i of one component issues fully coalesced 8-byte loads.
//   * The IB flag field nvert (0/1/3 in the reference, stored as doubles) is stored as
//     uint8: every threshold test of the reference (>0.1, <0.1, (int)(x+0.5)==1, >1.1,
//     (int)(x+0.1)==3 ...) is exact on small integers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/vfs_b200.h"

namespace vfs {

// Scalar run parameters passed by value to every kernel.
struct Grid {
  int mx, my, mz;
  long long N;          // mx*my*mz
  int iper, jper, kper; // i_periodic, j_periodic, k_periodic
  int bc[6];            // bctype
  int immersed, les;
  double ren, dt, st;
  int wallfunction;     // -wallfunction: wall model in the IB-node reconstruction
  int moving;           // movefsi || rotatefsi: moving bodies
  double roughness;     // -roughness: rough-wall log law for body 0 (0: unset)
};

__host__ __device__ inline long long lidx(const Grid &g, int i, int j, int k) {
  return ((long long)k * g.my + j) * g.mx + i;
}

// (i, j, k) of DA point p in 32-bit arithmetic (vfs_create admits grids of fewer than 2^31
// points), which costs a fraction of 64-bit division.
__device__ __forceinline__ void dijk(const Grid &g, long long p, int &i, int &j, int &k) {
  const unsigned up = (unsigned)p, umx = (unsigned)g.mx, umy = (unsigned)g.my;
  const unsigned r = up / umx, kk = r / umy;
  i = (int)(up - r * umx);
  j = (int)(r - kk * umy);
  k = (int)kk;
}

// Periodic image of a ghost index (0 -> m-2, m-1 -> 1) in a periodic direction, as the
// reference's periodic copy loops do (e.g. momentum.c:641-669); identity otherwise.
__host__ __device__ inline int wrapi(const Grid &g, int i) {
  if (g.iper) { if (i == 0) return g.mx - 2; if (i == g.mx - 1) return 1; }
  return i;
}
__host__ __device__ inline int wrapj(const Grid &g, int j) {
  if (g.jper) { if (j == 0) return g.my - 2; if (j == g.my - 1) return 1; }
  return j;
}
__host__ __device__ inline int wrapk(const Grid &g, int k) {
  if (g.kper) { if (k == 0) return g.mz - 2; if (k == g.mz - 1) return 1; }
  return k;
}

// Three-component SoA vector field.
struct V3 {
  double *x, *y, *z;
};
struct CV3 {
  const double *x, *y, *z;
};
inline CV3 cv(const V3 &v) { return CV3{v.x, v.y, v.z}; }

// Metric arrays (FormMetrics, metrics.c:4).
struct Metrics {
  CV3 csi, eta, zet;    // centre
  const double *aj;
  CV3 icsi, ieta, izet; // i-faces
  const double *iaj;
  CV3 jcsi, jeta, jzet; // j-faces
  const double *jaj;
  CV3 kcsi, keta, kzet; // k-faces
  const double *kaj;
};

// Poisson operator: 19 coefficients per cell in the slot order of PoissonLHSNew
// (poisson.c:951-969: CP EP WP NP SP TP BP NE SE NW SW TN BN TS BS TE BE TW BW).
enum { CP = 0, EP, WP, NP, SP, TP, BP, NE, SE, NW, SW, TN, BN, TS, BS, TE, BE, TW, BW, NSLOT };

// One multigrid level in zebra order (see vfs_mg.cu): cells ((k*ny + j)*2 + colour)*hx
// + i/2 with colour = (i xor k) & 1, hx = ceil(nx/2), n slots in all.
struct ZL {
  int nx, ny, nz, hx, ip, jp, kp;
  long long n;
};

struct MGLevel {
  ZL z;
  bool zebra = true;        // two-colour line Gauss-Seidel is race-free on this level
  double *op64 = nullptr;   // 6n: couplings +i, +j, +k, diagonal, Thomas factors cpr, 1/pivot
  double *pk64 = nullptr;   // 8n: packed operator (two 4-vectors per cell), FP64
  float *pk32 = nullptr;    // the same in FP32
  uint8_t *act = nullptr;   // n: 1 for an active unknown (non-zero diagonal)
  double *v64 = nullptr;    // 5n: x, b, previous x (line Jacobi), forward-elimination pairs (2n)
  float *v32 = nullptr;
};

struct Poisson {
  bool built = false;
  double *coef = nullptr;   // NSLOT * N doubles (SoA by slot)
  int nslot = NSLOT;        // 7 when every cross slot is zero (the apply reads slots 0..6)
  uint8_t *fluid = nullptr; // 1 if the cell is a Poisson unknown (gid >= 0)
  long long nfluid = 0;
  double sum_aj = 0;        // sum of aj over fluid cells (Remove_Nullspace_Scale)
  std::vector<MGLevel> lv;  // multigrid levels, finest first
  // FGMRES workspace (grid layout, N doubles each)
  int restart = 0;
  long long ldv = 0;        // distance between basis vectors (N rounded up to 32)
  double *V = nullptr;      // (restart+1) * ldv
  double *Z = nullptr;      // restart * ldv
  double *w = nullptr, *r = nullptr, *t = nullptr;
  // precision 2 (FP32 inner FGMRES): the basis, the preconditioned vectors and w in FP32
  int restart32 = 0;
  float *V32 = nullptr, *Z32 = nullptr, *w32 = nullptr;
  double *hdev = nullptr;   // Gram-Schmidt coefficients on the device (64 doubles)
  bool transpose = false;   // apply A^T (the adjoint solve)
  bool guess = false;       // VFS_PHI holds the last solution for the current unknowns
};

// One immersed-boundary node of the IB-node list (IBMInfo, variables.h:95-172, as
// ibm_search_advanced fills it, ibm.c:347-505): the node cell, the nearest surface
// triangle and the barycentric weights of its projection, and the three fluid cells
// whose velocities are interpolated across the surface normal.
struct IbNode {
  int i, j, k;        // node cell
  int cell;           // nearest surface triangle (nearestcell1)
  int imode;          // interception mode (0..7), -1 a boundary fallback, -2 unresolved
  int st[9];          // stencil cells i1 j1 k1 i2 j2 k2 i3 j3 k3
  double cr[3];       // stencil weights cr1..cr3
  double cs[3];       // surface weights cs1..cs3
  double ds, di;      // distance to the surface (d_s) and to the interception (d_i)
  int vtx[3];         // vertices of the triangle `cell` in the surface-velocity array
  double nf[3];       // its unit normal (the wall models' n)
};

// Forward quantities of one time step that its tangent and adjoint are linearised about:
// the Ucont and Ucat entering Formfunction_2 at each Runge-Kutta stage and the Ucont
// entering the immersed VolumeFlux (whose |flux| > 1e-8 test selects the corrected faces).
struct StepTape {
  double *uc[4][3] = {}, *uk[4][3] = {};
  double *vfi[3] = {};
  bool first_step = false;
};
struct Adjoint;

// Scalars that a step's reductions produce and later kernels of the same step read; they
// live on the device (Ctx::ds) so that no kernel waits for the host, and the host mirror
// (Ctx::scal) is refreshed from them after the step.  The first three are inputs the
// host sets.
enum DScal {
  DS_INLET_FLUX = 0, DS_INLET_AREA, DS_MEAN_K_AREA,
  DS_KFLUX_SUM, DS_MEAN_K_FLUX, DS_FLUX1, DS_FLUX_IN, DS_FLUX_OUT, DS_AREA_OUT,
  DS_BSUM, DS_PHISUM, DS_MAXDIV, DS_VF_FLUX, DS_VF_AREA,
  DS_COUNT = 16
};

// Device-side state of the flexible GMRES solve (restart <= kKryMax): the Hessenberg
// matrix, the Givens rotations and the loop control, so that the solve's kernels decide
// on the device (and a captured graph can loop on conditional nodes).
constexpr int kKryMax = 31;
struct KryDev {
  int j, it, jdone, reorth, degen, inner_go, outer_go, conv, fresh, check, maxit, m, cycles;
  double tol, bnorm, bb, r0, rnorm, rr, hn, scale;
  double inner_rtol, beta;  // precision 2: a cycle ends once its estimate is below inner_rtol * beta
  double hdev[kKryMax + 3];
  double h[kKryMax + 3], h2[kKryMax + 3], h3[kKryMax + 3];
  double H[(kKryMax + 1) * kKryMax], cs[kKryMax], sn[kKryMax], gv[kKryMax + 1], y[kKryMax];
};

// A step captured as one CUDA graph (vfs_solve_opts.graph), with the options it was
// captured for.
struct StepGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  vfs_solve_opts opts;
  long long key = -1;            // invalidation counter value at capture
  long long launches = 0;        // kernels of a replay with one Krylov cycle and iteration
  long long body_launches = 0;   // kernels of one Krylov iteration
  long long cycle_launches = 0;  // kernels of one Krylov restart cycle outside its iterations
};

struct Ctx {
  vfs_config cfg;
  Grid g;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;

  // fields (SoA component pointers; scalar fields use comp[0])
  double *f[VFS_NFIELDS][3] = {};
  int dof[VFS_NFIELDS] = {};
  uint8_t *nv = nullptr;        // nvert as uint8
  uint8_t *nvo = nullptr;       // Nvert_o: the flags at the end of the last step (immersed)
  double *ibv = nullptr;        // surface velocity of every body's vertices (ibm->u), 3 x nvtx
  int nvtx = 0;                 // vertices of all bodies searched so far
  std::vector<int> vtx_base;    // first vertex of body ibi in ibv
  // scratch for Formfunction_2 (face fluxes and Fp) and Contra2Cart
  double *div[3][3] = {};       // div1..3 x comps
  double *visc[3][3] = {};
  double *fp[3] = {};
  double *pucont[3] = {};
  double *bcbuf[3] = {};        // Contra2Cart boundary two-phase buffer
  uint8_t *bcflag = nullptr;    // points written by the boundary phase
  long long *solid = nullptr;   // indices of the solid (nvert 3) points
  long long nsolid = -1;        // their number; -1 until built for the current nvert
  // reductions
  double *red = nullptr;        // partial sums (device)
  double *red_host = nullptr;   // pinned host mirror
  int red_cap = 0;
  IbNode *ibn = nullptr;        // IB-node list of every searched body (device)
  int nib = 0;                  // its length
  int nib_unresolved = 0;       // nodes whose interception search failed (reference: garbage)
  int nib_body0 = 0;            // the first nib_body0 nodes belong to body 0
  double *ibbuf = nullptr;      // per-node gather buffer (4 doubles per node)
  double *inflow_plane = nullptr;  // inlet velocity plane, my*mx Cartesian triples (inletprofile 100)
  double *inlet_nodes = nullptr;   // grid nodes of the k = 1 node plane: x, y, z blocks of JM*IM
  double *stage = nullptr;      // host-transfer staging buffer (interleaved layout)
  size_t stage_bytes = 0;
  double scal[VFS_NSCALARS] = {};
  bool metrics_set = false, nvert_set = false;
  bool first_step = true;        // ti == tistart set-up pending (main.c:3488, solvers.c:603)
  int ti = 0, tistart = 0, rstart = 0, dynamic_freq = 1;  // time step index and LES schedule
  double max_cs = 0.5;           // upper clip of the Smagorinsky coefficient
  Poisson ps;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  StepTape *tape = nullptr;      // set while a step records its linearisation state
  Adjoint *adj = nullptr;        // tangent/adjoint workspace (vfs_adjoint.cu)
  // device-resident step (CUDA graph)
  double *ds = nullptr;          // DS_COUNT device scalars
  double *ds_in = nullptr;       // pinned: host inputs copied to ds at the start of a step
  double *ds_out = nullptr;      // pinned: ds read back after a step
  KryDev *kd = nullptr;          // FGMRES state on the device
  KryDev *kd_host = nullptr;     // pinned mirror of kd (solve statistics)
  bool capturing = false;        // launches are being captured: no host synchronisation
  StepGraph sg;
  long long setup_epoch = 0;     // bumped whenever a captured step would be stale
  cudaStream_t cap_streams[2] = {nullptr, nullptr};  // bodies of the solver's two loops
  double *imp = nullptr;         // implicit momentum workspace (vfs_implicit.cu)
  int imp_m = 0;                 // its GMRES restart length
  double *gab = nullptr;         // 9 x N face-metric products of Pressure_Gradient / Projection
  bool gab_valid = false;        // false after any metric upload
};

V3 field3(Ctx *c, int f);
Metrics metrics(Ctx *c);

// launch bookkeeping / error checking
int check_launch(Ctx *c, const char *what);
int set_err(Ctx *c, int code, const std::string &msg);
// device scalars: sum of parts into ds-slot memory without a host wait; read back
int reduce_to(Ctx *c, const double *parts, int nparts, double *dst);
int ds_fetch(Ctx *c);
int ds_upload(Ctx *c);
void step_graph_free(Ctx *c);

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// momentum path
int periodic_copy3(Ctx *c, V3 v);
int periodic_copy1(Ctx *c, double *s);
int ensure_gab(Ctx *c);
int contra2cart(Ctx *c);
int solid_list(Ctx *c);
int formfunction2(Ctx *c, double scale, bool rk_stage, double rk_coeff);
int formfunction2_split(Ctx *c, double scale, bool rk_stage, double rk_coeff);
int formfunction2_onepass(Ctx *c, double scale, bool rk_stage, double rk_coeff);
int pressure_gradient(Ctx *c);
int calc_k_flux(Ctx *c, double *flux);
int runge_kutta(Ctx *c);
int form_bcs(Ctx *c, bool outflow_scale);
int inflow_flux(Ctx *c);
int calc_inlet_area(Ctx *c);
int ib_bc(Ctx *c);
int pressure_forcing_mode(const Ctx *c);
int pressure_gradient_mode(Ctx *c, int mode, double kdiff);
int step_core(Ctx *c, const vfs_solve_opts *opts, vfs_step_stats *st);
int step_graph(Ctx *c, const vfs_solve_opts *opts, vfs_step_stats *st);
int form_bcs_tail(Ctx *c);
int outlet_rescale(Ctx *c);

// tangent / adjoint of one RK stage and of the periodic ghost copy (vfs_momentum.cu)
int ff2_stage_tangent(Ctx *c, const double *const uc[3], const double *const uk[3], double a, V3 dU, V3 du, V3 ddp,
                      V3 dpu, double *const tf[3][6]);
int ff2_stage_adjoint(Ctx *c, const double *const uc[3], const double *const uk[3], double a, V3 lU, V3 lu, V3 ldp,
                      V3 lpu, double *const lf[3][6], double *const lfp[3]);

// hand-written transposes of the projection step's stencils (vfs_adjoint_stencil.cu)
int periodic_copy1_adjoint(Ctx *c, double *a);
int periodic_copy3_adjoint(Ctx *c, V3 a);
int pressure_gradient_adjoint(Ctx *c, double *lP, V3 ldp);
int projection_adjoint(Ctx *c, double *lphi, V3 luc);
int update_pressure_adjoint(Ctx *c, double *lP, double *lphi);
int poisson_rhs_local_adjoint(Ctx *c, V3 luc, double *lb);
// hand-written transposes of the boundary operators (vfs_momentum.cu)
bool contra2cart_linear(const Grid &g);
int contra2cart_adjoint(Ctx *c, V3 luc, V3 lucat, V3 luo, V3 tmp);
int form_bcs_tail_adjoint(Ctx *c, V3 luc, V3 lucat, V3 luo, V3 tmp);
int ib_bc_adjoint(Ctx *c, V3 luc);

// tangent / adjoint support (vfs_adjoint.cu)
int tape_stage(Ctx *c, int stage);
int tape_vflux(Ctx *c);
void adjoint_free(Ctx *c);

// immersed boundary (vfs_ibm.cu)
int ibm_interpolation(Ctx *c);
int ib_faces(Ctx *c);
int volume_flux_ibm(Ctx *c, double *flux, double *area);

// dynamic Smagorinsky model (vfs_les.cu)
int smagorinsky_constant(Ctx *c);
int eddy_viscosity(Ctx *c);

// Poisson / correction path
int poisson_lhs(Ctx *c);
int poisson_rhs(Ctx *c);
int poisson_rhs_local(Ctx *c);
int poisson_set_transpose(Ctx *c, bool on);
int volume_flux(Ctx *c);
int poisson_solve(Ctx *c, const vfs_solve_opts *o, vfs_solve_stats *st);
int poisson_prepare(Ctx *c, const vfs_solve_opts *o);
int poisson_apply_dev(Ctx *c, const double *x, double *y);
int update_pressure(Ctx *c);
int projection(Ctx *c);
int divergence(Ctx *c, double *maxdiv);
int correction(Ctx *c, bool fuse_divergence);
// implicit momentum (implicit = 4)
int implicit_rhs_o(Ctx *c);
int implicit_residual(Ctx *c);
int implicit_momentum(Ctx *c, vfs_newton_stats *st);
int divergence_finish(Ctx *c, double *maxdiv);
int contra2cart_div(Ctx *c, bool with_divergence);

// multigrid preconditioner (vfs_mg.cu)
int mg_setup(Ctx *c);
void mg_free(Poisson &P);
int mg_precondition(Ctx *c, const double *v, double *z, const vfs_solve_opts &o);
int mg_precondition_dyn(Ctx *c, const double *V, double *Z, long long ldv, const int *jslot, const vfs_solve_opts &o);
int mg_precondition_dyn32(Ctx *c, const float *V, float *Z, long long ldv, const int *jslot, const vfs_solve_opts &o);
int mg_sweep_fine(Ctx *c, int precision);

// reductions (deterministic two-pass); result copied to host
int reduce_sum(Ctx *c, const double *parts, int nparts, double *out);
int ensure_red(Ctx *c, int n);

}  // namespace vfs
