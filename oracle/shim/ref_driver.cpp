// Driver for the shim-compiled reference (oracle/_ref/libvfsref.so).
//
// Test infrastructure only.  It replaces the reference's main()/Flow_Solver() with a
// handful of extern "C" entry points so the parity tests can run the reference's own
// hot-path functions (momentum.c, rhs.c, poisson.c, main.c, les.c ...) on synthetic
// grid.dat/bcs.dat inputs and read every field back.  The reference's scalar globals
// (i_periodic, les, immersed, ...) are plain C symbols of this library and are set by
// the caller by name.
//
// Set-up follows the reference: MG_Initial (init.c:270) reads grid.dat and bcs.dat,
// creates the DA and every Vec, and calls FormMetrics (metrics.c:4); main() then adds
// lUstar (main.c:2245) and Flow_Solver adds Fp/Div*/Visc* (solvers.c:779-785).
#include "variables.h"

#include <csetjmp>
#include <csignal>
#include <string>
#include <vector>

extern PetscInt ti, tistart;
extern char path[256], gridfile[256];
extern PetscReal L_dim;
extern int block_number;
extern PetscErrorCode VolumeFlux(UserCtx *user, PetscReal *ibm_Flux, PetscReal *ibm_Area, PetscInt flg);
extern PetscErrorCode VolumeFlux(UserCtx *user, Vec lUcor, PetscReal *ibm_Flux, PetscReal *ibm_Area);
extern void Convert_Phi2_Phi(UserCtx *user);
extern PetscInt setup_lidx2(UserCtx *user);
extern void Pressure_Gradient(UserCtx *user, Vec dP);
extern void IB_BC(UserCtx *user);
extern PetscErrorCode PoissonRHS2(UserCtx *user, Vec B);
extern PetscErrorCode ibm_interpolation_advanced(UserCtx *user);
extern void PoissonRHS2_hypre(UserCtx *user, HYPRE_IJVector &B, int i_lower);
extern void Remove_Nullspace(UserCtx *user, HYPRE_IJVector &B, int i_lower);

extern double inletArea;
extern PetscErrorCode FormFunction_SNES(SNES snes, Vec Ucont, Vec Rhs, void *ptr);  // momentum.c:2197
static Vec g_Uin = 0;  // the Ucont handed to FormFunction_SNES
extern char path[256];                                  // main.c:210
extern PetscErrorCode Ucont_P_Binary_Output(UserCtx *user);  // main.c:765
extern PetscErrorCode Ucont_P_Binary_Input(UserCtx *user);   // main.c:394
extern PetscInt point_cell_advanced(Cmpnts p, PetscInt ip, PetscInt jp, PetscInt kp, IBMNodes *ibm, PetscInt ncx,
                                    PetscInt ncy, PetscInt ncz, PetscReal dcx, PetscReal dcy, PetscReal xbp_min,
                                    PetscReal ybp_min, PetscReal zbp_max, LIST *cell_trg, PetscInt flg);
extern void initlist(LIST *ilist);
extern PetscErrorCode BoundingSphere(IBMNodes *ibm);
extern PetscErrorCode nearestcell1(Cmpnts p, IBMNodes *ibm, IBMInfo *ibminfo);
extern PetscErrorCode InterceptionPoint(Cmpnts p, PetscInt i, PetscInt j, PetscInt k, IBMInfo *ibminfo, UserCtx *user);
extern IBMNodes *ibm_ptr;  // main.c:296
extern void insertnode(LIST *ilist, PetscInt Node);
extern void destroy(LIST *ilist);
extern int ucont_plane_allocated;  // main.c:238
extern int outflow_scale;          // bcs.c:1839
extern int k_area_allocated;  // bcs.c:213, once per process in the reference

static UserMG g_usermg;
static UserCtx *g_user = 0;
static IBMNodes *g_ibm = 0;
static FSInfo *g_fsi = 0;
static Vec g_B = 0;  // compressed Poisson right-hand side (PoissonRHS2 output)

static Vec field_vec(const std::string &n) {
  UserCtx *u = g_user;
  if (n == "Ucont") return u->Ucont;
  if (n == "lUcont") return u->lUcont;
  if (n == "Ucat") return u->Ucat;
  if (n == "lUcat") return u->lUcat;
  if (n == "lUcat_old") return u->lUcat_old;
  if (n == "Ucont_o") return u->Ucont_o;
  if (n == "lUcont_o") return u->lUcont_o;
  if (n == "P") return u->P;
  if (n == "lP") return u->lP;
  if (n == "Phi") return u->Phi;
  if (n == "lPhi") return u->lPhi;
  if (n == "Nvert") return u->Nvert;
  if (n == "lNvert") return u->lNvert;
  if (n == "Nvert_o") return u->Nvert_o;
  if (n == "lNvert_o") return u->lNvert_o;
  if (n == "Rhs") return u->Rhs;
  if (n == "dP") return u->dP;
  if (n == "lNu_t") return u->lNu_t;
  if (n == "lCs") return u->lCs;
  if (n == "lUstar") return u->lUstar;
  if (n == "Gid") return u->Gid;
  if (n == "Fp") return u->Fp;
  if (n == "Div1") return u->Div1;
  if (n == "Div2") return u->Div2;
  if (n == "Div3") return u->Div3;
  if (n == "Visc1") return u->Visc1;
  if (n == "Visc2") return u->Visc2;
  if (n == "Visc3") return u->Visc3;
  if (n == "lCent") return u->lCent;
  if (n == "lCsi") return u->lCsi;
  if (n == "lEta") return u->lEta;
  if (n == "lZet") return u->lZet;
  if (n == "lAj") return u->lAj;
  if (n == "lICsi") return u->lICsi;
  if (n == "lIEta") return u->lIEta;
  if (n == "lIZet") return u->lIZet;
  if (n == "lIAj") return u->lIAj;
  if (n == "lJCsi") return u->lJCsi;
  if (n == "lJEta") return u->lJEta;
  if (n == "lJZet") return u->lJZet;
  if (n == "lJAj") return u->lJAj;
  if (n == "lKCsi") return u->lKCsi;
  if (n == "lKEta") return u->lKEta;
  if (n == "lKZet") return u->lKZet;
  if (n == "lKAj") return u->lKAj;
  if (n == "Phi2") return u->Phi2;
  if (n == "RHS_o") return u->RHS_o;
  if (n == "Uin") {
    if (!g_Uin) VecDuplicate(u->Ucont, &g_Uin);
    return g_Uin;
  }
  if (n == "B") return g_B;
  if (n == "coor") { Vec c; DAGetGhostedCoordinates(u->da, &c); return c; }
  return 0;
}

extern "C" {

// Reads <dir>/grid.dat and <dir>/bcs.dat with the reference's MG_Initial.  The caller
// sets the reference globals that MG_Initial consults (les, immersed, rans ...) first.
int ref_setup(const char *dir) {
  g_Uin = 0;  // sized for the grid of the last set-up
  strncpy(path, dir, sizeof(path) - 1);
  strcpy(gridfile, "grid.dat");
  L_dim = 1.0;
  memset(&g_usermg, 0, sizeof(g_usermg));
  g_ibm = (IBMNodes *)calloc(4, sizeof(IBMNodes));
  g_fsi = (FSInfo *)calloc(4, sizeof(FSInfo));
  if (MG_Initial(&g_usermg, g_ibm)) return 1;
  g_user = g_usermg.mgctx[g_usermg.mglevels - 1].user;
  VecDuplicate(g_user->lP, &g_user->lUstar);
  VecDuplicate(g_user->lUcont, &g_user->Fp);
  VecDuplicate(g_user->lUcont, &g_user->Div1);
  VecDuplicate(g_user->lUcont, &g_user->Div2);
  VecDuplicate(g_user->lUcont, &g_user->Div3);
  VecDuplicate(g_user->lUcont, &g_user->Visc1);
  VecDuplicate(g_user->lUcont, &g_user->Visc2);
  VecDuplicate(g_user->lUcont, &g_user->Visc3);
  VecDuplicate(g_user->Ucont, &g_user->Rhs);
  if (!g_user->lNu_t) VecDuplicate(g_user->lP, &g_user->lNu_t);
  if (!g_user->lCs) VecDuplicate(g_user->lP, &g_user->lCs);
  return 0;
}

void ref_dims(int *mx, int *my, int *mz) {
  *mx = g_user->info.mx; *my = g_user->info.my; *mz = g_user->info.mz;
}

UserCtx *ref_user(void) { return g_user; }

void ref_set_params(double ren, double dt, double st) { g_user->ren = ren; g_user->dt = dt; g_user->st = st; }
void ref_get_params(double *ren, double *dt, double *st) { *ren = g_user->ren; *dt = g_user->dt; *st = g_user->st; }
void ref_set_bctype(const int *bc) { for (int q = 0; q < 6; q++) g_user->bctype[q] = bc[q]; }
void ref_get_bctype(int *bc) { for (int q = 0; q < 6; q++) bc[q] = g_user->bctype[q]; }
void ref_get_kflux(double *flux, double *area) { *flux = g_user->mean_k_flux; *area = g_user->mean_k_area; }
void ref_set_kflux(double flux, double area) { g_user->mean_k_flux = flux; g_user->mean_k_area = area; }

// Entries of a named Vec (mx*my*mz*dof for DA vectors); -1 if unknown.
long ref_field_size(const char *name) {
  Vec v = field_vec(name);
  return v ? (long)v->n : -1;
}
int ref_get_field(const char *name, double *out) {
  Vec v = field_vec(name);
  if (!v) return 1;
  memcpy(out, v->data, sizeof(double) * v->n);
  return 0;
}
int ref_set_field(const char *name, const double *in) {
  Vec v = field_vec(name);
  if (!v) return 1;
  memcpy(v->data, in, sizeof(double) * v->n);
  return 0;
}

// ---- hot-path entry points, each a direct call of the reference function
int ref_contra2cart(void) { Contra2Cart(g_user); return 0; }
int ref_formfunction2(double scale) { return Formfunction_2(g_user, g_user->Rhs, scale); }
int ref_pressure_gradient(void) { Pressure_Gradient(g_user, g_user->dP); return 0; }
int ref_calc_k_flux(void) { Calc_k_Flux(g_user); return 0; }
// Calc_Inlet_Area (bcs.c:216), called once at the first time step (main.c:3488); it also
// allocates user->k_area, which Calc_k_Flux reads.
int ref_calc_inlet_area(void) {
  // each oracle set-up builds a fresh UserCtx, so its k_area must be allocated again
  k_area_allocated = 0;
  g_user->mean_k_area = 0;
  Calc_Inlet_Area(g_user);
  return 0;
}
double ref_inlet_area(void) { return inletArea; }
int ref_runge_kutta(void) { return RungeKutta(g_user, g_ibm, g_fsi); }
int ref_form_bcs(void) { return FormBCS(g_user, g_fsi); }
int ref_inflow_flux(void) { return InflowFlux(g_user); }
// FormBCS with the outlet rescaling switched as RungeKutta switches it (rhs.c:1598, 1670).
int ref_form_bcs_scaled(int scale) {
  outflow_scale = scale;
  int rc = FormBCS(g_user, g_fsi);
  outflow_scale = 1;
  return rc;
}
double ref_flux_in(void) { return FluxInSum; }
// The inflow plane of inletprofile 100 (user->ucont_plane, [j][i] of Cmpnts, as
// read_inflow_section fills it, rhs2.c:712-722).
int ref_set_inflow_plane(const double *plane) {
  const int mx = g_user->info.mx, my = g_user->info.my;
  // read_inflow_section allocates the plane once per process (ucont_plane_allocated); each
  // oracle set-up builds a new UserCtx, which gets its own plane here
  static UserCtx *owner = 0;
  if (owner != g_user) {
    ucont_plane_allocated = 1;
    g_user->ucont_plane = (Cmpnts **)malloc(sizeof(Cmpnts *) * my);
    for (int j = 0; j < my; j++) g_user->ucont_plane[j] = (Cmpnts *)malloc(sizeof(Cmpnts) * mx);
    owner = g_user;
  }
  for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
      const double *p = plane + 3 * ((long)j * mx + i);
      g_user->ucont_plane[j][i].x = p[0];
      g_user->ucont_plane[j][i].y = p[1];
      g_user->ucont_plane[j][i].z = p[2];
    }
  return 0;
}
int ref_ib_bc(void) { IB_BC(g_user); return 0; }

// FormFunction_SNES (momentum.c:2197): the implicit momentum residual of Uin into Rhs (it
// also leaves the evaluated Ucont in Ucont/lUcont and its Ucat in Ucat/lUcat).
int ref_formfunction_snes(void) {
  if (!g_Uin) VecDuplicate(g_user->Ucont, &g_Uin);
  return FormFunction_SNES(0, g_Uin, g_user->Rhs, g_user);
}
// Restart files of time step `step` in directory dir: Ucont_P_Binary_Output /
// Ucont_P_Binary_Input (main.c:765, main.c:394) with the run's `path` and `ti`.
int ref_restart_output(const char *dir, int step) {
  strncpy(path, dir, sizeof(path) - 1);
  const int saved = ti;
  ti = step;
  const int rc = Ucont_P_Binary_Output(g_user);
  ti = saved;
  return rc;
}
int ref_restart_input(const char *dir, int step) {
  strncpy(path, dir, sizeof(path) - 1);
  const int saved = ti;
  ti = step;
  const int rc = Ucont_P_Binary_Input(g_user);
  ti = saved;
  return rc;
}
// The end of one physical time step in the reference's time loop (main.c:3571-3602):
// the old-value copies that the next step reads (Ucont_o, Ucont_rm1, P_o, and lUcat_old,
// the slip-wall ghost source of Contra2Cart), for the single block of the oracle.
int ref_end_of_step(void) {
  UserCtx *user = g_user;
  if (immersed) {
    VecCopy(user->Nvert, user->Nvert_o);
    DAGlobalToLocalBegin(user->da, user->Nvert_o, INSERT_VALUES, user->lNvert_o);
    DAGlobalToLocalEnd(user->da, user->Nvert_o, INSERT_VALUES, user->lNvert_o);
  }
  VecCopy(user->Ucont_o, user->Ucont_rm1);
  VecCopy(user->Ucont, user->Ucont_o);
  VecCopy(user->P, user->P_o);
  DAGlobalToLocalBegin(user->fda, user->Ucont_o, INSERT_VALUES, user->lUcont_o);
  DAGlobalToLocalEnd(user->fda, user->Ucont_o, INSERT_VALUES, user->lUcont_o);
  DAGlobalToLocalBegin(user->fda, user->Ucont_rm1, INSERT_VALUES, user->lUcont_rm1);
  DAGlobalToLocalEnd(user->fda, user->Ucont_rm1, INSERT_VALUES, user->lUcont_rm1);
  DAGlobalToLocalBegin(user->fda, user->Ucat, INSERT_VALUES, user->lUcat_old);
  DAGlobalToLocalEnd(user->fda, user->Ucat, INSERT_VALUES, user->lUcat_old);
  return 0;
}
int ref_update_pressure(void) { return UpdatePressure(g_user); }
int ref_projection(void) { return Projection(g_user); }
int ref_divergence(void) { return Divergence(g_user); }
int ref_les(int recompute_cs) {
  if (recompute_cs) Compute_Smagorinsky_Constant_1(g_user, g_user->lUcont, g_user->lUcat);
  Compute_eddy_viscosity_LES(g_user);
  return 0;
}
int ref_volume_flux(double *flux, double *area) {
  return VolumeFlux(g_user, g_user->Ucont, flux, area);
}
// VolumeFlux(user, &ibm_Flux, &ibm_Area, 0) (poisson.c:3570), the immersed = 1 overload.
int ref_volume_flux_ibm(double *flux, double *area) {
  return VolumeFlux(g_user, flux, area, 0);
}

// nearestcell1 (ibm.c:1366-1512) ends without a return statement; g++ 13 compiles the end
// of the function to a trap instruction (ud2) at every optimisation level.  Everything the
// function computes is stored before that point, so the driver calls it under a SIGILL
// handler that jumps back to the call site: the reference's own arithmetic, run to its
// last statement.
static sigjmp_buf g_trap_jmp;
static void on_trap(int) { siglongjmp(g_trap_jmp, 1); }
static void call_nearestcell1(Cmpnts p, IBMNodes *ibm, IBMInfo *info) {
  struct sigaction sa, old;
  memset(&sa, 0, sizeof(sa));
  sa.sa_handler = on_trap;
  sigemptyset(&sa.sa_mask);
  sigaction(SIGILL, &sa, &old);
  if (sigsetjmp(g_trap_jmp, 1) == 0) nearestcell1(p, ibm, info);
  sigaction(SIGILL, &old, 0);
}

// The nvert classification of ibm_search_advanced (ibm.c:85-345, 507-514) for body ibi,
// with the reference's own ray test: the bins are built with its list functions
// (initlist/insertnode, variables.c:3-27) over the same bin ranges (ibm.c:132-198), every
// cell centre inside the widened box is classified by its point_cell_advanced (ibm.c:1068,
// with randomdirection and intsect_triangle), then the near-boundary marking and the
// 2 -> 1, 4 -> 3 remap follow ibm.c:322-345 and 507-514.  ibm_search_advanced itself goes
// on to build the IB-node interpolation list; under this shim that call does not return,
// so the driver runs the classification steps around the reference's ray test instead.
// Surface as the reader leaves it (ibm_io.c:582-905), normals formed as it forms them.
int ref_ibm_classify(int ibi, int n_v, const double *x, const double *y, const double *z, int n_elmt,
                     const int *n1, const int *n2, const int *n3, int build_list) {
  IBMNodes &ibm = g_ibm[ibi];  // heap storage of ref_setup (the struct is too large for the stack)
  memset(&ibm, 0, sizeof(IBMNodes));
  ibm.n_v = n_v;
  ibm.n_elmt = n_elmt;
  ibm.x_bp = (PetscReal *)x; ibm.y_bp = (PetscReal *)y; ibm.z_bp = (PetscReal *)z;
  // owned copies: the IB-node interpolation reads the surface at every step
  ibm.x_bp = (PetscReal *)malloc(sizeof(PetscReal) * n_v);
  ibm.y_bp = (PetscReal *)malloc(sizeof(PetscReal) * n_v);
  ibm.z_bp = (PetscReal *)malloc(sizeof(PetscReal) * n_v);
  memcpy(ibm.x_bp, x, sizeof(double) * n_v);
  memcpy(ibm.y_bp, y, sizeof(double) * n_v);
  memcpy(ibm.z_bp, z, sizeof(double) * n_v);
  ibm.nv1 = (PetscInt *)malloc(sizeof(PetscInt) * n_elmt);
  ibm.nv2 = (PetscInt *)malloc(sizeof(PetscInt) * n_elmt);
  ibm.nv3 = (PetscInt *)malloc(sizeof(PetscInt) * n_elmt);
  for (int e = 0; e < n_elmt; e++) { ibm.nv1[e] = n1[e]; ibm.nv2[e] = n2[e]; ibm.nv3[e] = n3[e]; }
  std::vector<PetscReal> fx(n_elmt), fy(n_elmt), fz(n_elmt);
  for (int e = 0; e < n_elmt; e++) {
    const double dx12 = x[n2[e]] - x[n1[e]], dy12 = y[n2[e]] - y[n1[e]], dz12 = z[n2[e]] - z[n1[e]];
    const double dx13 = x[n3[e]] - x[n1[e]], dy13 = y[n3[e]] - y[n1[e]], dz13 = z[n3[e]] - z[n1[e]];
    double nx = dy12 * dz13 - dz12 * dy13, ny = -dx12 * dz13 + dz12 * dx13, nz = dx12 * dy13 - dy12 * dx13;
    const double dr = sqrt(nx * nx + ny * ny + nz * nz);
    fx[e] = nx / dr; fy[e] = ny / dr; fz[e] = nz / dr;
  }
  ibm.nf_x = (PetscReal *)malloc(sizeof(PetscReal) * n_elmt);
  ibm.nf_y = (PetscReal *)malloc(sizeof(PetscReal) * n_elmt);
  ibm.nf_z = (PetscReal *)malloc(sizeof(PetscReal) * n_elmt);
  memcpy(ibm.nf_x, fx.data(), sizeof(double) * n_elmt);
  memcpy(ibm.nf_y, fy.data(), sizeof(double) * n_elmt);
  memcpy(ibm.nf_z, fz.data(), sizeof(double) * n_elmt);
  // fixed bodies: zero surface velocity; per-triangle statistics the interpolation fills
  ibm.u = (Cmpnts *)calloc(n_v, sizeof(Cmpnts));
  ibm.uold = (Cmpnts *)calloc(n_v, sizeof(Cmpnts));
  ibm.count = (PetscInt *)calloc(n_elmt, sizeof(PetscInt));
  ibm.shear = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm.mean_shear = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm.reynolds_stress1 = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm.reynolds_stress2 = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm.reynolds_stress3 = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm.pressure = (PetscReal *)calloc(n_elmt, sizeof(PetscReal));
  ibm_ptr = g_ibm;
  const int ncx = 40, ncy = 40, ncz = 40;
  double xmin = 1.e23, xmax = -1.e23, ymin = 1.e23, ymax = -1.e23, zmin = 1.e23, zmax = -1.e23;
  for (int q = 0; q < n_v; q++) {
    xmin = PetscMin(xmin, x[q]); xmax = PetscMax(xmax, x[q]);
    ymin = PetscMin(ymin, y[q]); ymax = PetscMax(ymax, y[q]);
    zmin = PetscMin(zmin, z[q]); zmax = PetscMax(zmax, z[q]);
  }
  xmin -= 0.05; xmax += 0.05; ymin -= 0.05; ymax += 0.05; zmin -= 0.05; zmax += 0.05;
  const double dcx = (xmax - xmin) / (ncx - 1.), dcy = (ymax - ymin) / (ncy - 1.), dcz = (zmax - zmin) / (ncz - 1.);
  std::vector<LIST> bins(ncx * ncy * ncz);
  for (auto &l : bins) initlist(&l);
  for (int e = 0; e < n_elmt; e++) {
    const int a = n1[e], b = n2[e], c = n3[e];
    PetscInt i0 = floor((PetscMin(PetscMin(x[a], x[b]), x[c]) - xmin) / dcx);
    PetscInt i1 = floor((PetscMax(PetscMax(x[a], x[b]), x[c]) - xmin) / dcx) + 1;
    PetscInt j0 = floor((PetscMin(PetscMin(y[a], y[b]), y[c]) - ymin) / dcy);
    PetscInt j1 = floor((PetscMax(PetscMax(y[a], y[b]), y[c]) - ymin) / dcy) + 1;
    PetscInt k0 = floor((PetscMin(PetscMin(z[a], z[b]), z[c]) - zmin) / dcz);
    PetscInt k1 = floor((PetscMax(PetscMax(z[a], z[b]), z[c]) - zmin) / dcz) + 1;
    i0 = i0 < 0 ? 0 : i0; i1 = i1 > ncx ? ncx : i1;
    j0 = j0 < 0 ? 0 : j0; j1 = j1 > ncx ? ncy : j1;
    k0 = k0 < 0 ? 0 : k0; k1 = k1 > ncz ? ncz : k1;
    for (int k = k0; k < k1; k++)
      for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) insertnode(&bins[k * ncx * ncy + j * ncx + i], e);
  }
  const int mx = g_user->info.mx, my = g_user->info.my, mz = g_user->info.mz;
  Vec lcent = g_user->lCent, lnv = g_user->lNvert;
  auto at = [&](int i, int j, int k) { return ((long)k * my + j) * mx + i; };
  double *nv = lnv->data;
  const Cmpnts *cent = (const Cmpnts *)lcent->data;
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const long p = at(i, j, k);
        if (ibi == 0 && nv[p] < 5.) nv[p] = 0;
        const Cmpnts c = cent[p];
        if (c.x > xmin && c.x < xmax && c.y > ymin && c.y < ymax && c.z > zmin && c.z < zmax) {
          const PetscInt ic = floor((c.x - xmin) / dcx), jc = floor((c.y - ymin) / dcy), kc = floor((c.z - zmin) / dcz);
          const double val = point_cell_advanced(c, ic, jc, kc, &ibm, ncx, ncy, ncz, dcx, dcy, xmin, ymin, zmax,
                                                 bins.data(), 0);
          nv[p] = PetscMax(nv[p], val);
          if (nv[p] < 0) nv[p] = 0;
        }
      }
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        const long p = at(i, j, k);
        if ((int)(nv[p] + 0.5) == 4) continue;
        const int ip = i < mx - 1 ? i + 1 : i, im = i > 0 ? i - 1 : i;
        const int jp = j < my - 1 ? j + 1 : j, jm = j > 0 ? j - 1 : j;
        const int kp = k < mz - 1 ? k + 1 : k, km = k > 0 ? k - 1 : k;
        for (int kk = km; kk <= kp; kk++)
          for (int jj = jm; jj <= jp; jj++)
            for (int ii = im; ii <= ip; ii++)
              if ((int)(nv[at(ii, jj, kk)] + 0.5) == 4) nv[p] = PetscMax(2, nv[p]);
      }
  // cells a moving body has uncovered since the last step (Nvert_o > 2.5, now fluid)
  // become IB nodes, at the search of the last body (ibm.c:346-357)
  extern PetscInt NumberOfBodies;  // main.c
  if (ibi == NumberOfBodies - 1) {
    const double *nvo = g_user->lNvert_o->data;
    for (long p = 0; p < (long)mx * my * mz; p++)
      if (nvo[p] > 2.5 && nv[p] < 0.5) nv[p] = 2;
  }
  if (build_list) {
    // the IB-node list of ibm.c:347-505 with the reference's own geometry (BoundingSphere,
    // nearestcell1, InterceptionPoint); the two fallbacks for a failed interception are
    // those of ibm.c:400-500
    static UserCtx *listed = 0;
    if (listed != g_user) {
      PetscMalloc(4 * sizeof(IBMList), &g_user->ibmlist);
      for (int b = 0; b < 4; b++) InitIBMList(&g_user->ibmlist[b]);
      listed = g_user;
    }
    if (g_user->ibmlist[ibi].head) DestroyIBMList(&g_user->ibmlist[ibi]);
    InitIBMList(&g_user->ibmlist[ibi]);
    BoundingSphere(&ibm);
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          if ((int)(nv[at(i, j, k)] + 0.5) != 2) continue;
          IBMInfo info;
          memset(&info, 0, sizeof(info));
          info.ni = i; info.nj = j; info.nk = k;
          const Cmpnts c = cent[at(i, j, k)];
          call_nearestcell1(c, &ibm, &info);
          InterceptionPoint(c, i, j, k, &info, g_user);
          if (info.imode < 0) {
            int dk = 0, dj = 0;
            if (i == 1 || i == mx - 2 || j == 1 || j == my - 2) dk = ibm.nf_z[info.cell] > 0 ? 1 : -1;
            else if (k == 1 || k == mz - 2) dj = 1;
            if (dk || dj) {
              const Cmpnts q = cent[at(i, j + dj, k + dk)];
              info.d_i = sqrt((c.x - q.x) * (c.x - q.x) + (c.y - q.y) * (c.y - q.y) + (c.z - q.z) * (c.z - q.z));
              info.cr1 = 1.; info.cr2 = 0.; info.cr3 = 0.;
              info.i1 = info.i2 = info.i3 = i;
              info.j1 = info.j2 = info.j3 = j + dj;
              info.k1 = info.k2 = info.k3 = k + dk;
            }
          }
          AddIBMNode(&g_user->ibmlist[ibi], info);
        }
    free(ibm.qvec);
    free(ibm.radvec);
  }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const long p = at(i, j, k);
        if ((int)(nv[p] + 0.5) == 2) nv[p] = 1;
        if ((int)(nv[p] + 0.5) == 4) nv[p] = 3;
      }
  VecCopy(lnv, g_user->Nvert);
  for (auto &l : bins) destroy(&l);
  return 0;
}

// The IB-node list of body ibi as arrays (node i j k, cell, imode, stencil i1 j1 k1 i2 ...
// k3, weights cr1..3, cs1..3, d_s, d_i); returns the number of nodes (list order).
int ref_ibm_list(int ibi, int *ints, double *dbls, int cap) {
  int n = 0;
  for (IBMListNode *c = g_user->ibmlist[ibi].head; c; c = c->next, n++) {
    if (n >= cap) continue;
    const IBMInfo &f = c->ibm_intp;
    int *q = ints + 14 * n;
    q[0] = f.ni; q[1] = f.nj; q[2] = f.nk; q[3] = f.cell; q[4] = f.imode;
    q[5] = f.i1; q[6] = f.j1; q[7] = f.k1; q[8] = f.i2; q[9] = f.j2; q[10] = f.k2;
    q[11] = f.i3; q[12] = f.j3; q[13] = f.k3;
    double *d = dbls + 8 * n;
    d[0] = f.cr1; d[1] = f.cr2; d[2] = f.cr3; d[3] = f.cs1; d[4] = f.cs2; d[5] = f.cs3; d[6] = f.d_s; d[7] = f.d_i;
  }
  return n;
}

// The surface velocity of body ibi's vertices (ibm->u), as a body-motion routine leaves it.
int ref_ibm_set_velocity(int ibi, int n_v, const double *u, const double *v, const double *w) {
  IBMNodes &ibm = g_ibm[ibi];
  if (n_v != ibm.n_v || !ibm.u) return 1;
  for (int q = 0; q < n_v; q++) { ibm.u[q].x = u[q]; ibm.u[q].y = v[q]; ibm.u[q].z = w[q]; }
  return 0;
}

// ibm_interpolation_advanced (ibm.c:3294) on the current fields.
int ref_ibm_interpolation(int nbodies) {
  extern PetscInt NumberOfBodies;
  NumberOfBodies = nbodies;
  return ibm_interpolation_advanced(g_user);
}

// PoissonLHSNew (poisson.c:971); the matrix stays recorded in user->A.
int ref_poisson_lhs(void) {
  g_user->assignedA = PETSC_FALSE;
  return PoissonLHSNew(g_user, g_ibm, g_user->ibm_intp);
}
long ref_poisson_csr(int *row_ptr, int *col, double *val, int *m) {
  return shim_mat_to_csr(g_user->A, row_ptr, col, val, m);
}
// PoissonRHS2 (poisson.c:1774) into a compressed vector sized like Phi2.
int ref_poisson_rhs2(void) {
  if (g_B) VecDestroy(g_B);
  VecDuplicate(g_user->Phi2, &g_B);
  return PoissonRHS2(g_user, g_B);
}
// PoissonRHS2_hypre (poisson_hypre.c:330, with Remove_Nullspace_Scale) into out[0..n);
// returns the number of unknowns (Phi2 size) or -1.
static HYPRE_IJVector g_ijb = 0;
int ref_poisson_rhs2_hypre(double *out) {
  int n = 0;
  VecGetLocalSize(g_user->Phi2, &n);
  if (g_ijb) HYPRE_IJVectorDestroy(g_ijb);
  HYPRE_IJVectorCreate(PETSC_COMM_WORLD, 0, n - 1, &g_ijb);
  PoissonRHS2_hypre(g_user, g_ijb, 0);
  int m = 0;
  double *d = shim_ij_data(g_ijb, &m);
  if (out) memcpy(out, d, sizeof(double) * m);
  return m;
}
// Remove_Nullspace (poisson_hypre.c:194) applied to a compressed solution in place.
int ref_remove_nullspace(double *x, int n) {
  HYPRE_IJVector v;
  HYPRE_IJVectorCreate(PETSC_COMM_WORLD, 0, n - 1, &v);
  int m = 0;
  double *d = shim_ij_data(v, &m);
  memcpy(d, x, sizeof(double) * n);
  Remove_Nullspace(g_user, v, 0);
  memcpy(x, d, sizeof(double) * n);
  HYPRE_IJVectorDestroy(v);
  return 0;
}
int ref_phi2_size(void) { int n = 0; VecGetLocalSize(g_user->Phi2, &n); return n; }

// Convert_Phi2_Phi (poisson.c:92): compressed solution -> grid Phi (and lPhi).
int ref_convert_phi2_phi(void) {
  Convert_Phi2_Phi(g_user);
  DAGlobalToLocalBegin(g_user->da, g_user->Phi, INSERT_VALUES, g_user->lPhi);
  DAGlobalToLocalEnd(g_user->da, g_user->Phi, INSERT_VALUES, g_user->lPhi);
  return 0;
}

}  // extern "C"
