/*
 * vfs_b200.h — C ABI of the B200 (sm_100a) fractional-step projection path of the
 * VFS-Geophysics curvilinear immersed-boundary solver.
 *
 * One context = one structured block on one GPU, one CUDA stream.  Every field lives
 * in device memory for the life of the context.  Host arrays cross the boundary only
 * through vfs_set_field / vfs_get_field, in the reference's own layout: the PETSc DA of
 * (IM+1) x (JM+1) x (KM+1) points, [k][j][i] with i fastest, vector fields as
 * interleaved {x,y,z} doubles (struct Cmpnts, variables.h:45-57).
 *
 * All entry points return 0 on success or a VFS_ERR_* code; vfs_last_error() gives a
 * one-line message.  No entry point exits the process, and no kernel waits on a flag.
 *
 * Each operator names the reference function it replaces (file:line in the reference
 * solver's sources).  Operators read and write the context's fields exactly where the
 * reference reads and writes its UserCtx vectors.
 */
#ifndef VFS_B200_H
#define VFS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define VFS_OK 0
#define VFS_ERR_INVALID 1        /* bad argument / unsupported option */
#define VFS_ERR_CUDA 2           /* CUDA runtime error (message in vfs_last_error) */
#define VFS_ERR_NOT_CONVERGED 3  /* Poisson solver hit its iteration cap */
#define VFS_ERR_NO_DEVICE 4      /* no CUDA device / kernels missing for this GPU */
#define VFS_ERR_STATE 5          /* operator called before its prerequisites */

typedef struct vfs_ctx vfs_ctx;

/* Run configuration: the subset of the reference's control.dat / bcs.dat options that
 * the projection path reads (main.c:1593-2250, init.c:52-69, init.c:562-568). */
typedef struct {
  int IM, JM, KM;        /* grid nodes per direction (grid.dat header, init.c:374) */
  int bctype[6];         /* bcs.dat codes: i-, i+, j-, j+, k-, k+ */
  int i_periodic, j_periodic, k_periodic; /* main.c:191-195 */
  int immersed;          /* -imm: 0 none, 1 sharp-interface IB (nvert masking + QUICK) */
  int les;               /* -les: 0 laminar, 1 constant Cs = 0.01, 2 dynamic Smagorinsky */
  int inletprofile;      /* -inlet (bcs.c:399-466) */
  int dynamic_freq;      /* -dynamic_freq: Cs recomputed when ti % dynamic_freq == 0 or ti ==
                            tistart (main.c:1747, solvers.c:652); values < 1 mean 1 */
  int tistart;           /* index of the first time step (main.c:5, -rstart) */
  int rstart;            /* non-zero for a restarted run (rstart_flg, main.c:1608) */
  int wallfunction;      /* -wallfunction: the IB-node reconstruction uses the wall model
                            wall_function_roughness_a (ks = 1e-4) from ti > 0 (ibm.c:3454-3474)
                            instead of noslip */
  int moving;            /* movefsi || rotatefsi: the bodies move (ibm.c:3444: IB nodes next
                            to solid cells are reconstructed all the same) */
  int implicit;          /* -imp: 0 explicit 4-stage Runge-Kutta; 4 the matrix-free implicit
                            momentum solve (Implicit_MatrixFree, implicitsolver.c:4196) */
  int reserved_i[2];
  double ren;            /* Reynolds number (user->ren) */
  double dt;             /* time step (user->dt) */
  double st;             /* Strouhal scaling (user->st) */
  double inlet_flux;     /* -inlet_flux target bulk flux (main.c:198; <0: unset) */
  double mean_pressure_gradient; /* -mean_pressure_gradient (main.c) */
  int dpdz_set;          /* non-zero: impose mean_pressure_gradient (momentum.c:379) */
  int reserved_j[7];
  double max_cs;         /* -max_cs upper clip of Cs (main.c:216, default 0.5; values <= 0
                            select the default) */
  double imp_tol;        /* -imp_tol: relative residual tolerance of the implicit momentum
                            solve (imp_free_tol, main.c:212; values <= 0 select 1e-4) */
  double roughness;      /* -roughness (roughness_size, rough_set, main.c:2073): > 0 makes the
                            wall model of body 0 the rough-wall log law
                            wall_function_roughness_loglaw (wallfunction.c:71, ibm.c:3469) */
  double reserved_d[5];
} vfs_config;

/* Field identifiers for vfs_set_field / vfs_get_field (dof in brackets). */
enum {
  VFS_UCONT = 0,    /* [3] contravariant face fluxes Ucont (variables.h:561) */
  VFS_UCAT = 1,     /* [3] Cartesian centre velocity Ucat (variables.h:562) */
  VFS_P = 2,        /* [1] pressure P */
  VFS_PHI = 3,      /* [1] pressure correction Phi */
  VFS_NVERT = 4,    /* [1] IB flags 0/1/3 as doubles (stored as uint8 on the device) */
  VFS_NU_T = 5,     /* [1] eddy viscosity lNu_t */
  VFS_RHS = 6,      /* [3] momentum right-hand side (Formfunction_2 accumulates here) */
  VFS_DP = 7,       /* [3] pressure gradient dP (Pressure_Gradient output) */
  VFS_UCONT_O = 8,  /* [3] Ucont of the previous time step */
  VFS_UCAT_O = 9,   /* [3] lUcat_old (slip-wall ghost source) */
  VFS_B = 10,       /* [1] Poisson right-hand side on the grid (PoissonRHS2 output) */
  VFS_CENT = 11,    /* [3] cell centres */
  VFS_CSI = 12, VFS_ETA = 13, VFS_ZET = 14, VFS_AJ = 15,     /* centre metrics */
  VFS_ICSI = 16, VFS_IETA = 17, VFS_IZET = 18, VFS_IAJ = 19, /* i-face metrics */
  VFS_JCSI = 20, VFS_JETA = 21, VFS_JZET = 22, VFS_JAJ = 23, /* j-face metrics */
  VFS_KCSI = 24, VFS_KETA = 25, VFS_KZET = 26, VFS_KAJ = 27, /* k-face metrics */
  VFS_CS = 28,      /* [1] dynamic Smagorinsky coefficient lCs */
  VFS_USTAR = 29,   /* [1] friction velocity at IB nodes (lUstar, ibm_interpolation_advanced) */
  VFS_RHS_O = 30,   /* [3] RHS_o: Formfunction_2 of the step's initial state (implicit = 4,
                       solvers.c:1284-1286) */
  VFS_NFIELDS = 31
};

/* Scalars for vfs_set_scalar / vfs_get_scalar. */
enum {
  VFS_S_MEAN_K_FLUX = 0,  /* user->mean_k_flux (Calc_k_Flux, rhs2.c:1562) */
  VFS_S_MEAN_K_AREA = 1,  /* user->mean_k_area (Calc_Inlet_Area, bcs.c:216) */
  VFS_S_INLET_FLUX = 2,   /* inlet_flux global */
  VFS_S_INLET_AREA = 3,   /* inletArea (bcs.c:212) */
  VFS_S_DT = 4, VFS_S_REN = 5, VFS_S_ST = 6,
  VFS_S_TI = 7,           /* time step index ti (main.c:3534); vfs_step advances it */
  VFS_S_FLUX_IN = 8,      /* FluxInSum: inlet flux of the last InflowFlux (bcs.c:785) */
  VFS_S_FLUX_OUT = 9,     /* FluxOutSum: outlet flux before the last rescaling (bcs.c:2369) */
  VFS_S_IB_UNRESOLVED = 10, /* IB nodes whose interception search failed ("IBM Searching Fail!") */
  VFS_S_NBODIES = 11,     /* NumberOfBodies (main.c): the search of the last body (ibi =
                           * NumberOfBodies-1) marks cells a moving body has uncovered
                           * since the last step as IB nodes (ibm.c:346-357); default 1 */
  VFS_NSCALARS = 12
};

/* Poisson solver options (replaces PoissonSolver_Hypre, poisson_hypre.c:498). */
typedef struct {
  int precision;     /* 0: mixed (FP32 V-cycle inside FP64 FGMRES), 1: all-FP64, 2: FP32 inner
                        FGMRES (basis, preconditioned vectors, operator apply and V-cycle in
                        FP32) as iterative refinement: every restart cycle starts from the FP64
                        residual b - A x and ends when its estimate has fallen by 1e-5 (or at
                        `restart`), x and the stopping test stay FP64; the transposed (adjoint)
                        solve runs as 0 */
  int restart;       /* FGMRES restart length (default 30) */
  int max_iter;      /* outer iteration cap (default 200) */
  int levels;        /* multigrid levels including the finest (default 0: every level
                        the grid coarsens to) */
  int pre_smooth, post_smooth; /* zebra line Gauss-Seidel sweeps per level (default 3, 3) */
  int coarse_iters;  /* sweeps on the coarsest level (default 4) */
  int zero_guess;    /* 0 (default): start from the last solution, the VFS_PHI left by the
                        previous solve, on the unknowns, as the reference's GMRES starts from
                        the persistent Phi2 (poisson_hypre.c:571; Phi2 is created once,
                        poisson.c:280-282); the first solve after the operator is built
                        starts from 0, and one after VFS_PHI is set through vfs_set_field
                        from the values set.  1: always start from 0. */
  int graph;         /* vfs_step only: 1 runs the step as one CUDA graph, captured on the
                        first such step (and again after a set-up change) and replayed: the
                        Poisson solve's loops are conditional nodes and no kernel waits for
                        the host.  Same kernels, same results as 0 (launched one by one).
                        Steps with set-up work (the first step, a new operator, moving
                        bodies, the first two LES steps of a fresh run, a recorded tape)
                        and implicit momentum steps run launched one by one. */
  int reserved[3];
  double rtol;       /* relative residual target (default 1e-10) */
  double atol;       /* absolute residual target (default 0) */
  double reserved_d[4];
} vfs_solve_opts;

typedef struct {
  int iterations;       /* outer FGMRES iterations taken */
  int converged;        /* 1 if rtol/atol met */
  double r0, rfinal;    /* initial / final residual 2-norms */
  double ms;            /* device time of the solve */
  double reserved[4];
} vfs_solve_stats;

typedef struct {
  double max_div;       /* Divergence() maximum (main.c:1083-1090) after the step */
  double mean_k_flux;   /* Calc_k_Flux result at the start of the step */
  vfs_solve_stats poisson;
  double ms;            /* device time of the whole step */
  double reserved[4];
} vfs_step_stats;

/* ---- context ---------------------------------------------------------------- */
int vfs_create(const vfs_config *cfg, int device, vfs_ctx **out);
int vfs_destroy(vfs_ctx *ctx);
const char *vfs_last_error(const vfs_ctx *ctx);   /* ctx may be NULL: last global error */
int vfs_dims(const vfs_ctx *ctx, int *mx, int *my, int *mz);
int vfs_synchronize(vfs_ctx *ctx);
/* Kernels launched by this context since creation (a diagnostic counter). */
long long vfs_launch_count(const vfs_ctx *ctx);

/* Host <-> device copies in the reference layout (mx*my*mz*dof doubles). */
int vfs_set_field(vfs_ctx *ctx, int field, const double *host);
int vfs_get_field(vfs_ctx *ctx, int field, double *host);
int vfs_set_scalar(vfs_ctx *ctx, int which, double value);
int vfs_get_scalar(vfs_ctx *ctx, int which, double *value);
/* Device address of a field's component (SoA, mx*my*mz doubles), for zero-copy callers. */
int vfs_field_device_ptr(vfs_ctx *ctx, int field, int component, void **dptr);

/* ---- set-up -------------------------------------------------------------------- */

/* FormMetrics (metrics.c:4, NEWMETRIC) on the device from the grid.dat node coordinates:
 * x, y, z each hold IM*JM*KM doubles in grid.dat order ([k][j][i], i fastest,
 * init.c:384-437).  Fills VFS_CENT and every centre and face metric field. */
int vfs_form_metrics(vfs_ctx *ctx, const double *x, const double *y, const double *z);

/* ibm_search_advanced (ibm.c:85-587), the nvert flags of body ibi: cells whose centre lies
 * inside the closed triangulated surface become 3, the cells around them 1 (2 on ghost
 * points, as the reference leaves them), bit for bit with the reference's ray casting
 * (point_cell_advanced ibm.c:1068, randomdirection ibm.c:52, intsect_triangle
 * compgeom.c:17).  The surface is given as the reference's reader leaves it in IBMNodes
 * (ibm_io.c:582-905): n_v vertices x/y/z and n_elmt triangles of 0-based vertex indices
 * nv1/nv2/nv3.  Body 0 starts from zero flags; later bodies add to them.  Needs the cell
 * centres (vfs_form_metrics or VFS_CENT); updates VFS_NVERT.  It also builds the body's
 * IB-node list (ibm.c:347-505): for each cell marked near the surface, the nearest surface
 * point (nearestcell1 ibm.c:1366), the interception of the surface normal with the
 * neighbouring cell-centre triangles (InterceptionPoint ibm.c:1759) and the three fluid
 * cells interpolated across it; body 0 starts a new list, later bodies append. */
int vfs_ibm_search(vfs_ctx *ctx, int ibi, int n_v, const double *x, const double *y, const double *z,
                   int n_elmt, const int *nv1, const int *nv2, const int *nv3);

/* The surface velocity of body ibi's vertices (ibm->u, set by the reference's body-motion
 * routines, e.g. Elmt_Move_FSI_TRANS), which the IB-node reconstruction interpolates to
 * each node's nearest point (ibm.c:3430-3433).  Zero after every vfs_ibm_search of the
 * body (a fixed body); n_v must be the body's vertex count. */
int vfs_ibm_set_velocity(vfs_ctx *ctx, int ibi, int n_v, const double *u, const double *v, const double *w);

/* The IB-node list: returns its length; with ints/dbls, copies up to cap nodes, 14 ints
 * each (i j k, nearest triangle, interception mode, stencil i1 j1 k1 i2 j2 k2 i3 j3 k3)
 * and 8 doubles each (stencil weights cr1..cr3, surface weights cs1..cs3, d_s, d_i).
 * A negative return is -VFS_ERR_*. */
int vfs_ibm_list(vfs_ctx *ctx, int *ints, double *dbls, int cap);

/* ibm_interpolation_advanced (ibm.c:3294) for fixed bodies with the no-slip
 * reconstruction (noslip, wallfunction.c:134): IB-node Ucat = (d_s/(d_s+d_i)) x the velocity
 * interpolated at its stencil (zero next to non-fluid stencil cells), IB-node P from its
 * stencil, the face fluxes around IB nodes from the averaged Ucat, then Contra2Cart.
 * vfs_step calls it where Flow_Solver and RungeKutta do when immersed = 1. */
int vfs_ibm_interpolation(vfs_ctx *ctx);

/* ---- hot-path operators (each replaces the cited reference function) --------------- */

/* Contra2Cart / Contra2Cart_2 (rhs.c:27, rhs.c:57): Ucat from Ucont at fluid cells,
 * then the boundary ghost values of Ucat. */
int vfs_contra2cart(vfs_ctx *ctx);

/* Formfunction_2(user, Rhs, scale) (momentum.c:456): ADDS scale * RHS into VFS_RHS. */
int vfs_formfunction2(vfs_ctx *ctx, double scale);

/* Pressure_Gradient(user, dP) (momentum.c:197): writes VFS_DP. */
int vfs_pressure_gradient(vfs_ctx *ctx);

/* Compute_Smagorinsky_Constant_1(user, lUcont, lUcat) (les.c:67): dynamic Smagorinsky
 * coefficient from VFS_UCAT -> VFS_CS.  Zero while ti < 2 on a fresh run, 0.01 for les = 1,
 * else the Germano-identity least-squares value with the 3-D box test filter, clipped to
 * [0, max_cs] with the wall floor 0.001 at IB nodes and filtered once more. */
int vfs_smagorinsky_constant(vfs_ctx *ctx);

/* Compute_eddy_viscosity_LES (les.c:1135): VFS_NU_T = Cs * (1/aj)^(2/3) * |S|. */
int vfs_eddy_viscosity(vfs_ctx *ctx);

/* Calc_k_Flux (rhs2.c:1562): mean k-face flux -> VFS_S_MEAN_K_FLUX. */
int vfs_calc_k_flux(vfs_ctx *ctx, double *mean_k_flux);

/* Calc_Inlet_Area (bcs.c:216): mean fluid k-face area -> VFS_S_MEAN_K_AREA and the
 * fluid inlet-plane area -> VFS_S_INLET_AREA (k inlet or periodic k). */
int vfs_calc_inlet_area(vfs_ctx *ctx);

/* InflowFlux (bcs.c:329) for an inlet on the k = 0 face (bctype[4] = 5): inlet-plane face
 * fluxes and ghost velocities for inletprofile 2 (uniform inlet_flux/inletArea), 21
 * (Poiseuille) or 100 (the plane of vfs_set_inflow_plane, rescaled to inlet_flux);
 * inletprofile 1 gives zero inflow, as in the reference (its second profile selection,
 * bcs.c:408-466, has no branch for 1 and sets uin = 0).  FluxInSum -> VFS_S_FLUX_IN.
 * No-op without a k = 0 inlet. */
int vfs_inflow_flux(vfs_ctx *ctx);

/* The inflow velocity plane of inletprofile 100 (user->ucont_plane filled by
 * read_inflow_section, rhs2.c:701): my*mx Cartesian {u,v,w} triples, [j][i] with i fastest,
 * the layout of one record of the reference's inflow files. */
int vfs_set_inflow_plane(vfs_ctx *ctx, const double *plane);

/* FormBCS (bcs.c:1841) for the boundary codes accepted by vfs_create: Contra2Cart; with
 * outflow_scale and an outlet on the k+ face (bctype[5] = 4), the last interior k-face
 * fluxes shifted so the outflow equals VFS_S_FLUX_IN (bcs.c:2285-2417); zero normal flux
 * through no-slip/free-slip i/j walls; Contra2Cart; Ucat = 0 on box edges.  RungeKutta
 * calls it with outflow_scale 0 before the stages and 1 after them (rhs.c:1598, 1670). */
int vfs_form_bcs(vfs_ctx *ctx, int outflow_scale);

/* IB_BC (momentum.c:1982): with immersed = 1 the face fluxes around IB nodes from the
 * averaged Ucat; zero normal flux on free-slip faces, periodic normal flux on ghost
 * planes. */
int vfs_ib_bc(vfs_ctx *ctx);

/* VolumeFlux: for immersed = 0 VolumeFlux(user, Ucont, ...) (poisson.c:3306), zero flux
 * through every interior face between a fluid and a non-fluid cell (blocked-cell bodies);
 * for immersed = 1 VolumeFlux(user, &flux, &area, 0) (poisson.c:3570), the net flux through
 * the fluid/IB-node faces spread back over them in proportion to their area. */
int vfs_volume_flux(vfs_ctx *ctx);

/* RungeKutta (rhs.c:1578), explicit momentum predictor, 4 stages: InflowFlux, FormBCS,
 * the stages, FormBCS with the outlet rescaling. */
int vfs_runge_kutta(vfs_ctx *ctx);

/* PoissonLHSNew (poisson.c:971): builds the 19-point operator of the fluid cells and
 * the multigrid hierarchy.  Call again whenever VFS_NVERT or the metrics change. */
int vfs_poisson_lhs(vfs_ctx *ctx);

/* PoissonRHS2 (poisson.c:1774) with the volume-weighted compatibility shift of
 * Remove_Nullspace_Scale (poisson_hypre.c:110): writes VFS_B. */
int vfs_poisson_rhs(vfs_ctx *ctx);

/* Poisson solve for VFS_PHI (replaces PoissonSolver_Hypre, poisson_hypre.c:498,
 * including Remove_Nullspace poisson_hypre.c:194 and Convert_Phi2_Phi poisson.c:92).
 * Starts from the previous solution unless opts->zero_guess (see vfs_solve_opts). */
int vfs_poisson_solve(vfs_ctx *ctx, const vfs_solve_opts *opts, vfs_solve_stats *stats);

/* y = A x with the operator of vfs_poisson_lhs, on the grid layout (mx*my*mz doubles;
 * entries of non-fluid cells are ignored in x and returned as 0 in y). */
int vfs_poisson_apply(vfs_ctx *ctx, const double *x_host, double *y_host);

/* UpdatePressure (poisson.c:3144): P += Phi at fluid cells, P = 0 where nvert > 1.1. */
int vfs_update_pressure(vfs_ctx *ctx);

/* Projection (poisson.c:2707): Ucont -= dt*st*G(Phi) on fluid faces, periodic copies,
 * then Contra2Cart. */
int vfs_projection(vfs_ctx *ctx);

/* Divergence (main.c:1047): max |div Ucont * aj| over cells with an all-fluid 7-point
 * neighbourhood. */
int vfs_divergence(vfs_ctx *ctx, double *max_div);

/* One projection time step: Calc_k_Flux, the eddy viscosity when les != 0
 * (Contra2Cart, Compute_Smagorinsky_Constant_1 every dynamic_freq steps,
 * Compute_eddy_viscosity_LES), Pressure_Gradient, RungeKutta (with implicit = 4: RHS_o and
 * vfs_implicit_momentum instead, solvers.c:1282-1289), Poisson (RHS, solve),
 * UpdatePressure, Projection, Divergence (solvers.c:562-1390); then ti advances by one.
 * opts may be NULL for the defaults. */
int vfs_step(vfs_ctx *ctx, const vfs_solve_opts *opts, vfs_step_stats *stats);

/* ---- implicit momentum (implicit = 4) ----------------------------------------------- */

typedef struct {
  int newton_iterations;  /* nonlinear iterations taken */
  int krylov_iterations;  /* GMRES iterations over all of them */
  int converged;          /* 1 if |F| <= imp_tol |F0| */
  int reserved_i;
  double f0, ffinal;      /* 2-norms of the residual at the start and the end */
  double reserved[4];
} vfs_newton_stats;

/* FormFunction_SNES (momentum.c:2197-2300) at the current VFS_UCONT: the wall faces of
 * Ucont take zero normal flux, Ucat follows (Contra2Cart, IB_BC), and VFS_RHS receives
 *   F = -Ucont/dt + Ucont_o/dt + 0.5 Formfunction_2(Ucont) + 0.5 RHS_o - dP
 * (the Crank-Nicolson form: time_coeff() = 1 without level set or RANS, poisson.c:17).
 * Reads VFS_UCONT_O, VFS_RHS_O, VFS_DP, VFS_NU_T; writes VFS_UCONT (its wall faces),
 * VFS_UCAT and VFS_RHS. */
int vfs_implicit_residual(vfs_ctx *ctx);

/* Implicit_MatrixFree (implicitsolver.c:4196-4420): InflowFlux and FormBCS without the
 * outlet rescaling, then Ucont solving F(Ucont) = 0 to |F| <= imp_tol |F0| by Newton's
 * method with matrix-free Jacobian products (J v = (F(U + h v) - F(U)) / h, h by the
 * Walker-Pernice rule), unpreconditioned GMRES(30) and a backtracking line search, all on
 * the device; then the reference's boundary fix-ups of the solution, FormBCS with the
 * outlet rescaling and, with immersed bodies after the first step, the IB-node
 * reconstruction.  The reference hands F to PETSc's SNES (trust region, Eisenstat-Walker
 * forcing); its iterates differ, the solution satisfies the same equations to the same
 * tolerance.  vfs_step runs this in place of RungeKutta when implicit = 4, after forming
 * VFS_RHS_O. */
int vfs_implicit_momentum(vfs_ctx *ctx, vfs_newton_stats *stats);

/* ---- restart files ---------------------------------------------------------------- */

/* One vector in PETSc's binary Vec format, as the reference's restart files hold it
 * (PetscViewerBinaryOpen + VecView / VecLoadIntoVector, main.c:777-780, 401-404): the
 * class id 1211214 and the length as 32-bit big-endian integers, then n big-endian
 * doubles.  values: host array of n doubles (a DA vector in its natural ordering, the
 * layout of vfs_get_field).  Reading fails with VFS_ERR_INVALID when the file's length
 * is not n.  Host-only: no context or GPU needed. */
int vfs_petsc_vec_write(const char *path, const double *values, long long n);
int vfs_petsc_vec_read(const char *path, double *values, long long n);

/* Ucont_P_Binary_Output (main.c:765-1035): writes <dir>/vfield%06d_%1d.dat (Ucont),
 * ufield (Ucat), pfield (P), nvfield (nvert) and, with les on, cs_ (the Smagorinsky
 * coefficient), for time step ti and block `block` (0-9), in the reference's format. */
int vfs_restart_write(vfs_ctx *ctx, const char *dir, int ti, int block);

/* Ucont_P_Binary_Input (main.c:394-760): loads Ucont (and Ucont_o), P, Ucat (and the
 * old Ucat of the slip walls), nvert when immersed = 1 (the reference's Nvert_o; classify
 * the bodies again with vfs_ibm_search for the current flags) and, with les on, Cs (0
 * when its file is absent); the run continues as a restart at time step ti (tistart = ti,
 * the first step repeats the set-up of ti == tistart). */
int vfs_restart_read(vfs_ctx *ctx, const char *dir, int ti, int block);

/* ---- grid.dat ---------------------------------------------------------------------- */

/* The grid reader of MG_Initial (init.c:313-440).  format: 0 grid.dat in ASCII, 1 grid.dat
 * in binary (the reference's -binary 1: native ints and doubles), 2 xyz.dat (-xyz 1: one
 * block of a tensor-product grid).  vfs_grid_read returns the node counts of block `block`
 * (0-based) in *IM, *JM, *KM and, when x is not NULL, its IM*JM*KM node coordinates
 * ([k][j][i], i fastest; the layout of vfs_form_metrics) in x, y, z, each value v stored as
 * v / cl * L_dim as the reference stores it (cl: -chact_leng, L_dim: both 1 for none); call
 * it with x = NULL first to size the arrays.  vfs_grid_write writes one block in the same
 * format (17 significant digits in the text forms); xyz.dat takes the tensor axes from the
 * grid and fails with VFS_ERR_INVALID when the grid is not a tensor product.  Host-only:
 * no context or GPU needed. */
int vfs_grid_read(const char *path, int format, int block, double cl, double L_dim, int *IM, int *JM, int *KM,
                  double *x, double *y, double *z);
int vfs_grid_write(const char *path, int format, int IM, int JM, int KM, const double *x, const double *y,
                   const double *z);

/* ---- allocation-free variant ---------------------------------------------------- */

/* Largest grid (DA points (IM+1)*(JM+1)*(KM+1)) vfs_contra2cart_noalloc accepts, and the
 * size of the static device scratch it keeps for that limit (26 bytes per point). */
#define VFS_NOALLOC_MAX_POINTS (1 << 21)
#define VFS_NOALLOC_SCRATCH_BYTES (26ull * (1ull << 21) + 256ull)

/* Contra2Cart for callers that cannot allocate device memory, for instance a solver
 * embedded in a framework that owns every device allocation through its own pool, or a
 * process whose device memory is fixed before the solver starts.  No counterpart in the
 * reference: it is the same computation as vfs_contra2cart of this library, on
 * caller-owned device buffers, without a context and without any allocation.
 *
 * All arrays are device pointers on the current device, in the reference's DA layout
 * with vector fields as three consecutive component blocks (x block, y block, z block,
 * each (IM+1)*(JM+1)*(KM+1) doubles):  ucont [3N, its periodic ghost values are
 * refreshed in place, as the reference does on lUcont], csi/eta/zet [3N each], nvert
 * [N, integer values], ucat_old [3N, slip-wall ghost source], ucat [3N, in/out: cells
 * with nvert >= 0.1 keep their value].  stream is a cudaStream_t (NULL: default).
 *
 * Scratch lives in one static device array of VFS_NOALLOC_SCRATCH_BYTES (about 52 MB)
 * that every GPU loading the library holds until the process exits.  Grids above
 * VFS_NOALLOC_MAX_POINTS are rejected with VFS_ERR_INVALID.  Every call looks up the
 * array's device address (cudaGetSymbolAddress) in the current device's context.  Every
 * call shares the array: serialise calls on one stream; calls that overlap on the GPU
 * (two streams, or two host threads) race.  The call reads back an error word and
 * synchronises its stream before returning, so it cannot be captured into a CUDA graph.
 * Nothing is allocated or freed. */
int vfs_contra2cart_noalloc(const vfs_config *cfg, double *ucont, const double *csi, const double *eta,
                            const double *zet, const double *nvert, const double *ucat_old, double *ucat,
                            void *stream);

/* ---- diagnostics ----------------------------------------------------------------- */

/* The context's CUDA stream (cudaStream_t), so callers can record events on it. */
int vfs_get_stream(vfs_ctx *ctx, void **stream);

/* Launch one kernel of the path `reps` times on the context's stream without a host
 * synchronisation, on the context's current fields: 0 face fluxes of Formfunction_2
 * (three-kernel form), 1 its Fp, 2 its RHS projection, 3 FP64 Poisson operator apply,
 * 4 FP32 fine-level zebra line sweep (both colours), 5 the same in FP64, 6 Projection,
 * 7 Formfunction_2 as three kernels (0-2), 8 Formfunction_2 as a step runs it, 9 one
 * multigrid V-cycle of the preconditioner (FP32) applied to VFS_B, 10 the same in FP64,
 * 11 Formfunction_2 as one k-marching kernel, 12 Pressure_Gradient, 13 UpdatePressure and
 * Projection as one kernel, 14 the Contra2Cart interior kernel that also forms the block
 * maxima of Divergence.  Kernels 7, 8 and 11 add into RHS as vfs_formfunction2 does.  For
 * timing only. */
int vfs_run_kernel(vfs_ctx *ctx, int which, int reps);

/* ------------------------------------------------------------------ adjoint
 * Tangent-linear and discrete adjoint of a window of vfs_step calls (implicit = 0,
 * les = 0; the boundary codes of vfs_create; an inlet only with inletprofile 100).  The
 * reference has no adjoint: these entry points differentiate this library's own step,
 * which reproduces the reference's Flow_Solver step.  Each call leaves the context in
 * the state it had on entry. */
enum {
  VFS_OBJ_KINETIC_ENERGY = 0, /* 0.5 * sum over interior fluid cells of |Ucat|^2 / aj */
  VFS_OBJ_PRESSURE_DRAG = 1,  /* sum over k-faces between a fluid cell and a body cell
                                 (nvert > 0) of +-P(fluid)*|zet|: streamwise pressure force */
  VFS_OBJ_DRAG = 2            /* VFS_OBJ_PRESSURE_DRAG plus the viscous traction on the i- and
                                 j-faces between a fluid cell and a body cell (at rest):
                                 2/ren * |csi|^2 (|eta|^2) * aj * w of the fluid cell per face,
                                 the streamwise force of the pressure and shear stresses that
                                 Calc_forces_SI (fsi.c:5151) sums over the body surface */
};
enum {
  VFS_CTRL_INITIAL_UCONT = 0, /* the Ucont the window starts from (DA layout, 3 per point) */
  VFS_CTRL_INFLOW_PLANE = 1   /* the inletprofile 100 plane (vfs_set_inflow_plane layout) */
};
typedef struct {
  int nsteps;            /* time steps in the window */
  int checkpoint_every;  /* steps between stored states; <= 0: ceil(sqrt(nsteps)) */
  int objective;         /* VFS_OBJ_* of the final state */
  int control;           /* VFS_CTRL_* */
  int reserved[4];
  vfs_solve_opts solve;  /* forward, tangent and adjoint Poisson solves */
} vfs_adjoint_opts;

typedef struct {
  double J;              /* objective */
  double ms_forward;     /* forward sweep that stores the checkpoints */
  double ms_adjoint;     /* reverse sweep: segment recomputation and adjoint steps */
  int recomputed_steps;
  int checkpoints;
  long long tape_bytes;  /* per-segment linearisation state held on the device */
  double poisson_iterations_forward;  /* mean FGMRES iterations of the forward steps' solves */
  double poisson_iterations_adjoint;  /* mean FGMRES iterations of the transposed solves */
  double reserved[2];
} vfs_adjoint_stats;

/* Sets up the adjoint.  The step's fixed linear operators (Contra2Cart, FormBCS tail,
 * Pressure_Gradient, VolumeFlux, Poisson right-hand side, UpdatePressure, Projection, IB_BC,
 * IB-node interpolation) are transposed by hand-written kernels, except IB_BC and the
 * IB-node interpolation of a grid with IB nodes: those two are measured here as sparse
 * matrices from the forward kernels (the others only when a test hook asks for their
 * matrices).  The tangent runs the kernels themselves.  Needs metrics and nvert (and the
 * IB-node list when immersed); a later change of nvert or of the grid needs a new context.
 * The other adjoint entry points call it when needed. */
int vfs_adjoint_setup(vfs_ctx *ctx);
/* J after opts->nsteps steps from the current state. */
int vfs_objective(vfs_ctx *ctx, const vfs_adjoint_opts *opts, double *J);
/* J and its directional derivative along dir (the control's layout) by the tangent-linear
 * steps. */
int vfs_tangent(vfs_ctx *ctx, const vfs_adjoint_opts *opts, const double *dir, double *J, double *dJ);
/* dJ/dcontrol by the adjoint steps, recomputing each checkpoint segment forward. */
int vfs_adjoint_gradient(vfs_ctx *ctx, const vfs_adjoint_opts *opts, double *grad, vfs_adjoint_stats *stats);
/* Test hooks: the slots (field, component pairs) and entry count (0 until measured) of
 * operator op (0 Contra2Cart, 1 FormBCS tail, 2 Pressure_Gradient, 3 VolumeFlux, 4 Poisson
 * RHS, 5 UpdatePressure, 6 Projection, 7 IB_BC, 8 IB-node interpolation); for vectors x and
 * y (slot-major, N per slot), L x by the operator's kernels and L^T y by the transpose the
 * adjoint sweep applies (the dot-product test <y, L x> = <L^T y, x>); and L^T y by the
 * operator's measured matrix (vfs_adjoint_op_measured, measured on first use), against
 * which the hand-written transposes are checked. */
int vfs_adjoint_op_info(vfs_ctx *ctx, int op, int *nslot, int *fields, long long *nnz);
int vfs_adjoint_op_check(vfs_ctx *ctx, int op, const double *x, const double *y, double *Lx, double *LTy);
int vfs_adjoint_op_measured(vfs_ctx *ctx, int op, const double *y, double *LTy);

#ifdef __cplusplus
}
#endif
#endif /* VFS_B200_H */
