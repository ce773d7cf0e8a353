// Implementation of the single-rank PETSc/MPI stand-in declared in petsc_shim.h.
// Test-oracle infrastructure only: it lets the reference's own hot-path sources be
// compiled unmodified into oracle/_ref.  The product library never links it.
#include "petsc_shim.h"

#include <cstdio>
#include <cstring>
#include <map>
#include <vector>
#include <sys/time.h>

static const int kSlackPlanes = 4;  // spare planes before/after the data of a DA vector

int shim_mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return (int)sizeof(int);
    case MPI_DOUBLE: return (int)sizeof(double);
    case MPI_FLOAT: return (int)sizeof(float);
    case MPI_CHAR: return 1;
    case MPI_LONG: return (int)sizeof(long);
    default: return 8;
  }
}

static int g_verbose = -1;
static bool verbose() {
  if (g_verbose < 0) g_verbose = getenv("VFS_REF_VERBOSE") ? 1 : 0;
  return g_verbose == 1;
}

// ------------------------------------------------------------------ vectors
static Vec vec_alloc(PetscInt n, DA da) {
  Vec v = (Vec)calloc(1, sizeof(struct _p_Vec));
  v->n = n;
  v->da = da;
  size_t slack = 0;
  if (da) slack = (size_t)kSlackPlanes * da->mx * da->my * da->dof;
  v->base = (double *)calloc((size_t)n + 2 * slack + 8, sizeof(double));
  v->data = v->base + slack;
  return v;
}

PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec *v) { *v = vec_alloc(n, 0); return 0; }
PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt n, PetscInt, Vec *v) { *v = vec_alloc(n, 0); return 0; }
PetscErrorCode VecCreate(MPI_Comm, Vec *v) { *v = vec_alloc(0, 0); return 0; }
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N) {
  PetscInt m = n >= 0 ? n : N;
  free(v->base);
  v->n = m;
  v->base = (double *)calloc((size_t)m + 8, sizeof(double));
  v->data = v->base;
  return 0;
}
PetscErrorCode VecSetFromOptions(Vec) { return 0; }
PetscErrorCode VecDuplicate(Vec a, Vec *b) { *b = vec_alloc(a->n, a->da); return 0; }
PetscErrorCode VecDestroy(Vec v) {
  if (!v) return 0;
  free(v->base);
  free(v->k_table);
  free(v->kj_store);
  free(v);
  return 0;
}
PetscErrorCode VecSet(Vec v, PetscScalar a) { for (PetscInt i = 0; i < v->n; i++) v->data[i] = a; return 0; }
PetscErrorCode VecCopy(Vec a, Vec b) { if (a != b) memcpy(b->data, a->data, sizeof(double) * a->n); return 0; }
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) { for (PetscInt i = 0; i < y->n; i++) y->data[i] += a * x->data[i]; return 0; }
PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x) { for (PetscInt i = 0; i < y->n; i++) y->data[i] = x->data[i] + a * y->data[i]; return 0; }
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y) { for (PetscInt i = 0; i < w->n; i++) w->data[i] = a * x->data[i] + y->data[i]; return 0; }
PetscErrorCode VecAXPBY(Vec y, PetscScalar a, PetscScalar b, Vec x) { for (PetscInt i = 0; i < y->n; i++) y->data[i] = a * x->data[i] + b * y->data[i]; return 0; }
PetscErrorCode VecScale(Vec v, PetscScalar a) { for (PetscInt i = 0; i < v->n; i++) v->data[i] *= a; return 0; }
PetscErrorCode VecShift(Vec v, PetscScalar a) { for (PetscInt i = 0; i < v->n; i++) v->data[i] += a; return 0; }
PetscErrorCode VecSum(Vec v, PetscScalar *s) { double t = 0; for (PetscInt i = 0; i < v->n; i++) t += v->data[i]; *s = t; return 0; }
PetscErrorCode VecMax(Vec v, PetscInt *idx, PetscReal *m) {
  double t = -1e300; PetscInt at = -1;
  for (PetscInt i = 0; i < v->n; i++) if (v->data[i] > t) { t = v->data[i]; at = i; }
  if (idx) *idx = at;
  *m = t;
  return 0;
}
PetscErrorCode VecMin(Vec v, PetscInt *idx, PetscReal *m) {
  double t = 1e300; PetscInt at = -1;
  for (PetscInt i = 0; i < v->n; i++) if (v->data[i] < t) { t = v->data[i]; at = i; }
  if (idx) *idx = at;
  *m = t;
  return 0;
}
PetscErrorCode VecNorm(Vec v, NormType t, PetscReal *r) {
  double s = 0;
  if (t == NORM_INFINITY) { for (PetscInt i = 0; i < v->n; i++) s = fmax(s, fabs(v->data[i])); }
  else if (t == NORM_1) { for (PetscInt i = 0; i < v->n; i++) s += fabs(v->data[i]); }
  else { for (PetscInt i = 0; i < v->n; i++) s += v->data[i] * v->data[i]; s = sqrt(s); }
  *r = s;
  return 0;
}
PetscErrorCode VecDot(Vec a, Vec b, PetscScalar *r) { double s = 0; for (PetscInt i = 0; i < a->n; i++) s += a->data[i] * b->data[i]; *r = s; return 0; }
PetscErrorCode VecPointwiseDivide(Vec w, Vec x, Vec y) { for (PetscInt i = 0; i < w->n; i++) w->data[i] = x->data[i] / y->data[i]; return 0; }
PetscErrorCode VecPointwiseMult(Vec w, Vec x, Vec y) { for (PetscInt i = 0; i < w->n; i++) w->data[i] = x->data[i] * y->data[i]; return 0; }
PetscErrorCode VecGetSize(Vec v, PetscInt *n) { *n = v->n; return 0; }
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n) { *n = v->n; return 0; }
PetscErrorCode VecGetOwnershipRange(Vec v, PetscInt *a, PetscInt *b) { if (a) *a = 0; if (b) *b = v->n; return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->data; return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar **) { return 0; }
PetscErrorCode VecGetArray3d(Vec v, PetscInt m, PetscInt n, PetscInt, PetscInt ms, PetscInt ns, PetscInt ps, PetscScalar ****a) {
  // Used only on DA vectors in the reference; build a [k][j][i] view of dof-1 data.
  PetscInt p = v->n / (m * n);
  double ***t = (double ***)malloc(sizeof(double **) * p);
  double **rows = (double **)malloc(sizeof(double *) * p * n);
  for (PetscInt k = 0; k < p; k++) {
    for (PetscInt j = 0; j < n; j++) rows[k * n + j] = v->data + ((size_t)k * n + j) * m - ms;
    t[k] = rows + k * n - ns;
  }
  *a = t - ps;
  return 0;
}
PetscErrorCode VecRestoreArray3d(Vec, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscScalar ****) { return 0; }
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar a, InsertMode mode) {
  if (i < 0 || i >= v->n) return 0;
  if (mode == ADD_VALUES) v->data[i] += a; else v->data[i] = a;
  return 0;
}
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt *ix, const PetscScalar *a, InsertMode mode) {
  for (PetscInt q = 0; q < n; q++) VecSetValue(v, ix[q], a[q], mode);
  return 0;
}
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt *ix, PetscScalar *a) {
  for (PetscInt q = 0; q < n; q++) a[q] = (ix[q] >= 0 && ix[q] < v->n) ? v->data[ix[q]] : 0.0;
  return 0;
}
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
// PETSc binary viewer for Vec (the published PETSc binary format: the Vec class id
// 1211214 and the global length as 32-bit big-endian integers, then the entries as
// big-endian doubles, a DA vector in the natural (k, j, i, component) ordering, which is
// this shim's storage order).
struct ShimBinViewer {
  FILE *f;
  int write;
};
static void put_be32(FILE *f, int v) {
  unsigned char b[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v};
  fwrite(b, 1, 4, f);
}
static int get_be32(FILE *f, int *v) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return 1;
  *v = (int)((unsigned)b[0] << 24 | (unsigned)b[1] << 16 | (unsigned)b[2] << 8 | (unsigned)b[3]);
  return 0;
}
PetscErrorCode VecView(Vec x, PetscViewer v) {
  ShimBinViewer *bv = (ShimBinViewer *)v;
  if (!bv || !bv->write) return 0;
  put_be32(bv->f, 1211214);
  put_be32(bv->f, (int)x->n);
  for (PetscInt q = 0; q < x->n; q++) {
    unsigned long long u;
    memcpy(&u, &x->data[q], 8);
    unsigned char b[8];
    for (int t = 0; t < 8; t++) b[t] = (unsigned char)(u >> (56 - 8 * t));
    fwrite(b, 1, 8, bv->f);
  }
  return 0;
}
PetscErrorCode VecLoadIntoVector(PetscViewer v, Vec x) {
  ShimBinViewer *bv = (ShimBinViewer *)v;
  if (!bv || bv->write) return 1;
  int cls = 0, n = 0;
  if (get_be32(bv->f, &cls) || get_be32(bv->f, &n) || cls != 1211214 || n != (int)x->n) return 1;
  for (PetscInt q = 0; q < x->n; q++) {
    unsigned char b[8];
    if (fread(b, 1, 8, bv->f) != 8) return 1;
    unsigned long long u = 0;
    for (int t = 0; t < 8; t++) u = (u << 8) | b[t];
    memcpy(&x->data[q], &u, 8);
  }
  return 0;
}
PetscErrorCode VecScatterCreateToAll(Vec a, VecScatter *s, Vec *b) { *s = 0; VecDuplicate(a, b); return 0; }
PetscErrorCode VecScatterCreateToZero(Vec a, VecScatter *s, Vec *b) { *s = 0; VecDuplicate(a, b); return 0; }
PetscErrorCode VecScatterBegin(VecScatter, Vec a, Vec b, InsertMode, ScatterMode m) {
  if (m == SCATTER_FORWARD) VecCopy(a, b); else VecCopy(b, a);
  return 0;
}
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterDestroy(VecScatter) { return 0; }
PetscErrorCode VecStrideScatter(Vec, PetscInt, Vec, InsertMode) { return 0; }

// ------------------------------------------------------------------ DA
PetscErrorCode DACreate3d(MPI_Comm, DAPeriodicType, DAStencilType, PetscInt M, PetscInt N,
                          PetscInt P, PetscInt, PetscInt, PetscInt, PetscInt dof, PetscInt s,
                          const PetscInt *, const PetscInt *, const PetscInt *, DA *out) {
  DA da = (DA)calloc(1, sizeof(struct _p_DA));
  da->mx = M; da->my = N; da->mz = P; da->dof = dof; da->s = s;
  *out = da;
  return 0;
}
PetscErrorCode DADestroy(DA) { return 0; }
PetscErrorCode DAGetLocalInfo(DA da, DALocalInfo *info) {
  memset(info, 0, sizeof(*info));
  info->dim = 3; info->dof = da->dof; info->sw = da->s;
  info->mx = da->mx; info->my = da->my; info->mz = da->mz;
  info->xm = da->mx; info->ym = da->my; info->zm = da->mz;
  info->gxm = da->mx; info->gym = da->my; info->gzm = da->mz;
  info->da = da;
  return 0;
}
PetscErrorCode DAGetInfo(DA da, PetscInt *dim, PetscInt *M, PetscInt *N, PetscInt *P, PetscInt *m,
                         PetscInt *n, PetscInt *p, PetscInt *dof, PetscInt *s, DAPeriodicType *wrap,
                         DAStencilType *st) {
  if (dim) *dim = 3;
  if (M) *M = da->mx;
  if (N) *N = da->my;
  if (P) *P = da->mz;
  if (m) *m = 1;
  if (n) *n = 1;
  if (p) *p = 1;
  if (dof) *dof = da->dof;
  if (s) *s = da->s;
  if (wrap) *wrap = DA_NONPERIODIC;
  if (st) *st = DA_STENCIL_BOX;
  return 0;
}
PetscErrorCode DAGetCorners(DA da, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p) {
  if (x) *x = 0; if (y) *y = 0; if (z) *z = 0;
  if (m) *m = da->mx; if (n) *n = da->my; if (p) *p = da->mz;
  return 0;
}
PetscErrorCode DAGetGhostCorners(DA da, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p) {
  return DAGetCorners(da, x, y, z, m, n, p);
}
PetscErrorCode DACreateGlobalVector(DA da, Vec *v) { *v = vec_alloc(da->mx * da->my * da->mz * da->dof, da); return 0; }
PetscErrorCode DACreateLocalVector(DA da, Vec *v) { return DACreateGlobalVector(da, v); }
PetscErrorCode DACreateNaturalVector(DA da, Vec *v) { return DACreateGlobalVector(da, v); }
PetscErrorCode DAGetLocalVector(DA da, Vec *v) { return DACreateGlobalVector(da, v); }
PetscErrorCode DARestoreLocalVector(DA, Vec *v) { VecDestroy(*v); *v = 0; return 0; }
PetscErrorCode DAGetGlobalVector(DA da, Vec *v) { return DACreateGlobalVector(da, v); }
PetscErrorCode DARestoreGlobalVector(DA, Vec *v) { VecDestroy(*v); *v = 0; return 0; }

// [k][j][i] view of a DA vector, element size = dof doubles.  Built once per vector.
PetscErrorCode DAVecGetArray(DA da, Vec v, void *out) {
  DA vda = v->da ? v->da : da;
  if (!v->k_table) {
    const PetscInt mx = vda->mx, my = vda->my, mz = vda->mz, dof = vda->dof;
    const PetscInt kp = mz + 2 * kSlackPlanes;
    char **rows = (char **)malloc(sizeof(char *) * (size_t)kp * my);
    void **ktab = (void **)malloc(sizeof(void *) * (size_t)kp);
    for (PetscInt kk = 0; kk < kp; kk++) {
      PetscInt k = kk - kSlackPlanes;
      for (PetscInt j = 0; j < my; j++)
        rows[(size_t)kk * my + j] = (char *)(v->data + (((size_t)k * my + j) * mx) * dof);
      ktab[kk] = (void *)(rows + (size_t)kk * my);
    }
    v->kj_store = rows;
    v->k_table = ktab;
  }
  *(void ***)out = v->k_table + kSlackPlanes;
  return 0;
}
PetscErrorCode DAVecRestoreArray(DA, Vec, void *) { return 0; }
PetscErrorCode DAGlobalToLocalBegin(DA, Vec g, InsertMode, Vec l) { return VecCopy(g, l); }
PetscErrorCode DAGlobalToLocalEnd(DA, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DALocalToLocalBegin(DA, Vec a, InsertMode, Vec b) { return VecCopy(a, b); }
PetscErrorCode DALocalToLocalEnd(DA, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DALocalToGlobal(DA, Vec l, InsertMode, Vec g) { return VecCopy(l, g); }
PetscErrorCode DALocalToGlobalBegin(DA, Vec l, Vec g) { return VecCopy(l, g); }
PetscErrorCode DALocalToGlobalEnd(DA, Vec, Vec) { return 0; }
PetscErrorCode DAGlobalToNaturalBegin(DA, Vec a, InsertMode, Vec b) { return VecCopy(a, b); }
PetscErrorCode DAGlobalToNaturalEnd(DA, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DANaturalToGlobalBegin(DA, Vec a, InsertMode, Vec b) { return VecCopy(a, b); }
PetscErrorCode DANaturalToGlobalEnd(DA, Vec, InsertMode, Vec) { return 0; }
PetscErrorCode DAGlobalToNaturalAllCreate(DA, VecScatter *s) { *s = 0; return 0; }
PetscErrorCode DAGetCoordinateDA(DA da, DA *cda) {
  if (!da->cda) DACreate3d(0, DA_NONPERIODIC, DA_STENCIL_BOX, da->mx, da->my, da->mz, 1, 1, 1, 3, da->s, 0, 0, 0, &da->cda);
  *cda = da->cda;
  return 0;
}
static void ensure_coords(DA da) {
  if (da->coords) return;
  DA cda;
  DAGetCoordinateDA(da, &cda);
  DACreateGlobalVector(cda, &da->coords);
  DACreateGlobalVector(cda, &da->gcoords);
}
PetscErrorCode DASetUniformCoordinates(DA da, PetscReal x0, PetscReal x1, PetscReal y0, PetscReal y1, PetscReal z0, PetscReal z1) {
  ensure_coords(da);
  const PetscInt mx = da->mx, my = da->my, mz = da->mz;
  for (PetscInt k = 0; k < mz; k++)
    for (PetscInt j = 0; j < my; j++)
      for (PetscInt i = 0; i < mx; i++) {
        double *c = da->coords->data + 3 * (((size_t)k * my + j) * mx + i);
        c[0] = x0 + (mx > 1 ? (x1 - x0) * i / (mx - 1) : 0);
        c[1] = y0 + (my > 1 ? (y1 - y0) * j / (my - 1) : 0);
        c[2] = z0 + (mz > 1 ? (z1 - z0) * k / (mz - 1) : 0);
      }
  VecCopy(da->coords, da->gcoords);
  return 0;
}
PetscErrorCode DAGetCoordinates(DA da, Vec *v) { ensure_coords(da); *v = da->coords; return 0; }
PetscErrorCode DAGetGhostedCoordinates(DA da, Vec *v) { ensure_coords(da); *v = da->gcoords; return 0; }
PetscErrorCode DAGetGlobalIndices(DA da, PetscInt *n, PetscInt **idx) {
  const PetscInt N = da->mx * da->my * da->mz;
  if (!da->gidx) {
    da->gidx = (PetscInt *)malloc(sizeof(PetscInt) * N);
    for (PetscInt q = 0; q < N; q++) da->gidx[q] = q;
  }
  if (n) *n = N;
  *idx = da->gidx;
  return 0;
}
PetscErrorCode DAGetAO(DA, AO *ao) { *ao = 0; return 0; }
PetscErrorCode DAGetMatrix(DA, MatType, Mat *m) { return MatCreate(0, m); }
PetscErrorCode DAGetInterpolation(DA, DA, Mat *m, Vec *v) { MatCreate(0, m); if (v) *v = 0; return 0; }

// ------------------------------------------------------------------ Mat (row-map recorder)
typedef std::vector<std::map<int, double> > RowMap;
static RowMap &rows_of(Mat A) {
  if (!A->rows) A->rows = new RowMap();
  return *(RowMap *)A->rows;
}
PetscErrorCode MatCreate(MPI_Comm, Mat *A) { *A = (Mat)calloc(1, sizeof(struct _p_Mat)); return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt, PetscInt) {
  A->m = m; A->n = n;
  rows_of(A).assign(m > 0 ? m : 0, std::map<int, double>());
  return 0;
}
PetscErrorCode MatSetType(Mat, MatType) { return 0; }
PetscErrorCode MatSetFromOptions(Mat) { return 0; }
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt *, PetscInt, const PetscInt *) { return 0; }
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt *) { return 0; }
PetscErrorCode MatCreateSeqAIJ(MPI_Comm c, PetscInt m, PetscInt n, PetscInt, const PetscInt *, Mat *A) {
  MatCreate(c, A); return MatSetSizes(*A, m, n, m, n);
}
PetscErrorCode MatCreateMPIAIJ(MPI_Comm c, PetscInt m, PetscInt n, PetscInt, PetscInt, PetscInt, const PetscInt *, PetscInt, const PetscInt *, Mat *A) {
  MatCreate(c, A); return MatSetSizes(*A, m, n, m, n);
}
PetscErrorCode MatZeroEntries(Mat A) { for (auto &r : rows_of(A)) r.clear(); return 0; }
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt *ir, PetscInt n, const PetscInt *ic, const PetscScalar *v, InsertMode mode) {
  RowMap &R = rows_of(A);
  for (PetscInt a = 0; a < m; a++) {
    if (ir[a] < 0) continue;
    if ((size_t)ir[a] >= R.size()) R.resize(ir[a] + 1);
    for (PetscInt b = 0; b < n; b++) {
      if (ic[b] < 0) continue;
      if (mode == ADD_VALUES) R[ir[a]][ic[b]] += v[a * n + b];
      else R[ir[a]][ic[b]] = v[a * n + b];
    }
  }
  return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  RowMap &R = rows_of(A);
  for (size_t r = 0; r < R.size() && (PetscInt)r < y->n; r++) {
    double s = 0;
    for (auto &e : R[r]) s += e.second * x->data[e.first];
    y->data[r] = s;
  }
  return 0;
}
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z) {
  Vec t; VecDuplicate(z, &t); MatMult(A, x, t); VecWAXPY(z, 1.0, y, t); VecDestroy(t); return 0;
}
PetscErrorCode MatDestroy(Mat A) { if (!A) return 0; delete (RowMap *)A->rows; free(A); return 0; }
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt *a, PetscInt *b) { if (a) *a = 0; if (b) *b = (PetscInt)rows_of(A).size(); return 0; }
static std::vector<int> g_row_cols;
static std::vector<double> g_row_vals;
PetscErrorCode MatGetRow(Mat A, PetscInt r, PetscInt *nc, const PetscInt **cols, const PetscScalar **vals) {
  RowMap &R = rows_of(A);
  g_row_cols.clear(); g_row_vals.clear();
  for (auto &e : R[r]) { g_row_cols.push_back(e.first); g_row_vals.push_back(e.second); }
  *nc = (PetscInt)g_row_cols.size();
  if (cols) *cols = g_row_cols.data();
  if (vals) *vals = g_row_vals.data();
  return 0;
}
PetscErrorCode MatRestoreRow(Mat, PetscInt, PetscInt *, const PetscInt **, const PetscScalar **) { return 0; }
PetscErrorCode MatCreateShell(MPI_Comm c, PetscInt m, PetscInt n, PetscInt, PetscInt, void *ctx, Mat *A) {
  MatCreate(c, A); (*A)->m = m; (*A)->n = n; (*A)->shell_ctx = ctx; return 0;
}
PetscErrorCode MatShellSetOperation(Mat, MatOperation, void (*)(void)) { return 0; }
PetscErrorCode MatShellGetContext(Mat A, void *ctx) { *(void **)ctx = A->shell_ctx; return 0; }
PetscErrorCode MatGetVecs(Mat A, Vec *r, Vec *l) {
  if (r) VecCreateSeq(0, A->n, r);
  if (l) VecCreateSeq(0, A->m, l);
  return 0;
}
PetscErrorCode MatNullSpaceCreate(MPI_Comm, PetscTruth, PetscInt, const Vec *, MatNullSpace *s) { *s = 0; return 0; }
PetscErrorCode MatNullSpaceDestroy(MatNullSpace) { return 0; }
PetscErrorCode MatNullSpaceRemove(MatNullSpace, Vec, Vec *) { return 0; }
PetscErrorCode MatNullSpaceSetFunction(MatNullSpace, PetscErrorCode (*)(Vec, void *), void *) { return 0; }
PetscErrorCode MatCreateSNESMF(SNES, Mat *A) { return MatCreate(0, A); }
PetscErrorCode MatMFFDComputeJacobian(SNES, Vec, Mat *, Mat *, MatStructure *, void *) { return 0; }
PetscErrorCode MatView(Mat, PetscViewer) { return 0; }

extern "C" long shim_mat_to_csr(Mat A, int *row_ptr, int *col, double *val, int *m_out) {
  RowMap &R = rows_of(A);
  long nnz = 0;
  if (row_ptr) row_ptr[0] = 0;
  for (size_t r = 0; r < R.size(); r++) {
    for (auto &e : R[r]) {
      if (col) col[nnz] = e.first;
      if (val) val[nnz] = e.second;
      nnz++;
    }
    if (row_ptr) row_ptr[r + 1] = (int)nnz;
  }
  if (m_out) *m_out = (int)R.size();
  return nnz;
}

// ------------------------------------------------------------------ misc
PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
PetscErrorCode PetscPrintf(MPI_Comm, const char *fmt, ...) {
  if (!verbose()) return 0;
  va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap); return 0;
}
PetscErrorCode PetscFPrintf(MPI_Comm, FILE *f, const char *fmt, ...) {
  if (!verbose() || !f) return 0;
  va_list ap; va_start(ap, fmt); vfprintf(f, fmt, ap); va_end(ap); return 0;
}
PetscErrorCode PetscSynchronizedPrintf(MPI_Comm, const char *fmt, ...) {
  if (!verbose()) return 0;
  va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap); return 0;
}
PetscErrorCode PetscSynchronizedFlush(MPI_Comm) { return 0; }
PetscErrorCode PetscGetTime(PetscLogDouble *t) {
  struct timeval tv; gettimeofday(&tv, 0); *t = tv.tv_sec + 1e-6 * tv.tv_usec; return 0;
}
PetscErrorCode PetscBarrier(void *) { return 0; }
PetscErrorCode PetscGlobalSum(const PetscReal *a, PetscReal *b, MPI_Comm) { *b = *a; return 0; }
PetscErrorCode PetscGlobalMax(const PetscReal *a, PetscReal *b, MPI_Comm) { *b = *a; return 0; }
PetscErrorCode PetscGlobalMin(const PetscReal *a, PetscReal *b, MPI_Comm) { *b = *a; return 0; }
PetscErrorCode PetscOptionsGetInt(const char *, const char *, PetscInt *, PetscTruth *f) { if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetReal(const char *, const char *, PetscReal *, PetscTruth *f) { if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetTruth(const char *, const char *, PetscTruth *, PetscTruth *f) { if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetString(const char *, const char *, char *, size_t, PetscTruth *f) { if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetIntArray(const char *, const char *, PetscInt *, PetscInt *n, PetscTruth *f) { if (n) *n = 0; if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetRealArray(const char *, const char *, PetscReal *, PetscInt *n, PetscTruth *f) { if (n) *n = 0; if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsHasName(const char *, const char *, PetscTruth *f) { if (f) *f = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsInsertString(const char *) { return 0; }
PetscErrorCode PetscOptionsInsertFile(MPI_Comm, const char *, PetscTruth) { return 0; }
PetscErrorCode PetscOptionsClearValue(const char *) { return 0; }
PetscErrorCode PetscOptionsSetValue(const char *, const char *) { return 0; }
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm, const char *name, PetscFileMode mode, PetscViewer *v) {
  FILE *f = fopen(name, mode == FILE_MODE_READ ? "rb" : "wb");
  if (!f) { *v = 0; return 1; }
  ShimBinViewer *bv = new ShimBinViewer;
  bv->f = f;
  bv->write = mode != FILE_MODE_READ;
  *v = bv;
  return 0;
}
PetscErrorCode PetscViewerDestroy(PetscViewer v) {
  ShimBinViewer *bv = (ShimBinViewer *)v;
  if (bv) { fclose(bv->f); delete bv; }
  return 0;
}

// ------------------------------------------------------------------ HYPRE IJ vectors
struct ShimIJ { int lo, hi; std::vector<double> v; };
int HYPRE_IJVectorCreate(MPI_Comm, int lower, int upper, HYPRE_IJVector *v) {
  ShimIJ *p = new ShimIJ();
  p->lo = lower; p->hi = upper;
  p->v.assign(upper >= lower ? upper - lower + 1 : 0, 0.0);
  *v = p;
  return 0;
}
int HYPRE_IJVectorDestroy(HYPRE_IJVector v) { delete (ShimIJ *)v; return 0; }
int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, int) { return 0; }
int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
int HYPRE_IJVectorSetValues(HYPRE_IJVector v, int n, const int *idx, const double *vals) {
  ShimIJ *p = (ShimIJ *)v;
  for (int q = 0; q < n; q++) {
    int r = idx[q] - p->lo;
    if (r >= 0 && r < (int)p->v.size()) p->v[r] = vals[q];
  }
  return 0;
}
int HYPRE_IJVectorAddToValues(HYPRE_IJVector v, int n, const int *idx, const double *vals) {
  ShimIJ *p = (ShimIJ *)v;
  for (int q = 0; q < n; q++) {
    int r = idx[q] - p->lo;
    if (r >= 0 && r < (int)p->v.size()) p->v[r] += vals[q];
  }
  return 0;
}
int HYPRE_IJVectorGetValues(HYPRE_IJVector v, int n, const int *idx, double *vals) {
  ShimIJ *p = (ShimIJ *)v;
  for (int q = 0; q < n; q++) {
    int r = idx[q] - p->lo;
    vals[q] = (r >= 0 && r < (int)p->v.size()) ? p->v[r] : 0.0;
  }
  return 0;
}
int HYPRE_IJVectorAssemble(HYPRE_IJVector) { return 0; }
int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **o) { *o = v; return 0; }
extern "C" double *shim_ij_data(HYPRE_IJVector v, int *n) {
  ShimIJ *p = (ShimIJ *)v;
  *n = (int)p->v.size();
  return p->v.data();
}

// Called by the generated stubs of reference functions that live in sources the oracle
// does not compile; reaching one means the oracle driver strayed off the hot path.
extern "C" void shim_unresolved(const char *name) {
  fprintf(stderr, "oracle/_ref: call to a reference function outside the compiled hot path: %s\n", name);
  abort();
}
