// Tangent-linear and discrete adjoint of the projection time step (implicit = 0,
// les = 0): the linearisation of step_core (vfs_step) about a recorded forward state,
// its transpose, and a checkpoint-and-recompute driver over a window of time steps.
//
// Every operator of the step that is linear with coefficients fixed by the grid, nvert
// and the boundary codes (Contra2Cart, the FormBCS wall/edge tail, Pressure_Gradient
// without its flux forcing, the blocked-cell VolumeFlux, the local Poisson right-hand
// side, UpdatePressure, Projection, IB_BC, the IB-node interpolation) is also taken as a
// sparse matrix measured from the forward kernels themselves: the operator is applied to
// coloured unit vectors (ColourMap below), each output is decoded to the one input of that
// colour it depends on with two index-weighted probes, and a conflict (two inputs of one
// colour reaching one output) is an error.  The matrix is therefore the forward code's,
// branch for branch.  The adjoint sweep applies the transposes of the boundary operators
// (Contra2Cart, the FormBCS tail, IB_BC, the IB-node interpolation) by these matrices; the
// stencils of the projection step (Pressure_Gradient, VolumeFlux, the Poisson right-hand
// side, UpdatePressure, Projection) by hand-written gather kernels (vfs_adjoint_stencil.cu),
// which the tests check against the measured matrices.
//
// Hand-written as well: Formfunction_2 with the RK stage update (vfs_momentum.cu), the
// global couplings (k-flux forcing, inflow rescaling, outlet rescaling, the null-space
// shift of the Poisson right-hand side, the immersed VolumeFlux correction), and the
// Poisson solve (tangent: the forward solver on the tangent right-hand side; adjoint:
// FGMRES on the transposed operator, right-hand side made mean-free on the unknowns).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include <cub/cub.cuh>

#include "vfs_internal.cuh"

namespace vfs {

// ---------------------------------------------------------------- linear operators
struct Slot { int field, comp; };
constexpr int kMaxSlots = 10;
struct SlotPtrs { double *p[kMaxSlots]; };

// A measured operator: its slots, the forward function (the tangent runs it on the
// tangent fields), and the transpose of its matrix.
struct LinOp {
  int nslot = 0;
  Slot slot[kMaxSlots];
  std::function<int(Ctx *)> fn;
  long long nnz = 0;
  // The transpose in sliced ELLPACK (slices of 32 rows; entry k of row 32 s + l at
  // off[s] + 32 k + l): a warp reads its slice's columns and values coalesced.  Columns
  // index the slots gathered end to end; padding points at a zero past them.
  long long nslice = 0;
  long long *off = nullptr; int *col = nullptr; double *val = nullptr;
};

enum { OP_C2C = 0, OP_FBT, OP_PG, OP_VF, OP_PRL, OP_UP, OP_PJ, OP_IBBC, OP_IBM, OP_N };

// Banks of tangent (0) and adjoint (1) fields, indexed like the forward fields.
enum { TAN = 0, ADJ = 1 };

struct Adjoint {
  LinOp op[OP_N];
  bool built = false;
  double *bank[2][VFS_NFIELDS][3] = {};
  double *pu[2][3] = {};            // tangent / adjoint of the RK base state pUcont
  double *xcat = nullptr;           // SpMV input: the slots end to end, then zeros (padding)
  double *lface[3][6] = {};         // adjoint of the face fluxes: dir x (div xyz, visc xyz)
  double *lfp[3] = {};              // adjoint of Fp
  double *tface[3][6] = {};         // tangent face fluxes
  double *cz = nullptr;             // d(dP.z)/d(flux deficit) of the k-periodic forcing
  double *plane[2] = {};            // tangent / adjoint of the inflow plane (3*mx*my)
  std::vector<StepTape> tapes;      // one per step of the recompute segment
  double *ckpt = nullptr;           // checkpoints of the state
  int nckpt = 0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // sweep timing (the step and the solver use the context's)
  long long it_fwd = 0, n_fwd = 0, it_adj = 0, n_adj = 0;  // Poisson iterations and solves
};

static int grow(Ctx *c, double **p, size_t n) {
  if (*p) return VFS_OK;
  if (cudaMalloc(p, sizeof(double) * n) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "adjoint: device allocation failed");
  cudaMemsetAsync(*p, 0, sizeof(double) * n, c->stream);
  return VFS_OK;
}

static double *bankp(Ctx *c, int b, int f, int q) { return c->adj->bank[b][f][q]; }
static V3 bank3(Ctx *c, int b, int f) {
  return V3{c->adj->bank[b][f][0], c->adj->bank[b][f][1], c->adj->bank[b][f][2]};
}

static int ensure_banks(Ctx *c) {
  Adjoint &A = *c->adj;
  const size_t N = c->g.N;
  const int fl[7] = {VFS_UCONT, VFS_UCAT, VFS_P, VFS_UCAT_O, VFS_DP, VFS_B, VFS_PHI};
  int rc;
  for (int b = 0; b < 2; b++) {
    for (int f : fl)
      for (int q = 0; q < c->dof[f]; q++)
        if ((rc = grow(c, &A.bank[b][f][q], N))) return rc;
    for (int q = 0; q < 3; q++)
      if ((rc = grow(c, &A.pu[b][q], N))) return rc;
    if ((rc = grow(c, &A.plane[b], 3 * (size_t)c->g.mx * c->g.my))) return rc;
  }
  if ((rc = grow(c, &A.xcat, kMaxSlots * N + 32))) return rc;
  for (int d = 0; d < 3; d++) {
    for (int q = 0; q < 6; q++) {
      if ((rc = grow(c, &A.lface[d][q], N))) return rc;
    }
    if ((rc = grow(c, &A.lfp[d], N))) return rc;
  }
  return grow(c, &A.cz, N);
}

static void free_op(LinOp &o) {
  cudaFree(o.off); cudaFree(o.col); cudaFree(o.val);
  o.off = nullptr; o.col = nullptr; o.val = nullptr; o.nnz = 0; o.nslice = 0;
}

static void free_tapes(Adjoint &A) {
  for (StepTape &t : A.tapes) {
    for (int s = 0; s < 4; s++)
      for (int q = 0; q < 3; q++) { cudaFree(t.uc[s][q]); cudaFree(t.uk[s][q]); }
    for (int q = 0; q < 3; q++) cudaFree(t.vfi[q]);
  }
  A.tapes.clear();
}

void adjoint_free(Ctx *c) {
  if (!c || !c->adj) return;
  Adjoint &A = *c->adj;
  for (int o = 0; o < OP_N; o++) free_op(A.op[o]);
  for (int b = 0; b < 2; b++) {
    for (int f = 0; f < VFS_NFIELDS; f++)
      for (int q = 0; q < 3; q++) cudaFree(A.bank[b][f][q]);
    for (int q = 0; q < 3; q++) cudaFree(A.pu[b][q]);
    cudaFree(A.plane[b]);
  }
  cudaFree(A.xcat);
  for (int d = 0; d < 3; d++) {
    for (int q = 0; q < 6; q++) { cudaFree(A.lface[d][q]); cudaFree(A.tface[d][q]); }
    cudaFree(A.lfp[d]);
  }
  cudaFree(A.cz);
  cudaFree(A.ckpt);
  if (A.t0) cudaEventDestroy(A.t0);
  if (A.t1) cudaEventDestroy(A.t1);
  free_tapes(A);
  delete c->adj;
  c->adj = nullptr;
}

// ---------------------------------------------------------------- tape recording
static int tape_alloc(Ctx *c, StepTape &t) {
  const size_t N = c->g.N;
  int rc;
  for (int s = 0; s < 4; s++)
    for (int q = 0; q < 3; q++) {
      if ((rc = grow(c, &t.uc[s][q], N))) return rc;
      if ((rc = grow(c, &t.uk[s][q], N))) return rc;
    }
  if (c->g.immersed)
    for (int q = 0; q < 3; q++)
      if ((rc = grow(c, &t.vfi[q], N))) return rc;
  return VFS_OK;
}

int tape_stage(Ctx *c, int stage) {
  StepTape &t = *c->tape;
  const size_t bytes = sizeof(double) * c->g.N;
  for (int q = 0; q < 3; q++) {
    cudaMemcpyAsync(t.uc[stage][q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(t.uk[stage][q], c->f[VFS_UCAT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  }
  return VFS_OK;
}

int tape_vflux(Ctx *c) {
  StepTape &t = *c->tape;
  const size_t bytes = sizeof(double) * c->g.N;
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(t.vfi[q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  return VFS_OK;
}

// ---------------------------------------------------------------- probing
// Colouring of the DA points.  Along a periodic direction of L = m-2 interior points the
// colour follows the position on the periodic circle: positions 0..L-r-1 take (position
// mod q), the last r = L mod q positions their own colours, so two interior points within
// q-1 of each other around the circle never share a colour; the two ghost planes (which
// operators read beside their periodic images) take two more colours of their own.  Other
// directions take (index mod q).  Any two inputs of an operator whose stencil spans at
// most q-1 points per direction therefore differ in colour.
struct ColourMap {
  int q, m[3], per[3], nc[3];
  __host__ __device__ int dim(int d, int i) const {
    if (!per[d]) return i % q;
    const int L = m[d] - 2, rem = L % q, main = L - rem;
    if (i == 0) return q + rem;
    if (i == m[d] - 1) return q + rem + 1;
    const int pos = i - 1;
    return pos < main ? pos % q : q + (pos - main);
  }
  __host__ __device__ int of(long long p) const {
    const int i = (int)(p % m[0]);
    const long long r = p / m[0];
    const int j = (int)(r % m[1]), k = (int)(r / m[1]);
    return dim(0, i) + nc[0] * (dim(1, j) + nc[1] * dim(2, k));
  }
  int count() const { return nc[0] * nc[1] * nc[2]; }
};

static ColourMap colour_map(const Grid &g, int q) {
  ColourMap cm;
  cm.q = q;
  cm.m[0] = g.mx; cm.m[1] = g.my; cm.m[2] = g.mz;
  cm.per[0] = g.iper; cm.per[1] = g.jper; cm.per[2] = g.kper;
  for (int d = 0; d < 3; d++) cm.nc[d] = cm.per[d] ? q + (cm.m[d] - 2) % q + 2 : q;
  return cm;
}

// Seed: value w(p) at the points of colour cc (w = 1, p+1, (p+1)^2), 0 elsewhere.
__global__ void k_probe_seed(long long N, ColourMap cm, int cc, int kind, double *x) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= N) return;
  double v = 0;
  if (cm.of(p) == cc) {
    const double w = (double)(p + 1);
    v = kind == 0 ? 1.0 : (kind == 1 ? w : w * w);
  }
  x[p] = v;
}

__global__ void k_absmax(long long n, SlotPtrs y, long long N, double *out) {
  __shared__ double sh[256];
  double m = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(y.p[t / N][t % N]));
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// Decodes the outputs of one (colour, input slot) probe: y0 (weights 1), y1 (weights p+1)
// and y2 (weights (p+1)^2, the live slot arrays).  Each non-zero output names its input n
// = y1/y0 - 1, checked against the colour and against y2/y0 = (n+1)^2.  Outputs at or
// below tiny (rounding residue of a cancelled coefficient) that fail the check are dropped.
__global__ void k_probe_decode(long long n, long long N, ColourMap cm, int cc, int s, const double *y0,
                               const double *y1, SlotPtrs y2, double tiny, int *rows, int *cols, double *vals,
                               unsigned long long *count, unsigned long long cap, int *conflicts,
                               unsigned long long *worst) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double a = y0[t];
  if (a == 0.0) return;
  const double r1 = y1[t] / a, r2 = y2.p[t / N][t % N] / a;
  const double w = rint(r1);
  const long long src = (long long)w - 1;
  bool ok = src >= 0 && src < N && fabs(r1 - w) <= 1e-6 * w && fabs(r2 - w * w) <= 1e-6 * w * w;
  if (ok) ok = cm.of(src) == cc;
  if (!ok) {
    if (fabs(a) > tiny) {
      atomicAdd(conflicts, 1);
      // the largest |output| that failed, as ordered bits of a non-negative double
      atomicMax(worst, (unsigned long long)__double_as_longlong(fabs(a)));
    }
    return;
  }
  const unsigned long long e = atomicAdd(count, 1ULL);
  if (e < cap) {
    rows[e] = (int)t;
    cols[e] = (int)(s * N + src);
    vals[e] = a;
  }
}

__global__ void k_gather_entries(long long n, const int *perm, const int *b, const double *v, int *bo, double *vo) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int s = perm[e];
  bo[e] = b[s]; vo[e] = v[s];
}
__global__ void k_iota(long long n, int *x) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e < n) x[e] = (int)e;
}
// row_ptr from sorted row indices: ptr[r] = first entry with row >= r.
__global__ void k_row_ptr(long long nnz, long long nrows, const int *sorted, int *ptr) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e > nnz) return;
  const int lo = e == 0 ? -1 : sorted[e - 1];
  const int hi = e == nnz ? (int)nrows : sorted[e];
  for (int r = lo + 1; r <= hi; r++) ptr[r] = (int)e;
}

// Sorts the entries by key a and builds the compressed form (ptr over a, idx = b, val).
static int compress(Ctx *c, long long nnz, long long nrows, const int *a, const int *b, const double *v, int **ptr,
                    int **idx, double **val) {
  int *ka_out = nullptr, *perm = nullptr, *perm_out = nullptr;
  void *tmp = nullptr;
  size_t tb = 0;
  bool ok = cudaMalloc(&ka_out, sizeof(int) * (nnz + 1)) == cudaSuccess &&
            cudaMalloc(&perm, sizeof(int) * (nnz + 1)) == cudaSuccess &&
            cudaMalloc(&perm_out, sizeof(int) * (nnz + 1)) == cudaSuccess;
  if (ok && nnz > 0) {
    c->launches++, k_iota<<<nblocks(nnz, 256), 256, 0, c->stream>>>(nnz, perm);
    cub::DeviceRadixSort::SortPairs(nullptr, tb, a, ka_out, perm, perm_out, (int)nnz, 0, 32, c->stream);
    ok = cudaMalloc(&tmp, tb) == cudaSuccess;
    if (ok) cub::DeviceRadixSort::SortPairs(tmp, tb, a, ka_out, perm, perm_out, (int)nnz, 0, 32, c->stream);
  }
  ok = ok && cudaMalloc(ptr, sizeof(int) * (nrows + 1)) == cudaSuccess &&
       cudaMalloc(idx, sizeof(int) * (nnz + 1)) == cudaSuccess && cudaMalloc(val, sizeof(double) * (nnz + 1)) == cudaSuccess;
  if (ok) {
    if (nnz > 0) c->launches++, k_gather_entries<<<nblocks(nnz, 256), 256, 0, c->stream>>>(nnz, perm_out, b, v, *idx, *val);
    c->launches++, k_row_ptr<<<nblocks(nnz + 1, 256), 256, 0, c->stream>>>(nnz, nrows, ka_out, *ptr);
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(tmp); cudaFree(perm); cudaFree(perm_out); cudaFree(ka_out);
  if (!ok) return set_err(c, VFS_ERR_CUDA, "adjoint: operator compression failed");
  return check_launch(c, "k_row_ptr");
}

// Width of each 32-row slice: its longest row, as 32 x width entries (rows past n: none).
__global__ void k_slice_width(long long n, long long nslice, const int *__restrict__ ptr, long long *w) {
  const long long sl = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (sl >= nslice) return;
  int m = 0;
  for (long long r = 32 * sl; r < 32 * sl + 32 && r < n; r++) m = max(m, ptr[r + 1] - ptr[r]);
  w[sl] = 32LL * m;
}

__global__ void k_sell_fill(long long n, long long nslice, const int *__restrict__ ptr, const int *__restrict__ idx,
                            const double *__restrict__ v, const long long *__restrict__ off, int pad, int *col,
                            double *val) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= 32 * nslice) return;
  const long long sl = r >> 5, l = r & 31;
  const int w = (int)((off[sl + 1] - off[sl]) >> 5);
  const int b = r < n ? ptr[r] : 0, len = r < n ? ptr[r + 1] - ptr[r] : 0;
  for (int k = 0; k < w; k++) {
    const long long e = off[sl] + 32LL * k + l;
    col[e] = k < len ? idx[b + k] : pad;
    val[e] = k < len ? v[b + k] : 0.0;
  }
}

// The row-compressed transpose (ptr, idx, val over n rows) in sliced ELLPACK; pad: the
// column that padding entries read (a zero).
static int to_sell(Ctx *c, long long n, const int *ptr, const int *idx, const double *v, int pad, LinOp &op) {
  const long long ns = (n + 31) / 32;
  long long *w = nullptr;
  void *tmp = nullptr;
  size_t tb = 0;
  bool ok = cudaMalloc(&w, sizeof(long long) * (ns + 1)) == cudaSuccess &&
            cudaMalloc(&op.off, sizeof(long long) * (ns + 1)) == cudaSuccess;
  if (ok) {
    cudaMemsetAsync(w + ns, 0, sizeof(long long), c->stream);
    c->launches++, k_slice_width<<<nblocks(ns, 256), 256, 0, c->stream>>>(n, ns, ptr, w);
    cub::DeviceScan::ExclusiveSum(nullptr, tb, w, op.off, (int)(ns + 1), c->stream);
    ok = cudaMalloc(&tmp, tb) == cudaSuccess;
    if (ok) cub::DeviceScan::ExclusiveSum(tmp, tb, w, op.off, (int)(ns + 1), c->stream);
  }
  long long total = 0;
  if (ok) {
    cudaMemcpyAsync(&total, op.off + ns, sizeof(long long), cudaMemcpyDeviceToHost, c->stream);
    ok = cudaStreamSynchronize(c->stream) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&op.col, sizeof(int) * (total + 1)) == cudaSuccess &&
       cudaMalloc(&op.val, sizeof(double) * (total + 1)) == cudaSuccess;
  if (ok) c->launches++, k_sell_fill<<<nblocks(32 * ns, 256), 256, 0, c->stream>>>(n, ns, ptr, idx, v, op.off, pad, op.col, op.val);
  cudaStreamSynchronize(c->stream);
  cudaFree(w); cudaFree(tmp);
  if (!ok) return set_err(c, VFS_ERR_CUDA, "adjoint: operator conversion failed");
  op.nslice = ns;
  return check_launch(c, "k_sell_fill");
}

static double host_max(Ctx *c, const double *dev) {
  double hm[256];
  cudaMemcpyAsync(hm, dev, sizeof(hm), cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  double m = 0;
  for (double v : hm) m = std::max(m, v);
  return m;
}

// Measures the matrix of the operator fn on the slots of op (see the file header).
static int probe(Ctx *c, const char *name, LinOp &op, int q, const std::function<int(Ctx *)> &fn) {
  const Grid &g = c->g;
  const long long N = g.N, n = (long long)op.nslot * N;
  const ColourMap cm = colour_map(g, q);
  const size_t bytes = sizeof(double) * N;
  int rc;
  if (kMaxSlots * N + 32 >= (1LL << 31)) return set_err(c, VFS_ERR_INVALID, "adjoint: grid too large for 32-bit indices");
  double *backup = nullptr, *y0 = nullptr, *y1 = nullptr, *amax = nullptr;
  int *rows = nullptr, *cols = nullptr, *conf = nullptr;
  double *vals = nullptr;
  unsigned long long *cnt = nullptr, *worst = nullptr;
  double gmax = 0;
  SlotPtrs live;
  for (int s = 0; s < op.nslot; s++) live.p[s] = c->f[op.slot[s].field][op.slot[s].comp];
  auto cleanup = [&]() {
    if (backup)
      for (int s = 0; s < op.nslot; s++)
        cudaMemcpyAsync(live.p[s], backup + s * N, bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(backup); cudaFree(y0); cudaFree(y1); cudaFree(amax);
    cudaFree(rows); cudaFree(cols); cudaFree(vals); cudaFree(cnt); cudaFree(conf); cudaFree(worst);
  };
  if (cudaMalloc(&backup, bytes * op.nslot) != cudaSuccess || cudaMalloc(&y0, bytes * op.nslot) != cudaSuccess ||
      cudaMalloc(&y1, bytes * op.nslot) != cudaSuccess || cudaMalloc(&amax, sizeof(double) * 256) != cudaSuccess ||
      cudaMalloc(&cnt, sizeof(unsigned long long)) != cudaSuccess || cudaMalloc(&conf, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&worst, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(backup); backup = nullptr;
    cleanup();
    return set_err(c, VFS_ERR_CUDA, "adjoint: probe allocation failed");
  }
  for (int s = 0; s < op.nslot; s++)
    cudaMemcpyAsync(backup + s * N, live.p[s], bytes, cudaMemcpyDeviceToDevice, c->stream);
  // room for 8 entries per output when that fits in 30 % of the free memory; else a
  // counting pass first and then the exact count
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  unsigned long long cap = (unsigned long long)(8 * n);
  if ((double)cap * (2 * sizeof(int) + sizeof(double)) > 0.3 * (double)free_b) cap = 0;
  for (int pass = 0; pass < 2; pass++) {
    cudaFree(rows); cudaFree(cols); cudaFree(vals);
    rows = cols = nullptr; vals = nullptr;
    const size_t ncap = cap > 0 ? cap : 1;
    if (cudaMalloc(&rows, sizeof(int) * ncap) != cudaSuccess || cudaMalloc(&cols, sizeof(int) * ncap) != cudaSuccess ||
        cudaMalloc(&vals, sizeof(double) * ncap) != cudaSuccess) {
      cleanup();
      return set_err(c, VFS_ERR_CUDA, "adjoint: probe entry allocation failed");
    }
    cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream);
    cudaMemsetAsync(conf, 0, sizeof(int), c->stream);
    cudaMemsetAsync(worst, 0, sizeof(unsigned long long), c->stream);
    // the operator must be linear: zero in, zero out
    for (int s = 0; s < op.nslot; s++) cudaMemsetAsync(live.p[s], 0, bytes, c->stream);
    if ((rc = fn(c))) { cleanup(); return rc; }
    c->launches++, k_absmax<<<256, 256, 0, c->stream>>>(n, live, N, amax);
    if (host_max(c, amax) != 0) {
      cleanup();
      return set_err(c, VFS_ERR_INVALID, "adjoint: an operator of the step is not linear here");
    }
    for (int cc = 0; cc < cm.count(); cc++) {
      for (int s = 0; s < op.nslot; s++) {
        double tiny = 0;
        for (int kind = 0; kind < 3; kind++) {
          for (int t = 0; t < op.nslot; t++) cudaMemsetAsync(live.p[t], 0, bytes, c->stream);
          c->launches++, k_probe_seed<<<nblocks(N, 256), 256, 0, c->stream>>>(N, cm, cc, kind, live.p[s]);
          if ((rc = fn(c))) { cleanup(); return rc; }
          if (kind < 2) {
            double *dst = kind == 0 ? y0 : y1;
            for (int t = 0; t < op.nslot; t++)
              cudaMemcpyAsync(dst + t * N, live.p[t], bytes, cudaMemcpyDeviceToDevice, c->stream);
          }
          if (kind == 0) {
            c->launches++, k_absmax<<<256, 256, 0, c->stream>>>(n, live, N, amax);
            const double m = host_max(c, amax);
            gmax = std::max(gmax, m);
            tiny = 1e-12 * m;
          }
        }
        c->launches++, k_probe_decode<<<nblocks(n, 256), 256, 0, c->stream>>>(n, N, cm, cc, s, y0, y1, live, tiny, rows, cols, vals,
                                                               cnt, cap, conf, worst);
        if ((rc = check_launch(c, "k_probe_decode"))) { cleanup(); return rc; }
      }
    }
    unsigned long long hn = 0;
    int hc = 0;
    cudaMemcpyAsync(&hn, cnt, sizeof(hn), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(&hc, conf, sizeof(hc), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { cleanup(); return set_err(c, VFS_ERR_CUDA, "adjoint: probe failed"); }
    if (hc) {
      unsigned long long hw = 0;
      cudaMemcpy(&hw, worst, sizeof(hw), cudaMemcpyDeviceToHost);
      double w;
      memcpy(&w, &hw, sizeof(w));
      cleanup();
      char msg[256];
      snprintf(msg, sizeof(msg), "adjoint: probing %s found %d outputs reached by two inputs of one colour "
               "(largest %.3e, largest output %.3e)", name, hc, w, gmax);
      return set_err(c, VFS_ERR_INVALID, msg);
    }
    if (hn <= cap) {
      free_op(op);
      op.nnz = (long long)hn;
      int *ptr = nullptr, *idx = nullptr;
      double *val = nullptr;
      rc = compress(c, (long long)hn, n, cols, rows, vals, &ptr, &idx, &val);
      cudaFree(rows); cudaFree(cols); cudaFree(vals);  // before the sliced copy is allocated
      rows = cols = nullptr; vals = nullptr;
      if (!rc) rc = to_sell(c, n, ptr, idx, val, (int)(kMaxSlots * N), op);
      cudaFree(ptr); cudaFree(idx); cudaFree(val);
      if (!rc) op.fn = fn;
      cleanup();
      return rc;
    }
    cap = hn;  // second pass with the exact size
  }
  cleanup();
  return set_err(c, VFS_ERR_INVALID, "adjoint: probe entry count changed between passes");
}

// y[r] = sum over the entries of row r of val * x[col], x the slots end to end; one
// thread per row, a warp per slice.
__global__ void __launch_bounds__(256) k_spmv_sell(long long n, long long N, const long long *__restrict__ off,
                                                   const int *__restrict__ col, const double *__restrict__ val,
                                                   const double *__restrict__ x, SlotPtrs y) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long long sl = r >> 5;
  const long long b = off[sl] + (r & 31), e = off[sl + 1];
  double s = 0;
  for (long long k = b; k < e; k += 32) s += val[k] * x[col[k]];
  const unsigned q = (unsigned)(r / N);
  double *dst = y.p[0];
#pragma unroll
  for (int t = 1; t < kMaxSlots; t++) dst = q == (unsigned)t ? y.p[t] : dst;  // no local copy of y
  dst[r - q * N] = s;
}

// In place on bank b: slots <- L slots (transpose = 0: the operator's own kernels run on
// the bank's arrays, swapped in for the context's fields) or L^T slots (transpose = 1: the
// measured matrix).
static int apply_op(Ctx *c, int o, int b, int transpose) {
  Adjoint &A = *c->adj;
  LinOp &op = A.op[o];
  const long long N = c->g.N, n = (long long)op.nslot * N;
  int rc;
  if (!transpose) {
    double *keep[kMaxSlots];
    for (int s = 0; s < op.nslot; s++) {
      double *&f = c->f[op.slot[s].field][op.slot[s].comp];
      keep[s] = f;
      f = A.bank[b][op.slot[s].field][op.slot[s].comp];
    }
    rc = op.fn(c);
    for (int s = 0; s < op.nslot; s++) c->f[op.slot[s].field][op.slot[s].comp] = keep[s];
    return rc;
  }
  SlotPtrs y;
  for (int s = 0; s < op.nslot; s++) {
    y.p[s] = A.bank[b][op.slot[s].field][op.slot[s].comp];
    cudaMemcpyAsync(A.xcat + s * N, y.p[s], sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream);
  }
  c->launches++, k_spmv_sell<<<nblocks(n, 256), 256, 0, c->stream>>>(n, N, op.off, op.col, op.val, A.xcat, y);
  return check_launch(c, "k_spmv_sell");
}

// In place on the adjoint bank: slots <- L^T slots by the hand-written transpose where the
// operator has one (vfs_adjoint_stencil.cu: Pressure_Gradient, the local Poisson right-hand
// side, UpdatePressure, Projection; the blocked-cell VolumeFlux is a 0/1 diagonal, its own
// transpose), else (or with measured) by the measured matrix.
static bool handwritten(const Ctx *c, int o) {
  switch (o) {
    case OP_PG: case OP_PRL: case OP_UP: return true;
    case OP_C2C: case OP_FBT: case OP_PJ: return contra2cart_linear(c->g);
    case OP_VF: case OP_IBBC: return !c->g.immersed;
    default: return false;
  }
}

static int ensure_measured(Ctx *c, int o);

static int adjoint_apply(Ctx *c, int o, bool measured = false) {
  int rc;
  if (measured || !handwritten(c, o)) {
    if ((rc = ensure_measured(c, o))) return rc;
    return apply_op(c, o, ADJ, 1);
  }
  const long long N = c->g.N;
  V3 lU = bank3(c, ADJ, VFS_UCONT), lu = bank3(c, ADJ, VFS_UCAT), luo = bank3(c, ADJ, VFS_UCAT_O);
  V3 tmp{c->adj->xcat, c->adj->xcat + N, c->adj->xcat + 2 * N};
  double *lP = bankp(c, ADJ, VFS_P, 0), *lphi = bankp(c, ADJ, VFS_PHI, 0);
  switch (o) {
    case OP_C2C: return contra2cart_adjoint(c, lU, lu, luo, tmp);
    case OP_FBT: return form_bcs_tail_adjoint(c, lU, lu, luo, tmp);
    case OP_IBBC: return ib_bc_adjoint(c, lU);
    case OP_PG: return pressure_gradient_adjoint(c, lP, bank3(c, ADJ, VFS_DP));
    case OP_PRL: return poisson_rhs_local_adjoint(c, lU, bankp(c, ADJ, VFS_B, 0));
    case OP_UP: return update_pressure_adjoint(c, lP, lphi);
    case OP_PJ:
      if ((rc = contra2cart_adjoint(c, lU, lu, luo, tmp))) return rc;  // Projection closes with Contra2Cart
      return projection_adjoint(c, lphi, lU);
    case OP_VF: return apply_op(c, OP_VF, ADJ, 0);
    default: return set_err(c, VFS_ERR_INVALID, "adjoint: no hand-written transpose");
  }
}

// ---------------------------------------------------------------- set-up
static void set_slots(LinOp &op, std::initializer_list<int> fields) {
  op.nslot = 0;
  for (int f : fields) {
    const int dof = (f == VFS_P || f == VFS_B || f == VFS_PHI) ? 1 : 3;
    for (int q = 0; q < dof; q++) op.slot[op.nslot++] = Slot{f, q};
  }
}

static int check_supported(Ctx *c) {
  const Grid &g = c->g;
  if (g.les) return set_err(c, VFS_ERR_INVALID, "adjoint: the eddy viscosity is not differentiated (les must be 0)");
  if (g.bc[4] == 5 && c->cfg.inletprofile != 100)
    return set_err(c, VFS_ERR_INVALID, "adjoint: an inlet is differentiated for inletprofile 100 only");
  return VFS_OK;
}

static const char *const kOpName[OP_N] = {"Contra2Cart", "the FormBCS tail", "Pressure_Gradient", "VolumeFlux",
                                          "the Poisson right-hand side", "UpdatePressure", "Projection", "IB_BC",
                                          "the IB-node interpolation"};

// The measured matrix of operator o (probed once).
static int ensure_measured(Ctx *c, int o) {
  LinOp &op = c->adj->op[o];
  if (op.off) return VFS_OK;
  if (!op.nslot) return set_err(c, VFS_ERR_INVALID, "adjoint: no such operator here");
  return probe(c, kOpName[o], op, o == OP_IBM ? 7 : 5, op.fn);
}

// Measures the operators of the step (once per grid, nvert and boundary set).
static int adjoint_setup(Ctx *c) {
  int rc;
  if (!c->adj) c->adj = new Adjoint();
  Adjoint &A = *c->adj;
  if (A.built) return VFS_OK;
  if ((rc = check_supported(c))) return rc;
  if ((rc = ensure_banks(c))) return rc;
  if (!c->ps.built && (rc = poisson_lhs(c))) return rc;
  if ((rc = calc_inlet_area(c))) return rc;
  const bool imm = c->g.immersed != 0;
  // every operator's slots and forward function (the tangent runs them); the matrices of
  // those the sweep transposes by measured matrix now, the others on first request
  set_slots(A.op[OP_C2C], {VFS_UCONT, VFS_UCAT, VFS_UCAT_O});
  A.op[OP_C2C].fn = [](Ctx *x) { return contra2cart(x); };
  set_slots(A.op[OP_FBT], {VFS_UCONT, VFS_UCAT, VFS_UCAT_O});
  A.op[OP_FBT].fn = [](Ctx *x) { return form_bcs_tail(x); };
  set_slots(A.op[OP_PG], {VFS_P, VFS_DP});
  A.op[OP_PG].fn = [](Ctx *x) { return pressure_gradient_mode(x, 0, 0.0); };
  if (!imm) {
    set_slots(A.op[OP_VF], {VFS_UCONT});
    A.op[OP_VF].fn = [](Ctx *x) { return volume_flux(x); };
  }
  set_slots(A.op[OP_PRL], {VFS_UCONT, VFS_B});
  A.op[OP_PRL].fn = [](Ctx *x) { return poisson_rhs_local(x); };
  set_slots(A.op[OP_UP], {VFS_PHI, VFS_P});
  A.op[OP_UP].fn = [](Ctx *x) { return update_pressure(x); };
  set_slots(A.op[OP_PJ], {VFS_PHI, VFS_UCONT, VFS_UCAT, VFS_UCAT_O});
  A.op[OP_PJ].fn = [](Ctx *x) { return projection(x); };
  set_slots(A.op[OP_IBBC], {VFS_UCONT, VFS_UCAT});
  A.op[OP_IBBC].fn = [](Ctx *x) { return ib_bc(x); };
  if (imm) {
    set_slots(A.op[OP_IBM], {VFS_UCAT, VFS_P, VFS_UCONT, VFS_UCAT_O});
    A.op[OP_IBM].fn = [](Ctx *x) { return ibm_interpolation(x); };
  }
  for (int o = 0; o < OP_N; o++)
    if (A.op[o].nslot && !handwritten(c, o) && (rc = ensure_measured(c, o))) return rc;
  // dP.z per unit flux deficit of the k-periodic forcing: Pressure_Gradient with P = 0
  if (c->g.kper && pressure_forcing_mode(c) == 2) {
    const size_t bytes = sizeof(double) * c->g.N;
    double *keep[4] = {};
    double *src[4] = {c->f[VFS_P][0], c->f[VFS_DP][0], c->f[VFS_DP][1], c->f[VFS_DP][2]};
    for (int t = 0; t < 4; t++) {
      if (cudaMalloc(&keep[t], bytes) != cudaSuccess) {
        for (int u = 0; u < t; u++) cudaFree(keep[u]);
        return set_err(c, VFS_ERR_CUDA, "adjoint: allocation failed");
      }
      cudaMemcpyAsync(keep[t], src[t], bytes, cudaMemcpyDeviceToDevice, c->stream);
    }
    cudaMemsetAsync(c->f[VFS_P][0], 0, bytes, c->stream);
    rc = pressure_gradient_mode(c, 2, 1.0);
    cudaMemcpyAsync(A.cz, c->f[VFS_DP][2], bytes, cudaMemcpyDeviceToDevice, c->stream);
    for (int t = 0; t < 4; t++) cudaMemcpyAsync(src[t], keep[t], bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    for (int t = 0; t < 4; t++) cudaFree(keep[t]);
    if (rc) return rc;
  }
  A.built = true;
  return VFS_OK;
}

// ---------------------------------------------------------------- reductions and small kernels
static const int kAdjBlocks = 296;

// mode 0: sum of a*b over all points; mode 1: of a over the interior k-faces with two
// fluid cells, k = 1..mz-2 (the faces Calc_k_Flux sums).
__global__ void k_dot_mask(long long N, int mode, Grid g, const uint8_t *__restrict__ nv, const double *__restrict__ a,
                           const double *__restrict__ b, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    if (mode == 1) {
      int i, j, k;
      dijk(g, p, i, j, k);
      if (k < 1 || k > g.mz - 2 || j < 1 || j > g.my - 2 || i < 1 || i > g.mx - 2) continue;
      if (nv[p - (long long)g.mx * g.my] + nv[p] != 0) continue;
    }
    s += a[p] * (b ? b[p] : 1.0);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

static int dot(Ctx *c, int mode, const double *a, const double *b, double *out) {
  int rc;
  if ((rc = ensure_red(c, kAdjBlocks + 64))) return rc;
  c->launches++, k_dot_mask<<<kAdjBlocks, 256, 0, c->stream>>>(c->g.N, mode, c->g, c->nv, a, b, c->red);
  if ((rc = check_launch(c, "k_dot_mask"))) return rc;
  return reduce_sum(c, c->red, kAdjBlocks, out);
}

__global__ void k_axpy(long long n, double s, const double *x, double *y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < n) y[p] += s * x[p];
}
// y += s on the interior k-faces with two fluid cells (Calc_k_Flux's faces).
__global__ void k_add_kflux(Grid g, const uint8_t *__restrict__ nv, double s, double *y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (k < 1 || k > g.mz - 2 || j < 1 || j > g.my - 2 || i < 1 || i > g.mx - 2) return;
  if (nv[p - (long long)g.mx * g.my] + nv[p] != 0) return;
  y[p] += s;
}
// y[p] += s * (w ? w[p] : 1) on fluid cells; off fluid y is zeroed when clear is set.
__global__ void k_fluid_shift(long long n, const uint8_t *fluid, const double *w, double s, int clear, double *y) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (!fluid[p]) { if (clear) y[p] = 0; return; }
  y[p] += s * (w ? w[p] : 1.0);
}
__global__ void k_fluid_sum(long long n, const uint8_t *fluid, const double *a, const double *w, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
    if (fluid[p]) s += a[p] * (w ? w[p] : 1.0);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int t = blockDim.x / 2; t > 0; t >>= 1) {
    if (threadIdx.x < t) sh[threadIdx.x] += sh[threadIdx.x + t];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}
static int fluid_sum(Ctx *c, const double *a, const double *w, double *out) {
  int rc;
  if ((rc = ensure_red(c, kAdjBlocks + 64))) return rc;
  c->launches++, k_fluid_sum<<<kAdjBlocks, 256, 0, c->stream>>>(c->g.N, c->ps.fluid, a, w, c->red);
  if ((rc = check_launch(c, "k_fluid_sum"))) return rc;
  return reduce_sum(c, c->red, kAdjBlocks, out);
}

// ---------------------------------------------------------------- inlet / outlet planes
// Plane kernels over the interior (i, j) of k = 0 (inlet faces) or k = mz-2 (outlet
// faces); a face counts as fluid when its downstream cell (inlet) or upstream cell
// (outlet) is fluid, as in k_inflow and k_outlet_parts.
__device__ __forceinline__ double zarea(const Metrics &m, long long p) {
  return sqrt(m.zet.x[p] * m.zet.x[p] + m.zet.y[p] * m.zet.y[p] + m.zet.z[p] * m.zet.z[p]);
}

__global__ void k_plane_sum(Grid g, Metrics m, const uint8_t *__restrict__ nv, int outlet, int fluid_only,
                            int area_weight, const double *a, double *parts) {
  __shared__ double sh[256];
  const int nx = g.mx - 2, ny = g.my - 2;
  double s = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * ny;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
    const long long p = lidx(g, i, j, outlet ? g.mz - 2 : 0);
    const long long pf = outlet ? p : p + (long long)g.mx * g.my;
    if (fluid_only && nv[pf] != 0) continue;
    const double w = area_weight ? zarea(m, p) : 1.0;
    s += w * (a ? a[p] : 1.0);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}
static int plane_sum(Ctx *c, int outlet, int fluid_only, int area_weight, const double *a, double *out) {
  int rc;
  if ((rc = ensure_red(c, kAdjBlocks + 64))) return rc;
  c->launches++, k_plane_sum<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, metrics(c), c->nv, outlet, fluid_only, area_weight, a, c->red);
  if ((rc = check_launch(c, "k_plane_sum"))) return rc;
  return reduce_sum(c, c->red, kAdjBlocks, out);
}
// y[p] += s * |zet| (area_weight) or s over the plane faces (fluid ones if fluid_only).
__global__ void k_plane_add(Grid g, Metrics m, const uint8_t *__restrict__ nv, int outlet, int fluid_only,
                            int area_weight, double s, double *y) {
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny) return;
  const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
  const long long p = lidx(g, i, j, outlet ? g.mz - 2 : 0);
  const long long pf = outlet ? p : p + (long long)g.mx * g.my;
  if (fluid_only && nv[pf] != 0) return;
  y[p] += s * (area_weight ? zarea(m, p) : 1.0);
}
static int plane_add(Ctx *c, int outlet, int fluid_only, int area_weight, double s, double *y) {
  const long long npl = (long long)(c->g.mx - 2) * (c->g.my - 2);
  c->launches++, k_plane_add<<<nblocks(npl, 256), 256, 0, c->stream>>>(c->g, metrics(c), c->nv, outlet, fluid_only, area_weight, s, y);
  return check_launch(c, "k_plane_add");
}

// Inlet (inletprofile 100, k_inflow): Ucat(k=0) = plane, Ucont.z(k=0) = 0.5*(plane +
// Ucat(k=1)) . zet on faces with a fluid downstream cell; Ucat.z = Ucont.z = 0 on the others.
__global__ void k_inflow_tan(Grid g, Metrics m, const uint8_t *__restrict__ nv, const double *__restrict__ dpl, V3 duc,
                             V3 duk) {
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny) return;
  const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
  const long long p = lidx(g, i, j, 0), p1 = p + (long long)g.mx * g.my;
  if (nv[p1] == 0) {
    const double *pl = dpl + 3 * ((long long)j * g.mx + i);
    duk.x[p] = pl[0]; duk.y[p] = pl[1]; duk.z[p] = pl[2];
    duc.z[p] = 0.5 * (pl[0] + duk.x[p1]) * m.zet.x[p] + 0.5 * (pl[1] + duk.y[p1]) * m.zet.y[p] +
               0.5 * (pl[2] + duk.z[p1]) * m.zet.z[p];
  } else {
    duk.z[p] = 0;
    duc.z[p] = 0;
  }
}
__global__ void k_inflow_adj(Grid g, Metrics m, const uint8_t *__restrict__ nv, double *lpl, V3 luc, V3 luk) {
  const int nx = g.mx - 2, ny = g.my - 2;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny) return;
  const int i = 1 + (int)(t % nx), j = 1 + (int)(t / nx);
  const long long p = lidx(g, i, j, 0), p1 = p + (long long)g.mx * g.my;
  if (nv[p1] == 0) {
    double *pl = lpl + 3 * ((long long)j * g.mx + i);
    const double l = luc.z[p];
    const double z[3] = {m.zet.x[p], m.zet.y[p], m.zet.z[p]};
    pl[0] += 0.5 * z[0] * l + luk.x[p];
    pl[1] += 0.5 * z[1] * l + luk.y[p];
    pl[2] += 0.5 * z[2] * l + luk.z[p];
    luk.x[p1] += 0.5 * z[0] * l;
    luk.y[p1] += 0.5 * z[1] * l;
    luk.z[p1] += 0.5 * z[2] * l;
    luk.x[p] = 0; luk.y[p] = 0; luk.z[p] = 0;
  } else {
    luk.z[p] = 0;
  }
  luc.z[p] = 0;
}

// ---------------------------------------------------------------- immersed VolumeFlux
// The faces the forward corrected (|flux| > 1e-8 between a fluid cell and an IB node), with
// sign +1 for a fluid cell below the node and -1 above; f' = f - sign*area*corr with
// corr = sum(sign*f)/sum(area).  Faces at or below 1e-8 were zeroed.
__device__ __forceinline__ double centre_area(CV3 m, long long p) {
  return sqrt(m.x[p] * m.x[p] + m.y[p] * m.y[p] + m.z[p] * m.z[p]);
}
// mode 0: parts of sum(sign*x) and of sum(area) over the corrected faces; mode 1: tangent
// x -= sign*area*s there and 0 on zeroed faces; mode 2: parts of sum(sign*area*x);
// mode 3: adjoint x += sign*s there and 0 on zeroed faces.
__global__ void k_vfi_lin(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 base, V3 x, int mode, double s,
                          double *parts) {
  __shared__ double s1[256], s2[256];
  double a1 = 0, a2 = 0;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) continue;
    const int v0 = nv[p];
    const double *bc[3] = {base.x, base.y, base.z};
    double *xc[3] = {x.x, x.y, x.z};
    const CV3 *met[3] = {&m.csi, &m.eta, &m.zet};
    const long long off[3] = {1, sy, sz};
    const bool inner[3] = {i < g.mx - 2, j < g.my - 2, k < g.mz - 2};
    for (int d = 0; d < 3; d++) {
      const int vn = nv[p + off[d]];
      double sign = 0;
      if (v0 == 0 && vn == 1 && inner[d]) sign = 1;
      if (v0 == 1 && vn == 0 && inner[d]) sign = -1;
      if (sign == 0) continue;
      const bool active = fabs(bc[d][p]) > 1.e-8;
      const double area = centre_area(*met[d], p);
      if (mode == 0) {
        if (active) { a1 += sign * xc[d][p]; a2 += area; }
      } else if (mode == 1) {
        xc[d][p] = active ? xc[d][p] - sign * area * s : 0.0;
      } else if (mode == 2) {
        if (active) a1 += sign * area * xc[d][p];
      } else {
        xc[d][p] = active ? xc[d][p] + sign * s : 0.0;
      }
    }
  }
  if (mode == 1 || mode == 3) return;
  s1[threadIdx.x] = a1; s2[threadIdx.x] = a2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { parts[blockIdx.x] = s1[0]; parts[gridDim.x + blockIdx.x] = s2[0]; }
}

static int vfi_lin(Ctx *c, const StepTape &t, int b, int adjoint) {
  int rc;
  if ((rc = ensure_red(c, 2 * kAdjBlocks + 64))) return rc;
  CV3 base{t.vfi[0], t.vfi[1], t.vfi[2]};
  V3 x = bank3(c, b, VFS_UCONT);
  Metrics m = metrics(c);
  double sx = 0, area = 0, unused = 0;
  if (adjoint) {
    c->launches++, k_vfi_lin<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, m, c->nv, base, x, 2, 0.0, c->red);
    if ((rc = check_launch(c, "k_vfi_lin"))) return rc;
    if ((rc = reduce_sum(c, c->red, kAdjBlocks, &sx))) return rc;
    c->launches++, k_vfi_lin<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, m, c->nv, base, x, 0, 0.0, c->red);
    if ((rc = check_launch(c, "k_vfi_lin"))) return rc;
    if ((rc = reduce_sum(c, c->red, kAdjBlocks, &unused))) return rc;
  } else {
    c->launches++, k_vfi_lin<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, m, c->nv, base, x, 0, 0.0, c->red);
    if ((rc = check_launch(c, "k_vfi_lin"))) return rc;
    if ((rc = reduce_sum(c, c->red, kAdjBlocks, &sx))) return rc;
  }
  if ((rc = reduce_sum(c, c->red + kAdjBlocks, kAdjBlocks, &area))) return rc;
  const double s = area > 1.e-15 ? sx / area : 0.0;
  c->launches++, k_vfi_lin<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, m, c->nv, base, x, adjoint ? 3 : 1, adjoint ? -s : s, c->red);
  return check_launch(c, "k_vfi_lin");
}

// ---------------------------------------------------------------- Poisson solve
// Tangent: the forward solver on the tangent right-hand side (Remove_Nullspace and the
// periodic ghosts of Phi included).  Adjoint: the transpose of that map: the ghost copy
// and the zero off the unknowns transposed, the fluid mean removed, then FGMRES with the
// transposed operator; lambda_b is the solution on the unknowns.  Both solve from 0 (a
// linear map of the right-hand side) straight into the bank arrays, with the context's
// B and Phi pointers swapped for the call, so the forward Phi, the next forward solve's
// starting point, stays untouched.
static int lin_solve_into(Ctx *c, double *rhs, double *sol, const vfs_solve_opts *o, bool transpose) {
  vfs_solve_opts lo;
  if (o) lo = *o;
  else { memset(&lo, 0, sizeof(lo)); }
  lo.zero_guess = 1;
  double *fb = c->f[VFS_B][0], *fphi = c->f[VFS_PHI][0];
  const bool guess = c->ps.guess;
  c->f[VFS_B][0] = rhs;
  c->f[VFS_PHI][0] = sol;
  poisson_set_transpose(c, transpose);
  vfs_solve_stats st;
  memset(&st, 0, sizeof(st));
  int rc = poisson_solve(c, &lo, &st);
  poisson_set_transpose(c, false);
  if (transpose) c->adj->it_adj += st.iterations, c->adj->n_adj++;
  c->f[VFS_B][0] = fb;
  c->f[VFS_PHI][0] = fphi;
  c->ps.guess = guess;
  return rc == VFS_ERR_NOT_CONVERGED ? VFS_OK : rc;
}

static int solve_lin(Ctx *c, int b, const vfs_solve_opts *o) {
  const size_t bytes = sizeof(double) * c->g.N;
  const long long N = c->g.N;
  int rc;
  double *bb = bankp(c, b, VFS_B, 0), *ph = bankp(c, b, VFS_PHI, 0);
  if (b == TAN) return lin_solve_into(c, bb, ph, o, false);
  if ((rc = periodic_copy1_adjoint(c, ph))) return rc;
  c->launches++, k_fluid_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, c->ps.fluid, nullptr, 0.0, 1, ph);
  double sum = 0;
  if ((rc = fluid_sum(c, ph, nullptr, &sum))) return rc;
  c->launches++, k_fluid_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, c->ps.fluid, nullptr, -sum / (double)c->ps.nfluid, 1, ph);
  if ((rc = lin_solve_into(c, ph, bb, o, true))) return rc;
  c->launches++, k_fluid_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, c->ps.fluid, nullptr, 0.0, 1, bb);
  cudaMemsetAsync(ph, 0, bytes, c->stream);
  return check_launch(c, "k_fluid_shift");
}

// Remove_Nullspace_Scale on b (b -= sum_fluid(b) * aj / sum(aj)) and its transpose.
static int nullspace_scale_lin(Ctx *c, int b) {
  int rc;
  const long long N = c->g.N;
  double *x = bankp(c, b, VFS_B, 0);
  const double *aj = c->f[VFS_AJ][0];
  double sum = 0;
  if (b == TAN) {
    if ((rc = fluid_sum(c, x, nullptr, &sum))) return rc;
    c->launches++, k_fluid_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, c->ps.fluid, aj, -sum / c->ps.sum_aj, 0, x);
  } else {
    if ((rc = fluid_sum(c, x, aj, &sum))) return rc;
    c->launches++, k_fluid_shift<<<nblocks(N, 256), 256, 0, c->stream>>>(N, c->ps.fluid, nullptr, -sum / c->ps.sum_aj, 0, x);
  }
  return check_launch(c, "k_fluid_shift");
}

// ---------------------------------------------------------------- one step, tangent and adjoint
static const double kAlfa[4] = {0.25, 1 / 3., 0.5, 1.};

static void copy3(Ctx *c, double *const dst[3], double *const src[3]) {
  const size_t bytes = sizeof(double) * c->g.N;
  for (int q = 0; q < 3; q++) cudaMemcpyAsync(dst[q], src[q], bytes, cudaMemcpyDeviceToDevice, c->stream);
}
// dst += src; src = 0.
static int move_add3(Ctx *c, double *const dst[3], double *const src[3]) {
  const long long N = c->g.N;
  for (int q = 0; q < 3; q++) {
    c->launches++, k_axpy<<<nblocks(N, 256), 256, 0, c->stream>>>(N, 1.0, src[q], dst[q]);
    cudaMemsetAsync(src[q], 0, sizeof(double) * N, c->stream);
  }
  return check_launch(c, "k_axpy");
}

static bool inlet100(const Ctx *c) { return c->g.bc[4] == 5 && c->cfg.inletprofile == 100; }
static bool kforce(const Ctx *c) { return c->g.kper && pressure_forcing_mode(c) == 2; }

static int tangent_step(Ctx *c, const StepTape &t, const vfs_solve_opts *o) {
  Adjoint &A = *c->adj;
  const Grid &g = c->g;
  int rc;
  for (int d = 0; d < 3; d++)  // the tangent's face fluxes (only the tangent uses them)
    for (int q = 0; q < 6; q++)
      if ((rc = grow(c, &A.tface[d][q], g.N))) return rc;
  const bool imm = g.immersed != 0;
  V3 dU = bank3(c, TAN, VFS_UCONT), du = bank3(c, TAN, VFS_UCAT), ddp = bank3(c, TAN, VFS_DP);
  V3 dpu{A.pu[TAN][0], A.pu[TAN][1], A.pu[TAN][2]};
  if (t.first_step) {
    if (imm && (rc = apply_op(c, OP_IBM, TAN, 0))) return rc;
    if ((rc = apply_op(c, OP_IBBC, TAN, 0))) return rc;
  }
  double dF = 0;
  if (kforce(c) && (rc = dot(c, 1, dU.z, nullptr, &dF))) return rc;
  if ((rc = apply_op(c, OP_PG, TAN, 0))) return rc;
  if (kforce(c)) {
    c->launches++, k_axpy<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g.N, dF / (g.mz - 2), A.cz, ddp.z);
    if ((rc = check_launch(c, "k_axpy"))) return rc;
  }
  // RungeKutta
  double dfin = 0;
  if (inlet100(c)) {
    const long long npl = (long long)(g.mx - 2) * (g.my - 2);
    c->launches++, k_inflow_tan<<<nblocks(npl, 256), 256, 0, c->stream>>>(g, metrics(c), c->nv, A.plane[TAN], dU, du);
    if ((rc = check_launch(c, "k_inflow_tan"))) return rc;
    double flux1 = 0;
    if ((rc = plane_sum(c, 0, 0, 0, dU.z, &flux1))) return rc;
    dfin = flux1;
    if (c->scal[VFS_S_INLET_FLUX] > 0) {
      if ((rc = plane_add(c, 0, 1, 1, -flux1 / c->scal[VFS_S_INLET_AREA], dU.z))) return rc;
      if ((rc = plane_sum(c, 0, 1, 0, dU.z, &dfin))) return rc;
    }
  }
  if ((rc = apply_op(c, OP_C2C, TAN, 0))) return rc;
  if ((rc = apply_op(c, OP_FBT, TAN, 0))) return rc;
  if (imm && (rc = apply_op(c, OP_IBM, TAN, 0))) return rc;
  copy3(c, A.pu[TAN], A.bank[TAN][VFS_UCONT]);
  for (int s = 0; s < 4; s++) {
    if (s == 0 && (rc = apply_op(c, OP_C2C, TAN, 0))) return rc;
    const double a = kAlfa[s] * g.dt * g.st;
    if ((rc = ff2_stage_tangent(c, t.uc[s], t.uk[s], a, dU, du, ddp, dpu, A.tface))) return rc;
    if ((rc = apply_op(c, OP_C2C, TAN, 0))) return rc;
  }
  if (g.bc[5] == 4) {
    double fo = 0, area = 0;
    if ((rc = plane_sum(c, 1, 1, 0, dU.z, &fo))) return rc;
    if ((rc = plane_sum(c, 1, 1, 1, nullptr, &area))) return rc;
    if ((rc = plane_add(c, 1, 1, 1, (dfin - fo) / area, dU.z))) return rc;
  }
  if ((rc = apply_op(c, OP_FBT, TAN, 0))) return rc;
  // Poisson
  if (imm) {
    if ((rc = vfi_lin(c, t, TAN, 0))) return rc;
  } else if ((rc = apply_op(c, OP_VF, TAN, 0))) {
    return rc;
  }
  if ((rc = apply_op(c, OP_PRL, TAN, 0))) return rc;
  if ((rc = nullspace_scale_lin(c, TAN))) return rc;
  if ((rc = solve_lin(c, TAN, o))) return rc;
  if ((rc = apply_op(c, OP_UP, TAN, 0))) return rc;
  if ((rc = apply_op(c, OP_PJ, TAN, 0))) return rc;
  if (imm && (rc = apply_op(c, OP_IBM, TAN, 0))) return rc;
  if ((rc = apply_op(c, OP_IBBC, TAN, 0))) return rc;
  if ((rc = apply_op(c, OP_C2C, TAN, 0))) return rc;
  copy3(c, A.bank[TAN][VFS_UCAT_O], A.bank[TAN][VFS_UCAT]);
  return VFS_OK;
}

static int adjoint_step(Ctx *c, const StepTape &t, const vfs_solve_opts *o) {
  Adjoint &A = *c->adj;
  const Grid &g = c->g;
  int rc;
  const bool imm = g.immersed != 0;
  V3 lU = bank3(c, ADJ, VFS_UCONT), lu = bank3(c, ADJ, VFS_UCAT), ldp = bank3(c, ADJ, VFS_DP);
  V3 lpu{A.pu[ADJ][0], A.pu[ADJ][1], A.pu[ADJ][2]};
  const size_t bytes = sizeof(double) * g.N;
  if ((rc = move_add3(c, A.bank[ADJ][VFS_UCAT], A.bank[ADJ][VFS_UCAT_O]))) return rc;  // Ucat_o = Ucat
  if ((rc = adjoint_apply(c, OP_C2C))) return rc;
  if ((rc = adjoint_apply(c, OP_IBBC))) return rc;
  if (imm && (rc = adjoint_apply(c, OP_IBM))) return rc;
  if ((rc = adjoint_apply(c, OP_PJ))) return rc;
  if ((rc = adjoint_apply(c, OP_UP))) return rc;
  if ((rc = solve_lin(c, ADJ, o))) return rc;
  if ((rc = nullspace_scale_lin(c, ADJ))) return rc;
  if ((rc = adjoint_apply(c, OP_PRL))) return rc;
  cudaMemsetAsync(bankp(c, ADJ, VFS_B, 0), 0, bytes, c->stream);
  if (imm) {
    if ((rc = vfi_lin(c, t, ADJ, 1))) return rc;
  } else if ((rc = adjoint_apply(c, OP_VF))) {
    return rc;
  }
  // RungeKutta, last to first
  if ((rc = adjoint_apply(c, OP_FBT))) return rc;
  double lfin = 0;
  if (g.bc[5] == 4) {
    double sa = 0, area = 0;
    if ((rc = plane_sum(c, 1, 1, 1, lU.z, &sa))) return rc;
    if ((rc = plane_sum(c, 1, 1, 1, nullptr, &area))) return rc;
    lfin = sa / area;
    if ((rc = plane_add(c, 1, 1, 0, -lfin, lU.z))) return rc;
  }
  for (int s = 3; s >= 0; s--) {
    const double a = kAlfa[s] * g.dt * g.st;
    if ((rc = adjoint_apply(c, OP_C2C))) return rc;
    if ((rc = ff2_stage_adjoint(c, t.uc[s], t.uk[s], a, lU, lu, ldp, lpu, A.lface, A.lfp))) return rc;
    if (s == 0 && (rc = adjoint_apply(c, OP_C2C))) return rc;
  }
  if ((rc = move_add3(c, A.bank[ADJ][VFS_UCONT], A.pu[ADJ]))) return rc;  // pUcont = Ucont
  if (imm && (rc = adjoint_apply(c, OP_IBM))) return rc;
  if ((rc = adjoint_apply(c, OP_FBT))) return rc;
  if ((rc = adjoint_apply(c, OP_C2C))) return rc;
  if (inlet100(c)) {
    const long long npl = (long long)(g.mx - 2) * (g.my - 2);
    if (c->scal[VFS_S_INLET_FLUX] > 0) {
      // FluxIn sums the fluid faces after the rescale, which subtracts flux1*|zet|/inletArea
      if ((rc = plane_add(c, 0, 1, 0, lfin, lU.z))) return rc;
      double sa = 0;
      if ((rc = plane_sum(c, 0, 1, 1, lU.z, &sa))) return rc;
      if ((rc = plane_add(c, 0, 0, 0, -sa / c->scal[VFS_S_INLET_AREA], lU.z))) return rc;
    } else if ((rc = plane_add(c, 0, 0, 0, lfin, lU.z))) {
      return rc;
    }
    c->launches++, k_inflow_adj<<<nblocks(npl, 256), 256, 0, c->stream>>>(g, metrics(c), c->nv, A.plane[ADJ], lU, lu);
    if ((rc = check_launch(c, "k_inflow_adj"))) return rc;
  }
  // Pressure_Gradient and the k-flux forcing
  if (kforce(c)) {
    double lF = 0;
    if ((rc = dot(c, 0, A.cz, ldp.z, &lF))) return rc;
    c->launches++, k_add_kflux<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nv, lF / (g.mz - 2), lU.z);
    if ((rc = check_launch(c, "k_add_kflux"))) return rc;
  }
  if ((rc = adjoint_apply(c, OP_PG))) return rc;  // clears ldP
  if (t.first_step) {
    if ((rc = adjoint_apply(c, OP_IBBC))) return rc;
    if (imm && (rc = adjoint_apply(c, OP_IBM))) return rc;
  }
  return VFS_OK;
}

// ---------------------------------------------------------------- state and objective
// Phi is part of the state: the next Poisson solve starts from it.  A checkpoint taken
// between two steps holds Ucont, Ucat, P and Phi (8 arrays): each step ends by copying Ucont
// and Ucat into Ucont_o and Ucat_o, which the load restores the same way.  The first
// checkpoint, of a state set by the caller, also holds Ucat_o and Ucont_o (14 arrays).
static const int kCkptFields[6] = {VFS_UCONT, VFS_UCAT, VFS_P, VFS_PHI, VFS_UCAT_O, VFS_UCONT_O};
static const int kCkptArrays = 14, kCkptShort = 8;

struct HostState { bool first_step = false, guess = false, full = true; int ti = 0; double scal[VFS_NSCALARS] = {}; };

static void save_state(Ctx *c, double *dst, HostState &h, bool full) {
  const size_t bytes = sizeof(double) * c->g.N;
  int a = 0;
  for (int f : kCkptFields) {
    if (!full && (f == VFS_UCAT_O || f == VFS_UCONT_O)) continue;
    for (int q = 0; q < c->dof[f]; q++, a++)
      cudaMemcpyAsync(dst + (size_t)a * c->g.N, c->f[f][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  }
  h.full = full;
  h.first_step = c->first_step;
  h.guess = c->ps.guess;
  h.ti = c->ti;
  memcpy(h.scal, c->scal, sizeof(h.scal));
}
static void load_state(Ctx *c, const double *src, const HostState &h) {
  const size_t bytes = sizeof(double) * c->g.N;
  int a = 0;
  for (int f : kCkptFields) {
    if (!h.full && (f == VFS_UCAT_O || f == VFS_UCONT_O)) continue;
    for (int q = 0; q < c->dof[f]; q++, a++)
      cudaMemcpyAsync(c->f[f][q], src + (size_t)a * c->g.N, bytes, cudaMemcpyDeviceToDevice, c->stream);
  }
  if (!h.full)
    for (int q = 0; q < 3; q++) {
      cudaMemcpyAsync(c->f[VFS_UCAT_O][q], c->f[VFS_UCAT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
      cudaMemcpyAsync(c->f[VFS_UCONT_O][q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
    }
  c->first_step = h.first_step;
  c->ps.guess = h.guess;
  c->ti = h.ti;
  memcpy(c->scal, h.scal, sizeof(h.scal));
}

// J of the final state and, with the seed arrays, dJ/dUcat or dJ/dP.
__global__ void k_objective(Grid g, Metrics m, const uint8_t *__restrict__ nv, int obj, CV3 u, const double *P,
                            V3 lu, double *lp, double *parts) {
  __shared__ double sh[256];
  double s = 0;
  const long long sz = (long long)g.mx * g.my;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    dijk(g, p, i, j, k);
    const bool interior = i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2;
    if (!interior || nv[p] != 0) continue;
    if (obj == VFS_OBJ_KINETIC_ENERGY) {
      const double ia = 1.0 / m.aj[p];
      s += 0.5 * (u.x[p] * u.x[p] + u.y[p] * u.y[p] + u.z[p] * u.z[p]) * ia;
      if (lu.x) { lu.x[p] = u.x[p] * ia; lu.y[p] = u.y[p] * ia; lu.z[p] = u.z[p] * ia; }
    } else {
      double w = 0;
      if (k + 1 <= g.mz - 2 && nv[p + sz] > 0) w += centre_area(m.zet, p);   // body downstream
      if (k - 1 >= 1 && nv[p - sz] > 0) w -= centre_area(m.zet, p - sz);     // body upstream
      s += w * P[p];
      if (lp) lp[p] = w;
      if (obj == VFS_OBJ_DRAG) {
        // viscous traction on the cell's i- and j-faces shared with a body cell (at rest):
        // nu * w / (dn/2) * area with the face area |csi| (|eta|) and the normal spacing
        // dn = 1/(|csi| aj), i.e. 2 nu |csi|^2 aj w per face
        const long long sy = g.mx;
        const double ci = m.csi.x[p] * m.csi.x[p] + m.csi.y[p] * m.csi.y[p] + m.csi.z[p] * m.csi.z[p];
        const double cj = m.eta.x[p] * m.eta.x[p] + m.eta.y[p] * m.eta.y[p] + m.eta.z[p] * m.eta.z[p];
        int ni = 0, nj = 0;
        if (i + 1 <= g.mx - 2 && nv[p + 1] > 0) ni++;
        if (i - 1 >= 1 && nv[p - 1] > 0) ni++;
        if (j + 1 <= g.my - 2 && nv[p + sy] > 0) nj++;
        if (j - 1 >= 1 && nv[p - sy] > 0) nj++;
        const double cv = 2.0 / g.ren * (ni * ci + nj * cj) * m.aj[p];
        s += cv * u.z[p];
        if (lu.z) lu.z[p] = cv;
      }
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int t = blockDim.x / 2; t > 0; t >>= 1) {
    if (threadIdx.x < t) sh[threadIdx.x] += sh[threadIdx.x + t];
    __syncthreads();
  }
  if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

static int objective(Ctx *c, int obj, bool seed, double *J) {
  int rc;
  if ((rc = ensure_red(c, kAdjBlocks + 64))) return rc;
  V3 lu{nullptr, nullptr, nullptr};
  double *lp = nullptr;
  if (seed) {
    lu = bank3(c, ADJ, VFS_UCAT);
    lp = bankp(c, ADJ, VFS_P, 0);
  }
  c->launches++, k_objective<<<kAdjBlocks, 256, 0, c->stream>>>(c->g, metrics(c), c->nv, obj, cv(field3(c, VFS_UCAT)), c->f[VFS_P][0],
                                                 lu, lp, c->red);
  if ((rc = check_launch(c, "k_objective"))) return rc;
  return reduce_sum(c, c->red, kAdjBlocks, J);
}

static void zero_bank(Ctx *c, int b) {
  Adjoint &A = *c->adj;
  const size_t bytes = sizeof(double) * c->g.N;
  for (int f = 0; f < VFS_NFIELDS; f++)
    for (int q = 0; q < 3; q++)
      if (A.bank[b][f][q]) cudaMemsetAsync(A.bank[b][f][q], 0, bytes, c->stream);
  for (int q = 0; q < 3; q++) cudaMemsetAsync(A.pu[b][q], 0, bytes, c->stream);
  cudaMemsetAsync(A.plane[b], 0, sizeof(double) * 3 * c->g.mx * c->g.my, c->stream);
}

__global__ void k_aos_to_soa(long long n, const double *aos, double *x, double *y, double *z) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  x[p] = aos[3 * p]; y[p] = aos[3 * p + 1]; z[p] = aos[3 * p + 2];
}
__global__ void k_soa_to_aos(long long n, double *aos, const double *x, const double *y, const double *z) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  aos[3 * p] = x[p]; aos[3 * p + 1] = y[p]; aos[3 * p + 2] = z[p];
}

static size_t control_size(const Ctx *c, int control) {
  return control == VFS_CTRL_INFLOW_PLANE ? 3 * (size_t)c->g.mx * c->g.my : 3 * (size_t)c->g.N;
}

static int check_opts(Ctx *c, const vfs_adjoint_opts *o) {
  if (!o || o->nsteps < 1) return set_err(c, VFS_ERR_INVALID, "adjoint: nsteps must be at least 1");
  if (c->cfg.implicit) return set_err(c, VFS_ERR_INVALID, "adjoint: the implicit momentum solve is not differentiated");
  if (o->objective != VFS_OBJ_KINETIC_ENERGY && o->objective != VFS_OBJ_PRESSURE_DRAG && o->objective != VFS_OBJ_DRAG)
    return set_err(c, VFS_ERR_INVALID, "adjoint: unknown objective");
  if (o->control != VFS_CTRL_INITIAL_UCONT && o->control != VFS_CTRL_INFLOW_PLANE)
    return set_err(c, VFS_ERR_INVALID, "adjoint: unknown control");
  if (o->control == VFS_CTRL_INFLOW_PLANE && !inlet100(c))
    return set_err(c, VFS_ERR_INVALID, "adjoint: the inflow-plane control needs an inletprofile 100 inlet");
  return VFS_OK;
}

static int ensure_tapes(Ctx *c, int n) {
  Adjoint &A = *c->adj;
  int rc;
  while ((int)A.tapes.size() < n) {
    A.tapes.emplace_back();
    if ((rc = tape_alloc(c, A.tapes.back()))) return rc;
  }
  return VFS_OK;
}

static int checkpoint_every(const vfs_adjoint_opts *o) {
  return o->checkpoint_every > 0 ? o->checkpoint_every : std::max(1, (int)ceil(sqrt((double)o->nsteps)));
}

// ---------------------------------------------------------------- drivers
static int prepare(Ctx *c, const vfs_adjoint_opts *o) {
  int rc;
  if ((rc = check_opts(c, o))) return rc;
  if ((rc = adjoint_setup(c))) return rc;
  Adjoint &A = *c->adj;
  const int every = checkpoint_every(o);
  const int nck = (o->nsteps + every - 1) / every + 1;
  if (A.nckpt < nck) {
    cudaFree(A.ckpt);
    A.ckpt = nullptr;
    A.nckpt = 0;
    if (cudaMalloc(&A.ckpt, sizeof(double) * (kCkptArrays + (size_t)kCkptShort * (nck - 1)) * c->g.N) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "adjoint: checkpoint allocation failed");
    A.nckpt = nck;
  }
  return VFS_OK;
}

static double *ckpt(Ctx *c, int n) {
  return c->adj->ckpt + (n == 0 ? 0 : kCkptArrays + (size_t)kCkptShort * (n - 1)) * c->g.N;
}

static int step_forward(Ctx *c, const vfs_adjoint_opts *o, StepTape *t) {
  c->tape = t;
  vfs_step_stats st;
  memset(&st, 0, sizeof(st));
  int rc = step_core(c, &o->solve, &st);
  c->tape = nullptr;
  c->adj->it_fwd += st.poisson.iterations, c->adj->n_fwd++;
  return rc == VFS_ERR_NOT_CONVERGED ? VFS_OK : rc;
}

static int objective_run(Ctx *c, const vfs_adjoint_opts *o, double *J) {
  int rc;
  if ((rc = prepare(c, o))) return rc;
  HostState h0;
  save_state(c, ckpt(c, 0), h0, true);
  for (int s = 0; s < o->nsteps && !rc; s++) rc = step_forward(c, o, nullptr);
  if (!rc) rc = objective(c, o->objective, false, J);
  load_state(c, ckpt(c, 0), h0);
  cudaStreamSynchronize(c->stream);
  return rc;
}

static int tangent_run(Ctx *c, const vfs_adjoint_opts *o, const double *dir, double *J, double *dJ) {
  int rc;
  if ((rc = prepare(c, o))) return rc;
  if ((rc = ensure_tapes(c, 1))) return rc;
  Adjoint &A = *c->adj;
  HostState h0;
  save_state(c, ckpt(c, 0), h0, true);
  zero_bank(c, TAN);
  zero_bank(c, ADJ);
  const size_t nc = control_size(c, o->control);
  double *dev = nullptr;
  if (cudaMalloc(&dev, sizeof(double) * nc) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "adjoint: allocation failed");
  cudaMemcpyAsync(dev, dir, sizeof(double) * nc, cudaMemcpyHostToDevice, c->stream);
  if (o->control == VFS_CTRL_INITIAL_UCONT) {
    V3 d = bank3(c, TAN, VFS_UCONT);
    c->launches++, k_aos_to_soa<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, dev, d.x, d.y, d.z);
  } else {
    cudaMemcpyAsync(A.plane[TAN], dev, sizeof(double) * nc, cudaMemcpyDeviceToDevice, c->stream);
  }
  for (int s = 0; s < o->nsteps && !rc; s++) {
    rc = step_forward(c, o, &A.tapes[0]);
    if (!rc) rc = tangent_step(c, A.tapes[0], &o->solve);
  }
  if (!rc) rc = objective(c, o->objective, true, J);
  double d = 0, t = 0;
  if (!rc) {  // dJ = <dJ/dUcat, dUcat> + <dJ/dP, dP> (the seeds not used by J are zero)
    for (int q = 0; q < 3 && !rc; q++) {
      rc = dot(c, 0, bankp(c, ADJ, VFS_UCAT, q), bankp(c, TAN, VFS_UCAT, q), &t);
      d += t;
    }
    if (!rc && o->objective != VFS_OBJ_KINETIC_ENERGY) {
      rc = dot(c, 0, bankp(c, ADJ, VFS_P, 0), bankp(c, TAN, VFS_P, 0), &t);
      d += t;
    }
  }
  *dJ = d;
  zero_bank(c, ADJ);
  cudaStreamSynchronize(c->stream);
  cudaFree(dev);
  load_state(c, ckpt(c, 0), h0);
  cudaStreamSynchronize(c->stream);
  return rc;
}

static int gradient_run(Ctx *c, const vfs_adjoint_opts *o, double *grad, vfs_adjoint_stats *stats) {
  int rc;
  if ((rc = prepare(c, o))) return rc;
  Adjoint &A = *c->adj;
  const int n = o->nsteps, every = checkpoint_every(o);
  const int nseg = (n + every - 1) / every;
  if ((rc = ensure_tapes(c, std::min(every, n)))) return rc;
  std::vector<HostState> hs(nseg);
  if (!A.t0) cudaEventCreate(&A.t0);
  if (!A.t1) cudaEventCreate(&A.t1);
  A.it_fwd = A.n_fwd = A.it_adj = A.n_adj = 0;
  cudaEventRecord(A.t0, c->stream);
  for (int sg = 0; sg < nseg && !rc; sg++) {
    save_state(c, ckpt(c, sg), hs[sg], sg == 0);
    for (int s = 0; s < std::min(every, n - sg * every) && !rc; s++) rc = step_forward(c, o, nullptr);
  }
  double J = 0;
  if (!rc) {
    zero_bank(c, ADJ);
    rc = objective(c, o->objective, true, &J);
  }
  cudaEventRecord(A.t1, c->stream);
  cudaEventSynchronize(A.t1);
  float msf = 0;
  cudaEventElapsedTime(&msf, A.t0, A.t1);
  cudaEventRecord(A.t0, c->stream);
  int recomputed = 0;
  for (int sg = nseg - 1; sg >= 0 && !rc; sg--) {
    const int len = std::min(every, n - sg * every);
    load_state(c, ckpt(c, sg), hs[sg]);
    for (int s = 0; s < len && !rc; s++, recomputed++) rc = step_forward(c, o, &A.tapes[s]);
    for (int s = len - 1; s >= 0 && !rc; s--) rc = adjoint_step(c, A.tapes[s], &o->solve);
  }
  cudaEventRecord(A.t1, c->stream);
  cudaEventSynchronize(A.t1);
  float msa = 0;
  cudaEventElapsedTime(&msa, A.t0, A.t1);
  const size_t nc = control_size(c, o->control);
  double *dev = nullptr;
  if (!rc && cudaMalloc(&dev, sizeof(double) * nc) != cudaSuccess) rc = set_err(c, VFS_ERR_CUDA, "adjoint: allocation failed");
  if (!rc) {
    if (o->control == VFS_CTRL_INITIAL_UCONT) {
      V3 l = bank3(c, ADJ, VFS_UCONT);
      c->launches++, k_soa_to_aos<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g.N, dev, l.x, l.y, l.z);
    } else {
      cudaMemcpyAsync(dev, A.plane[ADJ], sizeof(double) * nc, cudaMemcpyDeviceToDevice, c->stream);
    }
    cudaMemcpyAsync(grad, dev, sizeof(double) * nc, cudaMemcpyDeviceToHost, c->stream);
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(dev);
  zero_bank(c, ADJ);
  load_state(c, ckpt(c, 0), hs[0]);
  cudaStreamSynchronize(c->stream);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->J = J;
    stats->ms_forward = msf;
    stats->ms_adjoint = msa;
    stats->recomputed_steps = recomputed;
    stats->checkpoints = nseg;
    stats->tape_bytes = (long long)A.tapes.size() * (24 + (c->g.immersed ? 3 : 0)) * (long long)sizeof(double) * c->g.N;
    stats->poisson_iterations_forward = A.n_fwd ? (double)A.it_fwd / A.n_fwd : 0.0;
    stats->poisson_iterations_adjoint = A.n_adj ? (double)A.it_adj / A.n_adj : 0.0;
  }
  return rc;
}

// One operator on host vectors (slot-major, N per slot): L x by its forward kernels and
// L^T y by the transpose the adjoint sweep applies (hand-written where the operator has
// one, else measured; measured: always the measured matrix), for the dot-product test
// <y, L x> = <L^T y, x> and the comparison of the two transposes.
static int op_check(Ctx *c, int o, const double *x, const double *y, double *Lx, double *LTy, bool measured) {
  int rc;
  if ((rc = adjoint_setup(c))) return rc;
  Adjoint &A = *c->adj;
  if (o < 0 || o >= OP_N || A.op[o].nslot == 0) return set_err(c, VFS_ERR_INVALID, "adjoint: no such operator here");
  LinOp &op = A.op[o];
  const long long N = c->g.N;
  const size_t bytes = sizeof(double) * N;
  zero_bank(c, TAN);
  zero_bank(c, ADJ);
  for (int s = 0; s < op.nslot; s++) {
    if (x) cudaMemcpyAsync(A.bank[TAN][op.slot[s].field][op.slot[s].comp], x + s * N, bytes, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(A.bank[ADJ][op.slot[s].field][op.slot[s].comp], y + s * N, bytes, cudaMemcpyHostToDevice, c->stream);
  }
  rc = x ? apply_op(c, o, TAN, 0) : VFS_OK;
  if (!rc) rc = adjoint_apply(c, o, measured);
  for (int s = 0; s < op.nslot && !rc; s++) {
    if (Lx) cudaMemcpyAsync(Lx + s * N, A.bank[TAN][op.slot[s].field][op.slot[s].comp], bytes, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(LTy + s * N, A.bank[ADJ][op.slot[s].field][op.slot[s].comp], bytes, cudaMemcpyDeviceToHost, c->stream);
  }
  cudaStreamSynchronize(c->stream);
  zero_bank(c, TAN);
  zero_bank(c, ADJ);
  cudaStreamSynchronize(c->stream);
  return rc;
}

static int op_info(Ctx *c, int o, int *nslot, int *fields, long long *nnz) {
  int rc;
  if ((rc = adjoint_setup(c))) return rc;
  Adjoint &A = *c->adj;
  if (o < 0 || o >= OP_N) return set_err(c, VFS_ERR_INVALID, "adjoint: no such operator");
  *nslot = A.op[o].nslot;
  for (int s = 0; s < A.op[o].nslot && fields; s++) {
    fields[2 * s] = A.op[o].slot[s].field;
    fields[2 * s + 1] = A.op[o].slot[s].comp;
  }
  if (nnz) *nnz = A.op[o].nnz;
  return VFS_OK;
}

}  // namespace vfs

using namespace vfs;

extern "C" {

#define VFS_ADJ_REQUIRE(c)                                                                      \
  do {                                                                                          \
    if (!(c)) return set_err(nullptr, VFS_ERR_INVALID, "null context");                        \
    if (!(c)->metrics_set || !(c)->nvert_set)                                                   \
      return set_err((c), VFS_ERR_STATE, "adjoint: metrics and nvert must be uploaded first"); \
    cudaSetDevice((c)->device);                                                                 \
  } while (0)

int vfs_adjoint_setup(vfs_ctx *ctx) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  return adjoint_setup(c);
}

int vfs_objective(vfs_ctx *ctx, const vfs_adjoint_opts *opts, double *J) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!J) return set_err(c, VFS_ERR_INVALID, "vfs_objective: null J");
  return objective_run(c, opts, J);
}

int vfs_tangent(vfs_ctx *ctx, const vfs_adjoint_opts *opts, const double *dir, double *J, double *dJ) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!dir || !J || !dJ) return set_err(c, VFS_ERR_INVALID, "vfs_tangent: null argument");
  return tangent_run(c, opts, dir, J, dJ);
}

int vfs_adjoint_gradient(vfs_ctx *ctx, const vfs_adjoint_opts *opts, double *grad, vfs_adjoint_stats *stats) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!grad) return set_err(c, VFS_ERR_INVALID, "vfs_adjoint_gradient: null gradient");
  return gradient_run(c, opts, grad, stats);
}

int vfs_adjoint_op_info(vfs_ctx *ctx, int op, int *nslot, int *fields, long long *nnz) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!nslot) return set_err(c, VFS_ERR_INVALID, "vfs_adjoint_op_info: null argument");
  return op_info(c, op, nslot, fields, nnz);
}

int vfs_adjoint_op_check(vfs_ctx *ctx, int op, const double *x, const double *y, double *Lx, double *LTy) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!x || !y || !Lx || !LTy) return set_err(c, VFS_ERR_INVALID, "vfs_adjoint_op_check: null argument");
  return op_check(c, op, x, y, Lx, LTy, false);
}

int vfs_adjoint_op_measured(vfs_ctx *ctx, int op, const double *y, double *LTy) {
  Ctx *c = (Ctx *)ctx;
  VFS_ADJ_REQUIRE(c);
  if (!y || !LTy) return set_err(c, VFS_ERR_INVALID, "vfs_adjoint_op_measured: null argument");
  return op_check(c, op, nullptr, y, nullptr, LTy, true);
}

}  // extern "C"
