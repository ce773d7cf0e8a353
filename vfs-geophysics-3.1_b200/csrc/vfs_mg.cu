// Geometric multigrid preconditioner of the pressure-Poisson solve (one V-cycle per
// FGMRES iteration), FP32 or FP64.
//
// The reference preconditions its Krylov solve with HYPRE BoomerAMG
// (poisson_hypre.c:26-88); this is a B200-first geometric replacement, not a port:
//
//   * Levels are cell-centred and coarsened by 2 in every direction while all interior
//     dimensions are even and at least 4 (256x192x256 -> ... -> 4x3x4: seven levels).
//   * Every level, the finest included, smooths with the 7-point conductance form of the
//     operator: the coupling of two unknowns across a face is the symmetrised, clipped
//     main-term coefficient of the reference's 19-point row (exactly the operator on
//     orthogonal grids, where the reference's filter drops every cross term).  A coarse
//     face conducts 0.5 x the sum of the four fine faces it covers; diagonals are minus
//     the sum of a cell's couplings, so every level is a consistent Neumann operator.
//   * Smoother: line Gauss-Seidel along j (the wall-normal, most strongly coupled
//     direction of the channel grids) in zebra order: the columns with (i+k) even are
//     solved first, then the odd ones, so each column's i/k neighbours are fixed while it
//     is solved and the update is in place and deterministic.  The tridiagonal factors
//     (Thomas forward coefficients and pivots) are precomputed once per operator.
//   * Restriction sums the residuals of the 8 children; prolongation is cell-centred
//     trilinear (weights 27/64, 9/64, 3/64, 1/64), a missing or inactive coarse
//     neighbour giving its weight to the parent.  With these transfers the FGMRES
//     iteration count stays flat as the grid is refined.
//
// Layout: every level stores its cells in "zebra" order, ((k*ny + j)*2 + colour)*hx + i/2
// with colour = (i xor k) & 1 and hx = ceil(nx/2), so the columns of one colour are
// contiguous half-rows and each colour pass reads and writes with unit stride.  The
// finest level is indexed by interior cell (DA index minus one); conversion to and from
// the solver's DA-layout FP64 vectors happens once per V-cycle.
//
// A level with an odd number of cells along a periodic i or k direction cannot be two-
// coloured; it is smoothed by damped (0.8) line Jacobi instead.
#include <algorithm>
#include <cmath>

#include "vfs_internal.cuh"

namespace vfs {

enum { OP_CE = 0, OP_CN, OP_CT, OP_DG, OP_CPR, OP_IDEN, NOP };

// 32-bit index arithmetic: mg_setup refuses levels of 2^31 slots or more.
__host__ __device__ inline long long zidx(const ZL &L, int i, int j, int k) {
  return (long long)((((unsigned)k * (unsigned)L.ny + (unsigned)j) * 2u + (unsigned)((i ^ k) & 1)) * (unsigned)L.hx +
                     (unsigned)(i >> 1));
}

// Cell (i, j, k) of a level from its natural index t = (k*ny + j)*nx + i.
__device__ __forceinline__ void zcell(const ZL &L, long long t, int &i, int &j, int &k) {
  const unsigned ut = (unsigned)t, nx = (unsigned)L.nx, ny = (unsigned)L.ny;
  const unsigned r = ut / nx;
  i = (int)(ut - r * nx);
  const unsigned kk = r / ny;
  j = (int)(r - kk * ny);
  k = (int)kk;
}

// Programmatic dependent launch along the V-cycle's chain of short kernels: each kernel
// lets its successor be scheduled as soon as all its own blocks have started, then waits
// for its predecessor grid to complete (and its writes to be visible) before touching
// memory, so the launch gap between kernels overlaps the tail of the previous one and
// the results are those of plain stream order.  Outside such a launch both are no-ops.
#ifndef VFS_PDL
#define VFS_PDL 1
#endif
__device__ __forceinline__ void pdl_prologue() {
#if VFS_PDL
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
// Inside a captured step the chain is launched plainly: captured with programmatic
// dependent launch (VFS_PDL_CAPTURE 1) the same graph ran 0.5 ms per step slower on the B200
// (35.9 against 36.4 ms at 256 x 192 x 256).
#ifndef VFS_PDL_CAPTURE
#define VFS_PDL_CAPTURE 0
#endif
// Every launch is counted in the context's launch counter and its status is checked: the
// return value of cudaLaunchKernelEx, then the sticky launch error.
template <typename... KArgs, typename... Args>
static int launch_chain(Ctx *c, const char *what, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                        Args... args) {
  c->launches++;
#if VFS_PDL
  if (c->capturing && !VFS_PDL_CAPTURE) {  // plain launches inside a captured step
    kernel<<<grid, block, smem, c->stream>>>(static_cast<KArgs>(args)...);
    return check_launch(c, what);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(c, VFS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
#else
  kernel<<<grid, block, smem, c->stream>>>(static_cast<KArgs>(args)...);
#endif
  return check_launch(c, what);
}

// ------------------------------------------------------------------ set-up (FP64)
// Fine-level couplings from the reference operator (19 slots on the DA layout).
__global__ void k_mg_fine_couplings(Grid g, ZL L, const double *__restrict__ coef, const uint8_t *__restrict__ fluid,
                                    double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  const long long N = g.N;
  const long long p = lidx(g, i + 1, j + 1, k + 1);
  const long long q = zidx(L, i, j, k);
  double ce = 0, cn = 0, ct = 0;
  if (fluid[p]) {
    if (i + 1 < L.nx || L.ip) {
      const long long e = lidx(g, wrapi(g, i + 2), j + 1, k + 1);
      if (fluid[e]) ce = fmax(0.0, 0.5 * (coef[EP * N + p] + coef[WP * N + e]));
    }
    if (j + 1 < L.ny || L.jp) {
      const long long e = lidx(g, i + 1, wrapj(g, j + 2), k + 1);
      if (fluid[e]) cn = fmax(0.0, 0.5 * (coef[NP * N + p] + coef[SP * N + e]));
    }
    if (k + 1 < L.nz || L.kp) {
      const long long e = lidx(g, i + 1, j + 1, wrapk(g, k + 2));
      if (fluid[e]) ct = fmax(0.0, 0.5 * (coef[TP * N + p] + coef[BP * N + e]));
    }
  }
  op[OP_CE * L.n + q] = ce;
  op[OP_CN * L.n + q] = cn;
  op[OP_CT * L.n + q] = ct;
}

// Coarse couplings: 0.5 x the sum of the four fine couplings across each coarse face.
__global__ void k_mg_coarse_couplings(ZL F, ZL C, const double *__restrict__ opF, double *__restrict__ opC) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)C.nx * C.ny * C.nz;
  if (t >= ncell) return;
  const int I = (int)(t % C.nx);
  const long long r = t / C.nx;
  const int J = (int)(r % C.ny), K = (int)(r / C.ny);
  double sx = 0, sy = 0, sz = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      sx += opF[OP_CE * F.n + zidx(F, 2 * I + 1, 2 * J + u, 2 * K + v)];
      sy += opF[OP_CN * F.n + zidx(F, 2 * I + u, 2 * J + 1, 2 * K + v)];
      sz += opF[OP_CT * F.n + zidx(F, 2 * I + u, 2 * J + v, 2 * K + 1)];
    }
  const long long q = zidx(C, I, J, K);
  opC[OP_CE * C.n + q] = 0.5 * sx;
  opC[OP_CN * C.n + q] = 0.5 * sy;
  opC[OP_CT * C.n + q] = 0.5 * sz;
}

// Neighbour cells of (i,j,k) with the level's periodic wrap; -1 where there is none.
struct ZNb {
  int ie, iw, jn, js, kt, kb;
};
__device__ __forceinline__ ZNb znb(const ZL &L, int i, int j, int k) {
  ZNb r;
  r.ie = i + 1 < L.nx ? i + 1 : (L.ip ? 0 : -1);
  r.iw = i > 0 ? i - 1 : (L.ip ? L.nx - 1 : -1);
  r.jn = j + 1 < L.ny ? j + 1 : (L.jp ? 0 : -1);
  r.js = j > 0 ? j - 1 : (L.jp ? L.ny - 1 : -1);
  r.kt = k + 1 < L.nz ? k + 1 : (L.kp ? 0 : -1);
  r.kb = k > 0 ? k - 1 : (L.kp ? L.nz - 1 : -1);
  return r;
}

__global__ void k_mg_diag(ZL L, double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  const long long q = zidx(L, i, j, k), n = L.n;
  const ZNb b = znb(L, i, j, k);
  double s = op[OP_CE * n + q] + op[OP_CN * n + q] + op[OP_CT * n + q];
  if (b.iw >= 0) s += op[OP_CE * n + zidx(L, b.iw, j, k)];
  if (b.js >= 0) s += op[OP_CN * n + zidx(L, i, b.js, k)];
  if (b.kb >= 0) s += op[OP_CT * n + zidx(L, i, j, b.kb)];
  op[OP_DG * n + q] = -s;
}

// Thomas factors of every j-line (the in-line couplings only; a periodic j wrap is left
// to the right-hand side): cpr_j = upper_j / den_j, iden_j = 1 / den_j,
// den_j = dg_j - lower_j * cpr_{j-1}.  Inactive or degenerate rows get zero factors, so
// the smoother leaves their unknown at zero.
__global__ void k_mg_thomas(ZL L, double *__restrict__ op) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)L.nx * L.nz) return;
  const int i = (int)(t % L.nx), k = (int)(t / L.nx);
  const long long n = L.n;
  double cprev = 0, lower = 0;
  for (int j = 0; j < L.ny; j++) {
    const long long q = zidx(L, i, j, k);
    const double dg = op[OP_DG * n + q];
    const double upper = j + 1 < L.ny ? op[OP_CN * n + q] : 0.0;
    double cpr = 0, iden = 0;
    if (dg != 0) {
      const double den = dg - lower * cprev;
      if (fabs(den) > 1e-12 * fabs(dg)) {
        iden = 1.0 / den;
        cpr = upper * iden;
      }
    }
    op[OP_CPR * n + q] = cpr;
    op[OP_IDEN * n + q] = iden;
    cprev = cpr;
    lower = upper;
  }
}

// ------------------------------------------------------------------ packed operator
// The smoother and the transfers read the operator as two 4-vectors per cell, so a
// row costs two vector loads: cpl = {ce, cw, ct, cb} (couplings to i+1, i-1, k+1, k-1)
// and tri = {cs, iden, cpr, dg} (coupling to j-1, Thomas pivot inverse and factor,
// diagonal).  A missing neighbour has a zero coupling; cs at j = 0 is the periodic
// wrap coupling when j is periodic, else 0.
template <typename T>
struct __align__(4 * sizeof(T)) Q4 {
  T a, b, c, d;
};
template <typename T>
struct __align__(2 * sizeof(T)) Q2 {
  T a, b;
};

template <typename T>
__global__ void k_mg_pack(ZL L, const double *__restrict__ op, Q4<T> *__restrict__ cpl, Q4<T> *__restrict__ tri) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  const int i = (int)(t % L.nx);
  const long long r = t / L.nx;
  const int j = (int)(r % L.ny), k = (int)(r / L.ny);
  const long long q = zidx(L, i, j, k), n = L.n;
  const ZNb nb = znb(L, i, j, k);
  Q4<T> a, b;
  a.a = (T)op[OP_CE * n + q];
  a.b = nb.iw >= 0 ? (T)op[OP_CE * n + zidx(L, nb.iw, j, k)] : T(0);
  a.c = (T)op[OP_CT * n + q];
  a.d = nb.kb >= 0 ? (T)op[OP_CT * n + zidx(L, i, j, nb.kb)] : T(0);
  b.a = nb.js >= 0 ? (T)op[OP_CN * n + zidx(L, i, nb.js, k)] : T(0);
  b.b = (T)op[OP_IDEN * n + q];
  b.c = (T)op[OP_CPR * n + q];
  b.d = (T)op[OP_DG * n + q];
  cpl[q] = a;
  tri[q] = b;
}

// ------------------------------------------------------------------ smoother
// One colour pass of zebra line Gauss-Seidel (colour 0/1; x read for the other colour,
// written for this one), or, with colour < 0, one damped line-Jacobi sweep over all
// columns (neighbours read from xr = the previous iterate, a separate array).
// x_zero: the neighbours read are known to be zero (first pass from a zero guess).
// The forward elimination stores (d'_j, cpr_j) in ds; the back substitution writes x.
// Rows are processed in chunks of CH: every load of a chunk is issued before the
// recurrence consumes the first one, so a column keeps CH rows of loads in flight.
template <typename T, int CH>
__device__ __forceinline__ void zline_column(const ZL &L, const Q4<T> *__restrict__ cpl, const Q4<T> *__restrict__ tri,
                                             const T *__restrict__ b, const T *__restrict__ xr,
                                             Q2<T> *__restrict__ ds, T *__restrict__ xw, int colour, T omega,
                                             int x_zero, long long t) {
  const int hx = L.hx;
  int c, h, k;
  if (colour >= 0) {
    if (t >= (long long)L.nz * hx) return;
    h = (int)(t % hx); k = (int)(t / hx); c = colour;
  } else {
    if (t >= 2LL * L.nz * hx) return;
    h = (int)(t % hx); c = (int)((t / hx) & 1); k = (int)(t / (2LL * hx));
  }
  const int i = 2 * h + (c ^ (k & 1));
  if (i >= L.nx) return;
  const ZNb nb = znb(L, i, 0, k);
  const long long p0 = zidx(L, i, 0, k);
  // offsets of the neighbour columns (constant along j).  A missing neighbour (domain
  // edge, zero coupling) borrows the offset of the opposite one, so every x read is of
  // the other colour (every level has at least 2 cells along i and k).
  const long long oe = zidx(L, nb.ie >= 0 ? nb.ie : nb.iw, 0, k) - p0;
  const long long ow = zidx(L, nb.iw >= 0 ? nb.iw : nb.ie, 0, k) - p0;
  const long long ot = zidx(L, i, 0, nb.kt >= 0 ? nb.kt : nb.kb) - p0;
  const long long ob = zidx(L, i, 0, nb.kb >= 0 ? nb.kb : nb.kt) - p0;
  const long long sj = 2LL * hx;
  const int ny = L.ny;
  // periodic j: the wrap coupling and the far end of the own column (old values)
  T wrap_c = 0, x_first = 0, x_last = 0;
  if (L.jp && !x_zero) {
    const T *__restrict__ xs = colour >= 0 ? xw : xr;
    wrap_c = tri[p0].a;
    x_first = xs[p0];
    x_last = xs[p0 + (ny - 1) * sj];
  }
  T dprev = 0;
  for (int j0 = 0; j0 < ny; j0 += CH) {
    T bb[CH], xe[CH], xwv[CH], xt[CH], xb[CH];
    Q4<T> cp[CH], tr[CH];
#pragma unroll
    for (int u = 0; u < CH; u++) {
      const int j = j0 + u;
      if (j < ny) {
        const long long q = p0 + j * sj;
        bb[u] = b[q];
        tr[u] = tri[q];
        if (!x_zero) {
          cp[u] = cpl[q];
          xe[u] = xr[q + oe];
          xwv[u] = xr[q + ow];
          xt[u] = xr[q + ot];
          xb[u] = xr[q + ob];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < CH; u++) {
      const int j = j0 + u;
      if (j < ny) {
        T r = bb[u];
        if (!x_zero) {
          r -= cp[u].a * xe[u];
          r -= cp[u].b * xwv[u];
          r -= cp[u].c * xt[u];
          r -= cp[u].d * xb[u];
          if (L.jp) {
            if (j == 0) r -= wrap_c * x_last;
            if (j == ny - 1) r -= wrap_c * x_first;
          }
        }
        const T lower = j > 0 ? tr[u].a : T(0);
        const T d = (r - lower * dprev) * tr[u].b;
        Q2<T> o;
        o.a = d; o.b = tr[u].c;
        ds[p0 + j * sj] = o;
        dprev = d;
      }
    }
  }
  T xnext = 0;
  for (int j1 = ny - 1; j1 >= 0; j1 -= CH) {
    Q2<T> dd[CH];
    T xo[CH];
#pragma unroll
    for (int u = 0; u < CH; u++) {
      const int j = j1 - u;
      if (j >= 0) {
        dd[u] = ds[p0 + j * sj];
        if (colour < 0 && !x_zero) xo[u] = xr[p0 + j * sj];
      }
    }
#pragma unroll
    for (int u = 0; u < CH; u++) {
      const int j = j1 - u;
      if (j >= 0) {
        const T v = dd[u].a - dd[u].b * xnext;
        xnext = v;
        T out = v;
        if (colour < 0) out = x_zero ? omega * v : xo[u] + omega * (v - xo[u]);
        xw[p0 + j * sj] = out;
      }
    }
  }
}

template <typename T> struct ZChunk;
template <> struct ZChunk<float> { static constexpr int v = 8; };
template <> struct ZChunk<double> { static constexpr int v = 4; };

template <typename T>
__global__ void __launch_bounds__(64) k_zline(ZL L, const Q4<T> *__restrict__ cpl, const Q4<T> *__restrict__ tri,
                                              const T *__restrict__ b, const T *__restrict__ xr,
                                              Q2<T> *__restrict__ ds, T *__restrict__ xw, int colour, T omega,
                                              int x_zero) {
  zline_column<T, ZChunk<T>::v>(L, cpl, tri, b, xr, ds, xw, colour, omega, x_zero,
                                blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// Tiled zebra colour pass for the large levels.  One thread block owns W columns of
// one colour that are consecutive in memory (same k, half-row positions h0..h0+W-1):
//   A. all threads load the tile's rows (coalesced across the W columns, many loads in
//      flight) and form each row's scaled right-hand side r' = r / pivot, the scaled
//      lower coupling m = lower / pivot and the Thomas factor cpr, in shared memory;
//   B. each warp solves whole columns: the forward elimination d_j = r'_j - m_j d_{j-1}
//      and the back substitution x_j = d_j - cpr_j x_{j+1} are first-order linear
//      recurrences, evaluated as warp scans (each lane composes its run of rows, a
//      5-step shuffle scan combines the lanes, each lane then replays its rows);
//   C. all threads write the tile's x back, coalesced.
// Shared memory: 3 * W * P values of T, P = ny rounded up to odd (conflict-free rows).
#ifndef VFS_ZTILE_THREADS
#define VFS_ZTILE_THREADS 256
#endif
#ifndef VFS_ZTILE_W32
#define VFS_ZTILE_W32 16   // columns per tile, FP32
#endif
#ifndef VFS_ZTILE_W64
#define VFS_ZTILE_W64 8    // columns per tile, FP64
#endif
#ifndef VFS_ZTILE_U32
#define VFS_ZTILE_U32 1    // rows each thread loads before using them, FP32
#endif
// Measured at 256 x 192 x 256 (V-cycle ms, FP32 / FP64): FP32 rows per thread 1 1.42,
// 2 1.46, 4 1.78; FP32 columns 8 1.45, 16 1.46, 32 2.02; FP32 blocks per SM 3 1.62, 4 1.48,
// 5 1.46, 6 1.77; FP64 columns 8 2.20, 16 2.27, 32 2.75.
#ifndef VFS_ZTILE_MINB
#define VFS_ZTILE_MINB 5   // resident blocks per SM the register allocation must allow, FP32
#endif
#ifndef VFS_ZTILE_MINB64
#define VFS_ZTILE_MINB64 1  // the same, FP64
#endif
constexpr int kTileThreads = VFS_ZTILE_THREADS;

template <typename T>
__device__ __forceinline__ void scan_compose_up(T &A, T &B, int lane) {
  // inclusive scan over lanes 0..lane of x -> A x + B maps (later lanes applied last)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T pa = __shfl_up_sync(0xffffffffu, A, off), pb = __shfl_up_sync(0xffffffffu, B, off);
    if (lane >= off) { B = A * pb + B; A = A * pa; }
  }
}
template <typename T>
__device__ __forceinline__ void scan_compose_down(T &A, T &B, int lane) {
  // inclusive scan over lanes lane..31 (higher lanes applied first)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T pa = __shfl_down_sync(0xffffffffu, A, off), pb = __shfl_down_sync(0xffffffffu, B, off);
    if (lane + off < 32) { B = A * pb + B; A = A * pa; }
  }
}

template <typename T, int W>
__global__ void __launch_bounds__(kTileThreads, sizeof(T) == 4 ? VFS_ZTILE_MINB : VFS_ZTILE_MINB64) k_zline_tile(ZL L, const Q4<T> *__restrict__ cpl,
                                                             const Q4<T> *__restrict__ tri, const T *__restrict__ b,
                                                             const T *__restrict__ xr, T *__restrict__ xw, int colour,
                                                             int x_zero) {
  pdl_prologue();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int hx = L.hx, ny = L.ny;
  const int P = ny | 1;
  T *sr = reinterpret_cast<T *>(smem_raw);  // [W][P]: r', then d, then x
  T *sm = sr + W * P;                        // [W][P]: m
  T *sc = sm + W * P;                        // [W][P]: cpr
  const int tiles_per_row = (hx + W - 1) / W;
  const int k = blockIdx.x / tiles_per_row;
  const int h0 = (blockIdx.x % tiles_per_row) * W;
  if (k >= L.nz) return;
  const long long sj = 2LL * hx;
  // A: the block size is a multiple of W, so each thread keeps one column and takes
  // every (blockDim/W)-th row; U rows are loaded before any of them is used.
  {
    constexpr int U = sizeof(T) == 4 ? VFS_ZTILE_U32 : 3;
    const int w = threadIdx.x % W, jstep = blockDim.x / W;
    const int h = h0 + w;
    const int i = 2 * h + (colour ^ (k & 1));
    const bool valid = h < hx && i < L.nx;
    const int ic = valid ? i : (colour ^ (k & 1));  // a real column for the address arithmetic
    const ZNb nb = znb(L, ic, 0, k);
    const long long p0 = zidx(L, ic, 0, k);
    const long long oe = zidx(L, nb.ie >= 0 ? nb.ie : nb.iw, 0, k) - p0;
    const long long ow = zidx(L, nb.iw >= 0 ? nb.iw : nb.ie, 0, k) - p0;
    const long long ot = zidx(L, ic, 0, nb.kt >= 0 ? nb.kt : nb.kb) - p0;
    const long long ob = zidx(L, ic, 0, nb.kb >= 0 ? nb.kb : nb.kt) - p0;
    for (int jb = threadIdx.x / W; jb < ny; jb += U * jstep) {
      T bb[U], xe[U], xwv[U], xt[U], xb[U];
      Q4<T> tr[U], cp[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int j = jb + u * jstep;
        if (valid && j < ny) {
          const long long q = p0 + j * sj;
          bb[u] = b[q];
          tr[u] = tri[q];
          if (!x_zero) {
            cp[u] = cpl[q];
            xe[u] = xr[q + oe];
            xwv[u] = xr[q + ow];
            xt[u] = xr[q + ot];
            xb[u] = xr[q + ob];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int j = jb + u * jstep;
        if (j >= ny) continue;
        T rr = 0, mm = 0, cc = 0;
        if (valid) {
          T r = bb[u];
          if (!x_zero) {
            // a missing neighbour has a zero coupling (its offset is the opposite one's)
            r -= cp[u].a * xe[u];
            r -= cp[u].b * xwv[u];
            r -= cp[u].c * xt[u];
            r -= cp[u].d * xb[u];
            if (L.jp) {
              if (j == 0) r -= tr[u].a * xw[p0 + (ny - 1) * sj];
              if (j == ny - 1) r -= tri[p0].a * xw[p0];
            }
          }
          rr = r * tr[u].b;
          mm = j > 0 ? tr[u].a * tr[u].b : T(0);
          cc = tr[u].c;
        }
        sr[w * P + j] = rr;
        sm[w * P + j] = mm;
        sc[w * P + j] = cc;
      }
    }
  }
  __syncthreads();
  // B
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int seg = (ny + 31) >> 5;
  const int j0 = lane * seg, j1 = min(ny, j0 + seg);
  for (int w = warp; w < W; w += nwarp) {
    T *cr = sr + w * P;
    const T *cm = sm + w * P, *cx = sc + w * P;
    // forward: d_j = -m_j d_{j-1} + r'_j
    T A = 1, B = 0;
    for (int j = j0; j < j1; j++) { const T mj = cm[j]; B = -mj * B + cr[j]; A = -mj * A; }
    scan_compose_up<T>(A, B, lane);
    T d = __shfl_up_sync(0xffffffffu, B, 1);
    if (lane == 0) d = 0;
    for (int j = j0; j < j1; j++) { d = -cm[j] * d + cr[j]; cr[j] = d; }
    __syncwarp();
    // backward: x_j = -cpr_j x_{j+1} + d_j
    A = 1; B = 0;
    for (int j = j1 - 1; j >= j0; j--) { const T cj = cx[j]; B = -cj * B + cr[j]; A = -cj * A; }
    scan_compose_down<T>(A, B, lane);
    T x = __shfl_down_sync(0xffffffffu, B, 1);
    if (lane == 31) x = 0;
    for (int j = j1 - 1; j >= j0; j--) { x = -cx[j] * x + cr[j]; cr[j] = x; }
    __syncwarp();
  }
  __syncthreads();
  // C
  for (int e = threadIdx.x; e < ny * W; e += blockDim.x) {
    const int j = e / W, w = e - (e / W) * W;
    const int h = h0 + w;
    const int i = 2 * h + (colour ^ (k & 1));
    if (h < hx && i < L.nx) xw[zidx(L, i, j, k)] = sr[w * P + j];
  }
}

template <typename T, int W>
static size_t tile_smem(int ny) {
  return (size_t)3 * W * (ny | 1) * sizeof(T);
}
template <typename T, int W>
static bool tile_fits(int ny) {
  return tile_smem<T, W>(ny) <= 200 * 1024;
}

// Residual b - A x at one cell of a level.
template <typename T>
__device__ __forceinline__ T zresid(const ZL &L, const Q4<T> *__restrict__ cpl, const Q4<T> *__restrict__ tri,
                                    const T *__restrict__ x, const T *__restrict__ b, int i, int j, int k,
                                    long long q) {
  const ZNb nb = znb(L, i, j, k);
  const Q4<T> cp = cpl[q], tr = tri[q];
  T ax = tr.d * x[q];
  if (nb.ie >= 0) ax += cp.a * x[zidx(L, nb.ie, j, k)];
  if (nb.iw >= 0) ax += cp.b * x[zidx(L, nb.iw, j, k)];
  if (nb.js >= 0) ax += tr.a * x[zidx(L, i, nb.js, k)];
  if (nb.jn >= 0) { const long long s = zidx(L, i, nb.jn, k); ax += tri[s].a * x[s]; }
  if (nb.kt >= 0) ax += cp.c * x[zidx(L, i, j, nb.kt)];
  if (nb.kb >= 0) ax += cp.d * x[zidx(L, i, j, nb.kb)];
  return b[q] - ax;
}

// Coarse right-hand side: the sum of the residuals of the (active) children.  With
// colour0_only the children of colour 1 ((i xor k) odd) are left out: after a zebra sweep
// that ends with the colour-1 pass their line equations hold exactly (the j-line solve is
// exact when j is not periodic), so their residuals are rounding only.
template <typename T>
__device__ __forceinline__ void zrestrict_cell(const ZL &F, const ZL &C, const Q4<T> *__restrict__ cpl,
                                              const Q4<T> *__restrict__ tri, const T *__restrict__ x,
                                              const T *__restrict__ b, T *__restrict__ bc, long long t,
                                              bool colour0_only = false) {
  const long long ncell = (long long)C.nx * C.ny * C.nz;
  if (t >= ncell) return;
  int I, J, K;
  zcell(C, t, I, J, K);
  // every child's residual is formed (all its loads are in range) and an inactive child's
  // left out by a select, so the loads of all children are in flight together
  T s = 0;
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int bb = 0; bb < 2; bb++)
#pragma unroll
      for (int a = 0; a < 2; a++) {
        if (colour0_only && a != c) continue;
        const int i = 2 * I + a, j = 2 * J + bb, k = 2 * K + c;
        const long long q = zidx(F, i, j, k);
        const T r = zresid<T>(F, cpl, tri, x, b, i, j, k, q);
        if (tri[q].d != T(0)) s += r;
      }
  bc[zidx(C, I, J, K)] = s;
}

template <typename T, bool kColour0>
__global__ void k_zrestrict(ZL F, ZL C, const Q4<T> *__restrict__ cpl, const Q4<T> *__restrict__ tri,
                            const T *__restrict__ x, const T *__restrict__ b, T *__restrict__ bc) {
  pdl_prologue();
  zrestrict_cell<T>(F, C, cpl, tri, x, b, bc, blockIdx.x * (long long)blockDim.x + threadIdx.x, kColour0);
}

// x_fine += P x_coarse (cell-centred trilinear).
template <typename T>
__device__ __forceinline__ void zprolong_cell(const ZL &F, const ZL &C, const uint8_t *__restrict__ actF,
                                             const uint8_t *__restrict__ actC, T *__restrict__ x,
                                             const T *__restrict__ xc, long long t) {
  const long long ncell = (long long)F.nx * F.ny * F.nz;
  if (t >= ncell) return;
  int i, j, k;
  zcell(F, t, i, j, k);
  const long long q = zidx(F, i, j, k);
  if (!actF[q]) return;
  const int I = i >> 1, J = j >> 1, K = k >> 1;
  // the other coarse cell nearest along each direction, or -1
  int In = I + ((i & 1) ? 1 : -1), Jn = J + ((j & 1) ? 1 : -1), Kn = K + ((k & 1) ? 1 : -1);
  if (In < 0 || In >= C.nx) In = C.ip ? (In + C.nx) % C.nx : -1;
  if (Jn < 0 || Jn >= C.ny) Jn = C.jp ? (Jn + C.ny) % C.ny : -1;
  if (Kn < 0 || Kn >= C.nz) Kn = C.kp ? (Kn + C.nz) % C.nz : -1;
  const long long own = zidx(C, I, J, K);
  // every load first (the flag and the value of each coarse neighbour are independent
  // loads), then the sums in a fixed order: the loads do not wait on the flags
  T v[8];
  bool ok[8];
#pragma unroll
  for (int n = 1; n < 8; n++) {
    const int a = n & 1, bb = (n >> 1) & 1, c = n >> 2;
    const int ii = a ? In : I, jj = bb ? Jn : J, kk = c ? Kn : K;
    const bool in = ii >= 0 && jj >= 0 && kk >= 0;
    const long long qc = in ? zidx(C, ii, jj, kk) : own;
    ok[n] = in && actC[qc];
    v[n] = xc[qc];
  }
  const T xo = xc[own], xq = x[q];
  T wown = T(27) / T(64);
  T s = 0;
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int bb = 0; bb < 2; bb++)
#pragma unroll
      for (int a = 0; a < 2; a++) {
        if (a + bb + c == 0) continue;
        const T w = (a ? T(1) : T(3)) * (bb ? T(1) : T(3)) * (c ? T(1) : T(3)) / T(64);
        const int n = a + 2 * bb + 4 * c;
        if (!ok[n]) { wown += w; continue; }
        s += w * v[n];
      }
  x[q] = xq + (s + wown * xo);
}

template <typename T>
__global__ void k_zprolong(ZL F, ZL C, const uint8_t *__restrict__ actF, const uint8_t *__restrict__ actC,
                           T *__restrict__ x, const T *__restrict__ xc) {
  pdl_prologue();
  zprolong_cell<T>(F, C, actF, actC, x, xc, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// The same prolongation from the coarse side: coarse cell t (natural index) loads its
// 3 x 3 x 3 neighbourhood (values and activity) once and updates its eight children, each
// child with zprolong_cell's neighbours, weights and order of summation, so the results are
// the same bits.  Needs a fine level of exactly twice the coarse cells in every direction.
template <typename T>
__device__ __forceinline__ void zprolong8_cell(const ZL &F, const ZL &C, const uint8_t *__restrict__ actF,
                                               const uint8_t *__restrict__ actC, T *__restrict__ x,
                                               const T *__restrict__ xc, long long t) {
  const long long nc = (long long)C.nx * C.ny * C.nz;
  if (t >= nc) return;
  int I, J, K;
  zcell(C, t, I, J, K);
  // neighbour index along one direction, wrapped on a periodic level, -1 beyond an edge
  auto nb = [](int v, int n, int per) { return (v >= 0 && v < n) ? v : (per ? (v + n) % n : -1); };
  const int Ii[3] = {nb(I - 1, C.nx, C.ip), I, nb(I + 1, C.nx, C.ip)};
  const int Jj[3] = {nb(J - 1, C.ny, C.jp), J, nb(J + 1, C.ny, C.jp)};
  const int Kk[3] = {nb(K - 1, C.nz, C.kp), K, nb(K + 1, C.nz, C.kp)};
  const long long own = zidx(C, I, J, K);
  T v[27];
  unsigned ok = 0;
#pragma unroll
  for (int e = 0; e < 27; e++) {
    const int a = e % 3, b = (e / 3) % 3, cc = e / 9;
    const bool in = Ii[a] >= 0 && Jj[b] >= 0 && Kk[cc] >= 0;
    const long long qc = in ? zidx(C, Ii[a], Jj[b], Kk[cc]) : own;
    v[e] = xc[qc];
    if (in && actC[qc]) ok |= 1u << e;
  }
  const T xo = v[13];
#pragma unroll
  for (int ch = 0; ch < 8; ch++) {
    const int ai = ch & 1, aj = (ch >> 1) & 1, ak = ch >> 2;
    const int i = 2 * I + ai, j = 2 * J + aj, k = 2 * K + ak;
    const long long q = zidx(F, i, j, k);
    if (!actF[q]) continue;
    // offset of the other nearest coarse cell: +1 for an odd child index, -1 for an even one
    const int di = ai ? 2 : 0, dj = aj ? 2 : 0, dk = ak ? 2 : 0;
    const T xq = x[q];
    T wown = T(27) / T(64);
    T s = 0;
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int bb = 0; bb < 2; bb++)
#pragma unroll
        for (int a = 0; a < 2; a++) {
          if (a + bb + c == 0) continue;
          const T w = (a ? T(1) : T(3)) * (bb ? T(1) : T(3)) * (c ? T(1) : T(3)) / T(64);
          const int e = (a ? di : 1) + 3 * (bb ? dj : 1) + 9 * (c ? dk : 1);
          if (!((ok >> e) & 1u)) { wown += w; continue; }
          s += w * v[e];
        }
    x[q] = xq + (s + wown * xo);
  }
}

template <typename T>
__global__ void k_zprolong8(ZL F, ZL C, const uint8_t *__restrict__ actF, const uint8_t *__restrict__ actC,
                            T *__restrict__ x, const T *__restrict__ xc) {
  pdl_prologue();
  zprolong8_cell<T>(F, C, actF, actC, x, xc, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// act[q] = 1 where the level's diagonal is non-zero (an active unknown).
__global__ void k_mg_active(long long n, const double *__restrict__ op, uint8_t *__restrict__ act) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q < n) act[q] = op[OP_DG * n + q] != 0.0 ? 1 : 0;
}

// ------------------------------------------------------------------ bottom of the V-cycle
// The coarse levels are too small to fill the GPU, and a launch per colour pass costs
// more than the work.  From the first level of at most kBottomCells cells down, one thread
// block runs the rest of the V-cycle (smoothing, restriction, coarsest sweeps,
// prolongation) with block barriers between the phases; the level data stay in L2.  On the
// B200 at 256 x 192 x 256 (V-cycle ms, FP32 / FP64): 512 cells (the 8 x 6 x 8 level down)
// 1.450 / 2.268, 4096 or 8192 1.470 / 2.313, 32768 1.772 / 2.738.
constexpr int kBottomMaxLevels = 12;
#ifndef VFS_BOTTOM_THREADS
#define VFS_BOTTOM_THREADS 512
#endif
constexpr int kBottomThreads = VFS_BOTTOM_THREADS;
#ifndef VFS_BOTTOM_CELLS
#define VFS_BOTTOM_CELLS 512
#endif
constexpr long long kBottomCells = VFS_BOTTOM_CELLS;

template <typename T>
struct BLevel {
  ZL z;
  const uint8_t *act;
  const Q4<T> *cpl, *tri;
  T *x, *b, *xo;
  Q2<T> *ds;
  int zebra;
};
template <typename T>
struct Bottom {
  int nl;
  int pre, post, coarse;
  T omega;
  BLevel<T> lv[kBottomMaxLevels];
};

template <typename T>
__device__ void blk_smooth(const BLevel<T> &L, int sweeps, bool x_zero, T omega) {
  const long long half = (long long)L.z.nz * L.z.hx;
  for (int s = 0; s < sweeps; s++) {
    const bool z = x_zero && s == 0;
    if (L.zebra) {
      for (int col = 0; col < 2; col++) {
        for (long long t = threadIdx.x; t < half; t += blockDim.x)
          zline_column<T, 2>(L.z, L.cpl, L.tri, L.b, L.x, L.ds, L.x, col, T(1), (z && col == 0) ? 1 : 0, t);
        __syncthreads();
      }
    } else {
      if (!z) {
        for (long long t = threadIdx.x; t < L.z.n; t += blockDim.x) L.xo[t] = L.x[t];
        __syncthreads();
      }
      for (long long t = threadIdx.x; t < 2 * half; t += blockDim.x)
        zline_column<T, 2>(L.z, L.cpl, L.tri, L.b, L.xo, L.ds, L.x, -1, omega, z ? 1 : 0, t);
      __syncthreads();
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kBottomThreads) k_mg_bottom(Bottom<T> B) {
  pdl_prologue();
  for (int l = 0; l < B.nl - 1; l++) {
    const BLevel<T> &F = B.lv[l], &C = B.lv[l + 1];
    blk_smooth<T>(F, B.pre, true, B.omega);
    const long long nc = (long long)C.z.nx * C.z.ny * C.z.nz;
    for (long long t = threadIdx.x; t < nc; t += blockDim.x)
      zrestrict_cell<T>(F.z, C.z, F.cpl, F.tri, F.x, F.b, C.b, t);
    __syncthreads();
  }
  blk_smooth<T>(B.lv[B.nl - 1], B.coarse, true, B.omega);
  for (int l = B.nl - 2; l >= 0; l--) {
    const BLevel<T> &F = B.lv[l], &C = B.lv[l + 1];
    const long long nf = (long long)F.z.nx * F.z.ny * F.z.nz;
    for (long long t = threadIdx.x; t < nf; t += blockDim.x) zprolong_cell<T>(F.z, C.z, F.act, C.act, F.x, C.x, t);
    __syncthreads();
    blk_smooth<T>(F, B.post, false, B.omega);
  }
}

// DA-layout vector (FP64, or FP32 in the FP32 inner Krylov) -> finest-level right-hand side.
template <typename T, typename VT>
__global__ void k_to_zebra(Grid g, ZL L, const VT *__restrict__ v, const int *__restrict__ jslot, long long ldv,
                           T *__restrict__ b) {
  pdl_prologue();
  if (jslot) v += (long long)(*jslot) * ldv;  // the j-th basis vector of a device-driven solve
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)L.nx * L.ny * L.nz;
  if (t >= ncell) return;
  int i, j, k;
  zcell(L, t, i, j, k);
  b[zidx(L, i, j, k)] = (T)v[lidx(g, i + 1, j + 1, k + 1)];
}

// Finest-level solution -> DA-layout vector (zero off the unknowns).
template <typename T, typename VT>
__global__ void k_from_zebra(Grid g, ZL L, const uint8_t *__restrict__ fluid, const T *__restrict__ x,
                             const int *__restrict__ jslot, long long ldv, VT *__restrict__ z) {
  pdl_prologue();
  if (jslot) z += (long long)(*jslot) * ldv;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const unsigned up = (unsigned)p, umx = (unsigned)g.mx, umy = (unsigned)g.my;
  const unsigned r = up / umx, kk = r / umy;
  const int i = (int)(up - r * umx), j = (int)(r - kk * umy), k = (int)kk;
  double v = 0;
  if (fluid[p] && i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2)
    v = (double)x[zidx(L, i - 1, j - 1, k - 1)];
  z[p] = (VT)v;
}

// ------------------------------------------------------------------ host side
static ZL make_zl(int nx, int ny, int nz, const Grid &g) {
  ZL L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.hx = (nx + 1) / 2;
  L.ip = g.iper; L.jp = g.jper; L.kp = g.kper;
  L.n = (long long)nz * ny * 2 * L.hx;
  return L;
}

void mg_free(Poisson &P) {
  for (MGLevel &L : P.lv) {
    cudaFree(L.op64); cudaFree(L.pk64); cudaFree(L.pk32); cudaFree(L.v64); cudaFree(L.v32); cudaFree(L.act);
  }
  P.lv.clear();
}

// Per level: raw FP64 couplings and Thomas factors (op64, used to build the next level),
// the packed FP64 and FP32 operators, and the work vectors x | b | xo | ds (2n).  A rebuild
// on the same grid (every first time step runs PoissonLHSNew) keeps the levels' buffers.
int mg_setup(Ctx *c) {
  Poisson &P = c->ps;
  const Grid &g = c->g;
  int rc;
  std::vector<MGLevel> old;
  old.swap(P.lv);
  int nx = g.mx - 2, ny = g.my - 2, nz = g.mz - 2;
  const int maxlev = 12;
  auto fail = [&](int code, const char *msg) {
    for (size_t l = P.lv.size(); l < old.size(); l++) P.lv.push_back(old[l]);  // freed by mg_free
    return set_err(c, code, msg);
  };
  while ((int)P.lv.size() < maxlev) {
    MGLevel L;
    L.z = make_zl(nx, ny, nz, g);
    L.zebra = !((L.z.ip && (nx & 1)) || (L.z.kp && (nz & 1)));
    const long long n = L.z.n;
    if (n >= (1LL << 31)) return fail(VFS_ERR_INVALID, "poisson_lhs: grid too large for the multigrid indexing");
    const size_t l = P.lv.size();
    if (l < old.size() && old[l].z.n == n && old[l].op64) {
      L.op64 = old[l].op64; L.pk64 = old[l].pk64; L.pk32 = old[l].pk32;
      L.v64 = old[l].v64; L.v32 = old[l].v32; L.act = old[l].act;
      old[l].op64 = nullptr;  // taken
    } else {
      if (l < old.size()) {
        MGLevel &O = old[l];
        cudaFree(O.op64); cudaFree(O.pk64); cudaFree(O.pk32); cudaFree(O.v64); cudaFree(O.v32); cudaFree(O.act);
        O.op64 = nullptr;
      }
      bool ok = cudaMalloc(&L.op64, sizeof(double) * NOP * n) == cudaSuccess;
      ok &= cudaMalloc(&L.pk64, sizeof(double) * 8 * n) == cudaSuccess;
      ok &= cudaMalloc(&L.pk32, sizeof(float) * 8 * n) == cudaSuccess;
      ok &= cudaMalloc(&L.v64, sizeof(double) * 5 * n) == cudaSuccess;
      ok &= cudaMalloc(&L.v32, sizeof(float) * 5 * n) == cudaSuccess;
      ok &= cudaMalloc(&L.act, n) == cudaSuccess;
      if (!ok) {
        P.lv.push_back(L);
        return fail(VFS_ERR_CUDA, "poisson_lhs: multigrid allocation failed");
      }
    }
    cudaMemsetAsync(L.op64, 0, sizeof(double) * NOP * n, c->stream);
    cudaMemsetAsync(L.pk64, 0, sizeof(double) * 8 * n, c->stream);
    cudaMemsetAsync(L.pk32, 0, sizeof(float) * 8 * n, c->stream);
    cudaMemsetAsync(L.v64, 0, sizeof(double) * 5 * n, c->stream);
    cudaMemsetAsync(L.v32, 0, sizeof(float) * 5 * n, c->stream);
    const long long ncell = (long long)nx * ny * nz;
    if (P.lv.empty()) {
      c->launches++, k_mg_fine_couplings<<<nblocks(ncell, 128), 128, 0, c->stream>>>(g, L.z, P.coef, P.fluid, L.op64);
    } else {
      const MGLevel &F = P.lv.back();
      c->launches++, k_mg_coarse_couplings<<<nblocks(ncell, 128), 128, 0, c->stream>>>(F.z, L.z, F.op64, L.op64);
    }
    if ((rc = check_launch(c, "k_mg_couplings"))) { P.lv.push_back(L); return fail(rc, "poisson_lhs: multigrid set-up failed"); }
    c->launches++, k_mg_diag<<<nblocks(ncell, 128), 128, 0, c->stream>>>(L.z, L.op64);
    c->launches++, k_mg_thomas<<<nblocks((long long)nx * nz, 64), 64, 0, c->stream>>>(L.z, L.op64);
    c->launches++, k_mg_active<<<nblocks(n, 256), 256, 0, c->stream>>>(n, L.op64, L.act);
    c->launches++, k_mg_pack<double><<<nblocks(ncell, 128), 128, 0, c->stream>>>(L.z, L.op64, (Q4<double> *)L.pk64,
                                                                 (Q4<double> *)L.pk64 + n);
    c->launches++, k_mg_pack<float><<<nblocks(ncell, 128), 128, 0, c->stream>>>(L.z, L.op64, (Q4<float> *)L.pk32,
                                                                (Q4<float> *)L.pk32 + n);
    P.lv.push_back(L);
    if ((rc = check_launch(c, "k_mg_setup"))) return fail(rc, "poisson_lhs: multigrid set-up failed");
    if ((nx & 1) || (ny & 1) || (nz & 1) || nx < 4 || ny < 4 || nz < 4) break;
    nx /= 2; ny /= 2; nz /= 2;
  }
  for (size_t l = P.lv.size(); l < old.size(); l++) {  // levels the new hierarchy does not reach
    MGLevel &O = old[l];
    cudaFree(O.op64); cudaFree(O.pk64); cudaFree(O.pk32); cudaFree(O.v64); cudaFree(O.v32); cudaFree(O.act);
  }
  return VFS_OK;
}

// Typed views of a level's packed operator and work vectors.
template <typename T>
struct LvT {
  const Q4<T> *cpl, *tri;
  T *x, *b, *xo;
  Q2<T> *ds;
};
template <typename T>
static LvT<T> lvt(const MGLevel &L);
template <>
LvT<float> lvt<float>(const MGLevel &L) {
  const long long n = L.z.n;
  LvT<float> r;
  r.cpl = (const Q4<float> *)L.pk32; r.tri = (const Q4<float> *)L.pk32 + n;
  r.x = L.v32; r.b = L.v32 + n; r.xo = L.v32 + 2 * n; r.ds = (Q2<float> *)(L.v32 + 3 * n);
  return r;
}
template <>
LvT<double> lvt<double>(const MGLevel &L) {
  const long long n = L.z.n;
  LvT<double> r;
  r.cpl = (const Q4<double> *)L.pk64; r.tri = (const Q4<double> *)L.pk64 + n;
  r.x = L.v64; r.b = L.v64 + n; r.xo = L.v64 + 2 * n; r.ds = (Q2<double> *)(L.v64 + 3 * n);
  return r;
}

static const double kJacobiOmega = 0.8;

// Launches one tiled colour pass; false when the level's columns do not fit the tile.
// rc receives the launch status.
template <typename T, int W>
static bool launch_tile_w(Ctx *c, const MGLevel &L, const LvT<T> &v, int colour, int x_zero, int &rc) {
  if (!tile_fits<T, W>(L.z.ny)) return false;
  const size_t smem = tile_smem<T, W>(L.z.ny);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_zline_tile<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const int tiles = (L.z.hx + W - 1) / W;
  rc = launch_chain(c, "k_zline_tile", k_zline_tile<T, W>, dim3(tiles * L.z.nz), dim3(kTileThreads), smem, L.z,
                    v.cpl, v.tri, v.b, v.x, v.x, colour, x_zero);
  return true;
}
template <typename T>
static bool launch_zline_tile(Ctx *c, const MGLevel &L, const LvT<T> &v, int colour, int x_zero, int &rc) {
  if (sizeof(T) == 4)
    return launch_tile_w<T, VFS_ZTILE_W32>(c, L, v, colour, x_zero, rc) ||
           launch_tile_w<T, 8>(c, L, v, colour, x_zero, rc);
  return launch_tile_w<T, VFS_ZTILE_W64>(c, L, v, colour, x_zero, rc) ||
         launch_tile_w<T, 8>(c, L, v, colour, x_zero, rc);
}

// `sweeps` smoothing sweeps on level l; x_zero: x is taken as zero on entry.
template <typename T>
static int mg_smooth(Ctx *c, int l, int sweeps, bool x_zero) {
  const MGLevel &L = c->ps.lv[l];
  const LvT<T> v = lvt<T>(L);
  const long long half = (long long)L.z.nz * L.z.hx;
  int rc = VFS_OK;
  for (int s = 0; s < sweeps; s++) {
    const bool z = x_zero && s == 0;
    if (L.zebra) {
      for (int col = 0; col < 2; col++) {
        const int xz = (z && col == 0) ? 1 : 0;
        if (!launch_zline_tile<T>(c, L, v, col, xz, rc)) {
          c->launches++, k_zline<T><<<nblocks(half, 64), 64, 0, c->stream>>>(L.z, v.cpl, v.tri, v.b, v.x, v.ds, v.x, col, T(1), xz);
          rc = check_launch(c, "k_zline");
        }
        if (rc) return rc;
      }
    } else {
      if (!z) cudaMemcpyAsync(v.xo, v.x, sizeof(T) * L.z.n, cudaMemcpyDeviceToDevice, c->stream);
      c->launches++, k_zline<T><<<nblocks(2 * half, 64), 64, 0, c->stream>>>(L.z, v.cpl, v.tri, v.b, v.xo, v.ds, v.x, -1,
                                                               T(kJacobiOmega), z ? 1 : 0);
      if ((rc = check_launch(c, "k_zline"))) return rc;
    }
  }
  return rc;
}

template <typename T>
static int mg_bottom(Ctx *c, int l, int nl, const vfs_solve_opts &o) {
  Bottom<T> B;
  B.nl = nl - l;
  if (B.nl > kBottomMaxLevels) return set_err(c, VFS_ERR_INVALID, "multigrid: too many levels");
  B.pre = o.pre_smooth; B.post = o.post_smooth; B.coarse = o.coarse_iters;
  B.omega = T(kJacobiOmega);
  for (int q = 0; q < B.nl; q++) {
    const MGLevel &L = c->ps.lv[l + q];
    const LvT<T> v = lvt<T>(L);
    BLevel<T> &d = B.lv[q];
    d.z = L.z;
    d.act = L.act;
    d.cpl = v.cpl; d.tri = v.tri;
    d.x = v.x; d.b = v.b; d.xo = v.xo; d.ds = v.ds;
    d.zebra = L.zebra ? 1 : 0;
  }
  return launch_chain(c, "k_mg_bottom", k_mg_bottom<T>, dim3(1), dim3(kBottomThreads), 0, B);
}

// V-cycle from level l (its right-hand side already in place); levels at or below
// kBottomCells run inside one thread block.
#ifndef VFS_PROLONG8
#define VFS_PROLONG8 1
#endif
template <typename T>
static int mg_vcycle(Ctx *c, int l, int nl, const vfs_solve_opts &o) {
  int rc;
  const MGLevel &Lv = c->ps.lv[l];
  if ((long long)Lv.z.nx * Lv.z.ny * Lv.z.nz <= kBottomCells) return mg_bottom<T>(c, l, nl, o);
  if (l == nl - 1) return mg_smooth<T>(c, l, o.coarse_iters, true);
  if ((rc = mg_smooth<T>(c, l, o.pre_smooth, true))) return rc;
  const MGLevel &F = c->ps.lv[l], &C = c->ps.lv[l + 1];
  const long long nc = (long long)C.z.nx * C.z.ny * C.z.nz, nf = (long long)F.z.nx * F.z.ny * F.z.nz;
  const LvT<T> f = lvt<T>(F), cc = lvt<T>(C);
  // the pre-smoothing ends with a colour-1 pass: on a zebra level without periodic j only
  // the colour-0 residuals are left
  if (F.zebra && !F.z.jp)
    rc = launch_chain(c, "k_zrestrict", k_zrestrict<T, true>, dim3(nblocks(nc, 128)), dim3(128), 0, F.z, C.z, f.cpl,
                      f.tri, f.x, f.b, cc.b);
  else
    rc = launch_chain(c, "k_zrestrict", k_zrestrict<T, false>, dim3(nblocks(nc, 128)), dim3(128), 0, F.z, C.z, f.cpl,
                      f.tri, f.x, f.b, cc.b);
  if (rc) return rc;
  if ((rc = mg_vcycle<T>(c, l + 1, nl, o))) return rc;
  if (VFS_PROLONG8 && F.z.nx == 2 * C.z.nx && F.z.ny == 2 * C.z.ny && F.z.nz == 2 * C.z.nz)
    rc = launch_chain(c, "k_zprolong8", k_zprolong8<T>, dim3(nblocks(nc, 128)), dim3(128), 0, F.z, C.z, F.act,
                      C.act, f.x, cc.x);
  else
    rc = launch_chain(c, "k_zprolong", k_zprolong<T>, dim3(nblocks(nf, 256)), dim3(256), 0, F.z, C.z, F.act,
                      C.act, f.x, cc.x);
  if (rc) return rc;
  return mg_smooth<T>(c, l, o.post_smooth, false);
}

template <typename T, typename VT = double>
static int mg_apply(Ctx *c, const VT *v, VT *z, const vfs_solve_opts &o, const int *jslot = nullptr,
                    long long ldv = 0) {
  Poisson &P = c->ps;
  const MGLevel &L0 = P.lv[0];
  const long long ncell = (long long)L0.z.nx * L0.z.ny * L0.z.nz;
  const LvT<T> l0 = lvt<T>(L0);
  int rc;
  if ((rc = launch_chain(c, "k_to_zebra", k_to_zebra<T, VT>, dim3(nblocks(ncell, 256)), dim3(256), 0, c->g, L0.z, v,
                         jslot, ldv, l0.b)))
    return rc;
  const int nl = o.levels > 0 ? std::min((int)P.lv.size(), o.levels) : (int)P.lv.size();
  if ((rc = mg_vcycle<T>(c, 0, nl, o))) return rc;
  return launch_chain(c, "k_from_zebra", k_from_zebra<T, VT>, dim3(nblocks(c->g.N, 256)), dim3(256), 0, c->g, L0.z,
                      P.fluid, l0.x, jslot, ldv, z);
}

// z = M^-1 v: one V-cycle in FP32 (precision 0) or FP64.
int mg_precondition(Ctx *c, const double *v, double *z, const vfs_solve_opts &o) {
  return o.precision != 1 ? mg_apply<float>(c, v, z, o) : mg_apply<double>(c, v, z, o);
}

// z_j = M^-1 v_j with v_j = V + j ldv, z_j = Z + j ldv and j read on the device (*jslot).
int mg_precondition_dyn(Ctx *c, const double *V, double *Z, long long ldv, const int *jslot, const vfs_solve_opts &o) {
  return o.precision != 1 ? mg_apply<float>(c, V, Z, o, jslot, ldv) : mg_apply<double>(c, V, Z, o, jslot, ldv);
}

// The same with FP32 vectors (the FP32 inner Krylov of precision 2): an FP32 V-cycle.
int mg_precondition_dyn32(Ctx *c, const float *V, float *Z, long long ldv, const int *jslot, const vfs_solve_opts &o) {
  return mg_apply<float, float>(c, V, Z, o, jslot, ldv);
}

// One smoothing sweep of the finest level (both colours), for timing.
int mg_sweep_fine(Ctx *c, int precision) {
  return precision == 0 ? mg_smooth<float>(c, 0, 1, false) : mg_smooth<double>(c, 0, 1, false);
}

}  // namespace vfs
