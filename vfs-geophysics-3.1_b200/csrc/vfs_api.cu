// C-ABI layer: context life cycle, host<->device field transfer in the reference's
// AoS DA layout, scalars, errors and the operator entry points declared in
// include/vfs_b200.h.
#include <cstdio>
#include <cstring>
#include <cmath>

#include "vfs_internal.cuh"

using namespace vfs;

static std::string g_last_err;

namespace vfs {

int set_err(Ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  g_last_err = msg;
  return code;
}

int check_launch(Ctx *c, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return VFS_OK;
}

V3 field3(Ctx *c, int f) { return V3{c->f[f][0], c->f[f][1], c->f[f][2]}; }

Metrics metrics(Ctx *c) {
  Metrics m;
  m.csi = cv(field3(c, VFS_CSI)); m.eta = cv(field3(c, VFS_ETA)); m.zet = cv(field3(c, VFS_ZET));
  m.aj = c->f[VFS_AJ][0];
  m.icsi = cv(field3(c, VFS_ICSI)); m.ieta = cv(field3(c, VFS_IETA)); m.izet = cv(field3(c, VFS_IZET));
  m.iaj = c->f[VFS_IAJ][0];
  m.jcsi = cv(field3(c, VFS_JCSI)); m.jeta = cv(field3(c, VFS_JETA)); m.jzet = cv(field3(c, VFS_JZET));
  m.jaj = c->f[VFS_JAJ][0];
  m.kcsi = cv(field3(c, VFS_KCSI)); m.keta = cv(field3(c, VFS_KETA)); m.kzet = cv(field3(c, VFS_KZET));
  m.kaj = c->f[VFS_KAJ][0];
  return m;
}

int ensure_red(Ctx *c, int n) {
  if (n <= c->red_cap) return VFS_OK;
  c->setup_epoch++;  // a captured step holds the old buffer
  if (c->red) cudaFree(c->red);
  if (c->red_host) cudaFreeHost(c->red_host);
  c->red = nullptr; c->red_host = nullptr;
  if (cudaMalloc(&c->red, sizeof(double) * n) != cudaSuccess ||
      cudaMallocHost(&c->red_host, sizeof(double) * n) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "reduction buffer allocation failed");
  c->red_cap = n;
  return VFS_OK;
}

// Sum of nparts partial sums in a fixed order (single block, deterministic).
// One block of kSumThreads threads; eight independent partial sums per thread keep eight
// loads in flight (the block partials of a one-point-per-thread pass number N/256, about
// 50,000 at 12.6 M points), combined in a fixed order: the result depends only on n.
// parts may overlap out (reduce_sum writes at red + 63): every load precedes the barrier.
constexpr int kSumThreads = 1024;
__global__ void __launch_bounds__(kSumThreads) k_sum_parts(const double *parts, int n, double *out) {
  __shared__ double sh[kSumThreads / 32];
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int q = threadIdx.x;
  for (; q + 7 * kSumThreads < n; q += 8 * kSumThreads) {
#pragma unroll
    for (int u = 0; u < 8; u++) s[u] += parts[q + u * kSumThreads];
  }
  for (; q < n; q += kSumThreads) s[0] += parts[q];
  double t = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x < 32) {
    t = sh[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) out[0] = t;
  }
}

// Staging buffer for vfs_set_field / vfs_get_field: allocated on first use, kept for
// the life of the context so that repeated transfers allocate nothing.
static int ensure_stage(Ctx *c, size_t bytes) {
  if (bytes <= c->stage_bytes) return VFS_OK;
  if (c->stage) cudaFree(c->stage);
  c->stage = nullptr;
  c->stage_bytes = 0;
  if (cudaMalloc(&c->stage, bytes) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "staging buffer allocation failed");
  c->stage_bytes = bytes;
  return VFS_OK;
}

// Sum of nparts partials into device memory dst (a device scalar), no host wait.
int reduce_to(Ctx *c, const double *parts, int nparts, double *dst) {
  c->launches++, k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(parts, nparts, dst);
  return check_launch(c, "k_sum_parts");
}

// Reads the device scalars into ds_out and refreshes the host mirror of the scalars a
// step computes.  No-op while a step is being captured (the captured step reads them back
// with its last node).
int ds_fetch(Ctx *c) {
  if (c->capturing) return VFS_OK;
  cudaMemcpyAsync(c->ds_out, c->ds, sizeof(double) * DS_COUNT, cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "device scalar read failed");
  c->scal[VFS_S_MEAN_K_FLUX] = c->ds_out[DS_MEAN_K_FLUX];
  c->scal[VFS_S_FLUX_IN] = c->ds_out[DS_FLUX_IN];
  c->scal[VFS_S_FLUX_OUT] = c->ds_out[DS_FLUX_OUT];
  return VFS_OK;
}

// Host scalars with a device copy in ds (the step's kernels read ds).
static const int kMirror[][2] = {{VFS_S_INLET_FLUX, DS_INLET_FLUX}, {VFS_S_INLET_AREA, DS_INLET_AREA},
                                 {VFS_S_MEAN_K_AREA, DS_MEAN_K_AREA}, {VFS_S_MEAN_K_FLUX, DS_MEAN_K_FLUX},
                                 {VFS_S_FLUX_IN, DS_FLUX_IN}, {VFS_S_FLUX_OUT, DS_FLUX_OUT}};

// Writes the host scalars that have a device copy into ds (outside a step: vfs_create,
// vfs_set_scalar, the set-up that computes them on the host), so that host and device
// agree between steps.
int ds_upload(Ctx *c) {
  for (const auto &m : kMirror) {
    c->ds_in[m[1]] = c->scal[m[0]];
    cudaMemcpyAsync(c->ds + m[1], c->ds_in + m[1], sizeof(double), cudaMemcpyHostToDevice, c->stream);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "device scalar upload failed");
  return VFS_OK;
}

int reduce_sum(Ctx *c, const double *parts, int nparts, double *out) {
  int rc = ensure_red(c, 64);
  if (rc) return rc;
  c->launches++, k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(parts, nparts, c->red + 63);
  if ((rc = check_launch(c, "k_sum_parts"))) return rc;
  cudaMemcpyAsync(c->red_host + 63, c->red + 63, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "reduce_sum: stream sync failed");
  *out = c->red_host[63];
  return VFS_OK;
}

}  // namespace vfs

// ---------------------------------------------------------------- pack kernels
// AoS (reference Cmpnts layout) <-> SoA component arrays.
__global__ void k_unpack(const double *__restrict__ aos, int dof, long long n, double *c0,
                         double *c1, double *c2) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (dof == 1) { c0[p] = aos[p]; return; }
  c0[p] = aos[3 * p]; c1[p] = aos[3 * p + 1]; c2[p] = aos[3 * p + 2];
}
__global__ void k_pack(double *__restrict__ aos, int dof, long long n, const double *c0,
                       const double *c1, const double *c2) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (dof == 1) { aos[p] = c0[p]; return; }
  aos[3 * p] = c0[p]; aos[3 * p + 1] = c1[p]; aos[3 * p + 2] = c2[p];
}
// nvert (double 0/1/3) -> uint8, flagging non-integral or out-of-range values.
__global__ void k_nvert_to_u8(const double *__restrict__ nvd, long long n, uint8_t *nv, int *bad) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  double v = nvd[p];
  double r = rint(v);
  if (!(v >= 0.0 && v <= 255.0) || r != v) { atomicExch(bad, 1); nv[p] = 0; return; }
  nv[p] = (uint8_t)r;
}

static const int kDof[VFS_NFIELDS] = {
    3, 3, 1, 1, 1, 1, 3, 3, 3, 3, 1, 3,  // UCONT..CENT
    3, 3, 3, 1,                            // CSI ETA ZET AJ
    3, 3, 3, 1, 3, 3, 3, 1, 3, 3, 3, 1,    // I J K face metrics
    1, 1,                                   // CS USTAR
    3};                                     // RHS_O

extern "C" {

const char *vfs_last_error(const vfs_ctx *ctx) {
  const Ctx *c = (const Ctx *)ctx;
  return c ? c->err.c_str() : g_last_err.c_str();
}

int vfs_create(const vfs_config *cfg, int device, vfs_ctx **out) {
  if (!cfg || !out) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, VFS_ERR_NO_DEVICE, "vfs_create: no CUDA device");
  if (device < 0 || device >= ndev) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: bad device");
  if (cfg->IM < 4 || cfg->JM < 4 || cfg->KM < 4)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: grid needs at least 4 nodes per direction");
  if ((long long)(cfg->IM + 1) * (cfg->JM + 1) * (cfg->KM + 1) >= (1LL << 31))
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: grids of 2^31 DA points or more are not supported");
  // Boundary codes handled on this path: 0 (unset), 1 no-slip wall, 2 moving lid (j+),
  // 4 outlet (k+ or j+), 5 inlet (k-), 7 periodic face, 10 free-slip, 12 moving wall,
  // 13/14 slip lid.
  for (int q = 0; q < 6; q++) {
    int b = cfg->bctype[q];
    bool ok = (b == 0 || b == 1 || b == 2 || b == 4 || b == 5 || b == 7 || b == 10 || b == 12 ||
               b == 13 || b == 14 || b == -10);
    if (!ok) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: unsupported bctype " + std::to_string(b));
    if (b == 5 && q != 4) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: an inlet (5) is supported on the k = 0 face only");
    if (b == 4 && q != 5 && q != 3) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: an outlet (4) is supported on the k+ and j+ faces only");
  }
  if (cfg->bctype[4] == 5) {
    const int ip = cfg->inletprofile;
    if (!(ip == 1 || ip == 2 || ip == 21 || ip == 100))
      return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: inlet profiles 1, 2, 21 and 100 are supported");
    if (cfg->k_periodic) return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: an inlet face cannot be k-periodic");
  }
  if (cfg->immersed < 0 || cfg->immersed > 1)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: immersed must be 0 or 1");
  if (cfg->les != 0 && cfg->les != 1 && cfg->les != 2)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: les must be 0, 1 or 2");
  if (cfg->implicit != 0 && cfg->implicit != 4)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_create: implicit must be 0 (Runge-Kutta) or 4 (matrix-free)");
  if (cudaSetDevice(device) != cudaSuccess) return set_err(nullptr, VFS_ERR_CUDA, "cudaSetDevice failed");
  // The kernels are built for sm_100a only; refuse other GPUs up front.
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major != 10)
    return set_err(nullptr, VFS_ERR_NO_DEVICE, "vfs_create: this library is built for sm_100a (B200)");

  Ctx *c = new Ctx();
  c->cfg = *cfg;
  c->device = device;
  Grid &g = c->g;
  g.mx = cfg->IM + 1; g.my = cfg->JM + 1; g.mz = cfg->KM + 1;
  g.N = (long long)g.mx * g.my * g.mz;
  g.iper = cfg->i_periodic; g.jper = cfg->j_periodic; g.kper = cfg->k_periodic;
  for (int q = 0; q < 6; q++) g.bc[q] = cfg->bctype[q];
  g.immersed = cfg->immersed; g.les = cfg->les;
  g.wallfunction = cfg->wallfunction; g.moving = cfg->moving;
  g.roughness = cfg->roughness > 0 ? cfg->roughness : 0.0;
  g.ren = cfg->ren; g.dt = cfg->dt; g.st = cfg->st;
  c->scal[VFS_S_DT] = cfg->dt; c->scal[VFS_S_REN] = cfg->ren; c->scal[VFS_S_ST] = cfg->st;
  c->scal[VFS_S_INLET_FLUX] = cfg->inlet_flux;
  c->scal[VFS_S_NBODIES] = 1;
  c->tistart = cfg->tistart;
  c->ti = cfg->tistart;
  c->rstart = cfg->rstart;
  c->dynamic_freq = cfg->dynamic_freq < 1 ? 1 : cfg->dynamic_freq;
  c->max_cs = cfg->max_cs > 0 ? cfg->max_cs : 0.5;
  c->scal[VFS_S_TI] = c->ti;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return set_err(nullptr, VFS_ERR_CUDA, "stream creation failed");
  }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  const size_t bytes = sizeof(double) * (size_t)g.N;
  bool okm = true;
  for (int f = 0; f < VFS_NFIELDS; f++) {
    c->dof[f] = kDof[f];
    for (int q = 0; q < kDof[f]; q++) {
      okm &= cudaMalloc(&c->f[f][q], bytes) == cudaSuccess;
      if (okm) cudaMemsetAsync(c->f[f][q], 0, bytes, c->stream);
    }
  }
  okm &= cudaMalloc(&c->nv, (size_t)g.N) == cudaSuccess;
  if (okm) cudaMemsetAsync(c->nv, 0, (size_t)g.N, c->stream);
  for (int d = 0; d < 3; d++)
    for (int q = 0; q < 3; q++) {
      okm &= cudaMalloc(&c->div[d][q], bytes) == cudaSuccess;
      okm &= cudaMalloc(&c->visc[d][q], bytes) == cudaSuccess;
      if (okm) { cudaMemsetAsync(c->div[d][q], 0, bytes, c->stream); cudaMemsetAsync(c->visc[d][q], 0, bytes, c->stream); }
    }
  for (int q = 0; q < 3; q++) {
    okm &= cudaMalloc(&c->fp[q], bytes) == cudaSuccess;
    okm &= cudaMalloc(&c->pucont[q], bytes) == cudaSuccess;
    okm &= cudaMalloc(&c->bcbuf[q], bytes) == cudaSuccess;
    if (okm) {
      cudaMemsetAsync(c->fp[q], 0, bytes, c->stream);
      cudaMemsetAsync(c->pucont[q], 0, bytes, c->stream);
      cudaMemsetAsync(c->bcbuf[q], 0, bytes, c->stream);
    }
  }
  okm &= cudaMalloc(&c->bcflag, (size_t)g.N) == cudaSuccess;
  if (okm) cudaMemsetAsync(c->bcflag, 0, (size_t)g.N, c->stream);
  okm &= ensure_red(c, 16384) == VFS_OK;
  okm &= cudaMalloc(&c->ds, sizeof(double) * DS_COUNT) == cudaSuccess;
  okm &= cudaMallocHost(&c->ds_in, sizeof(double) * DS_COUNT) == cudaSuccess;
  okm &= cudaMallocHost(&c->ds_out, sizeof(double) * DS_COUNT) == cudaSuccess;
  okm &= cudaMalloc(&c->kd, sizeof(KryDev)) == cudaSuccess;
  okm &= cudaMallocHost(&c->kd_host, sizeof(KryDev)) == cudaSuccess;
  if (okm) {
    cudaMemsetAsync(c->ds, 0, sizeof(double) * DS_COUNT, c->stream);
    cudaMemsetAsync(c->kd, 0, sizeof(KryDev), c->stream);
    memset(c->ds_in, 0, sizeof(double) * DS_COUNT);
    memset(c->ds_out, 0, sizeof(double) * DS_COUNT);
  }
  if (!okm) {
    vfs_destroy((vfs_ctx *)c);
    return set_err(nullptr, VFS_ERR_CUDA, "vfs_create: device allocation failed");
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess || ds_upload(c) != VFS_OK) {
    vfs_destroy((vfs_ctx *)c);
    return set_err(nullptr, VFS_ERR_CUDA, "vfs_create: initialisation failed");
  }
  *out = (vfs_ctx *)c;
  return VFS_OK;
}

int vfs_destroy(vfs_ctx *ctx) {
  Ctx *c = (Ctx *)ctx;
  if (!c) return VFS_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int f = 0; f < VFS_NFIELDS; f++)
    for (int q = 0; q < 3; q++) if (c->f[f][q]) cudaFree(c->f[f][q]);
  if (c->nv) cudaFree(c->nv);
  if (c->nvo) cudaFree(c->nvo);
  if (c->gab) cudaFree(c->gab);
  if (c->imp) cudaFree(c->imp);
  if (c->ibv) cudaFree(c->ibv);
  if (c->bcflag) cudaFree(c->bcflag);
  if (c->solid) cudaFree(c->solid);
  for (int d = 0; d < 3; d++)
    for (int q = 0; q < 3; q++) { cudaFree(c->div[d][q]); cudaFree(c->visc[d][q]); }
  for (int q = 0; q < 3; q++) { cudaFree(c->fp[q]); cudaFree(c->pucont[q]); cudaFree(c->bcbuf[q]); }
  if (c->red) cudaFree(c->red);
  if (c->red_host) cudaFreeHost(c->red_host);
  if (c->stage) cudaFree(c->stage);
  if (c->inflow_plane) cudaFree(c->inflow_plane);
  if (c->inlet_nodes) cudaFree(c->inlet_nodes);
  if (c->ibn) cudaFree(c->ibn);
  if (c->ibbuf) cudaFree(c->ibbuf);
  step_graph_free(c);
  if (c->ds) cudaFree(c->ds);
  if (c->ds_in) cudaFreeHost(c->ds_in);
  if (c->ds_out) cudaFreeHost(c->ds_out);
  if (c->kd) cudaFree(c->kd);
  if (c->kd_host) cudaFreeHost(c->kd_host);
  for (int q = 0; q < 2; q++)
    if (c->cap_streams[q]) cudaStreamDestroy(c->cap_streams[q]);
  adjoint_free(c);
  Poisson &P = c->ps;
  cudaFree(P.coef); cudaFree(P.fluid);
  cudaFree(P.V); cudaFree(P.Z); cudaFree(P.w); cudaFree(P.r); cudaFree(P.t); cudaFree(P.hdev);
  cudaFree(P.V32); cudaFree(P.Z32); cudaFree(P.w32);
  mg_free(P);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return VFS_OK;
}

int vfs_dims(const vfs_ctx *ctx, int *mx, int *my, int *mz) {
  const Ctx *c = (const Ctx *)ctx;
  if (!c) return VFS_ERR_INVALID;
  if (mx) *mx = c->g.mx;
  if (my) *my = c->g.my;
  if (mz) *mz = c->g.mz;
  return VFS_OK;
}

long long vfs_launch_count(const vfs_ctx *ctx) { return ctx ? ((const Ctx *)ctx)->launches : 0; }

int vfs_synchronize(vfs_ctx *ctx) {
  Ctx *c = (Ctx *)ctx;
  if (!c) return VFS_ERR_INVALID;
  cudaSetDevice(c->device);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, std::string("synchronize: ") + cudaGetErrorString(cudaGetLastError()));
  return VFS_OK;
}

int vfs_set_field(vfs_ctx *ctx, int field, const double *host) {
  Ctx *c = (Ctx *)ctx;
  if (!c || !host || field < 0 || field >= VFS_NFIELDS) return set_err(c, VFS_ERR_INVALID, "vfs_set_field: bad argument");
  cudaSetDevice(c->device);
  if (field == VFS_NVERT || (field >= VFS_CSI && field <= VFS_KAJ)) c->setup_epoch++;
  const int dof = c->dof[field];
  const size_t bytes = sizeof(double) * (size_t)c->g.N * dof;
  int rc = ensure_stage(c, sizeof(double) * (size_t)c->g.N * 3);
  if (rc) return rc;
  double *stage = c->stage;
  cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, c->stream);
  if (field == VFS_NVERT) {
    int *bad = (int *)c->red;  // first word of the reduction buffer as a flag
    cudaMemsetAsync(bad, 0, sizeof(int), c->stream);
    c->launches++, k_nvert_to_u8<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(stage, c->g.N, c->nv, bad);
    rc = check_launch(c, "k_nvert_to_u8");
    int hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(c->f[field][0], stage, bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    if (!rc && hbad) rc = set_err(c, VFS_ERR_INVALID, "vfs_set_field: nvert must hold integers 0..255");
    c->nvert_set = true;
    c->nsolid = -1;
    c->ps.built = false;
    return rc;
  }
  c->launches++, k_unpack<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(stage, dof, c->g.N, c->f[field][0],
                                                       c->f[field][1], c->f[field][2]);
  rc = check_launch(c, "k_unpack");
  if (field >= VFS_CSI && field <= VFS_KAJ) { c->metrics_set = true; c->ps.built = false; c->gab_valid = false; }
  if (field == VFS_PHI) c->ps.guess = c->ps.built;  // the next solve starts from the values set
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "vfs_set_field: copy failed");
  return rc;
}

int vfs_get_field(vfs_ctx *ctx, int field, double *host) {
  Ctx *c = (Ctx *)ctx;
  if (!c || !host || field < 0 || field >= VFS_NFIELDS) return set_err(c, VFS_ERR_INVALID, "vfs_get_field: bad argument");
  cudaSetDevice(c->device);
  const int dof = c->dof[field];
  const size_t bytes = sizeof(double) * (size_t)c->g.N * dof;
  int rc = ensure_stage(c, sizeof(double) * (size_t)c->g.N * 3);
  if (rc) return rc;
  double *stage = c->stage;
  c->launches++, k_pack<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(stage, dof, c->g.N, c->f[field][0],
                                                     c->f[field][1], c->f[field][2]);
  rc = check_launch(c, "k_pack");
  cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "vfs_get_field: copy failed");
  return rc;
}

int vfs_field_device_ptr(vfs_ctx *ctx, int field, int component, void **dptr) {
  Ctx *c = (Ctx *)ctx;
  if (!c || !dptr || field < 0 || field >= VFS_NFIELDS || component < 0 || component >= c->dof[field])
    return set_err(c, VFS_ERR_INVALID, "vfs_field_device_ptr: bad argument");
  *dptr = c->f[field][component];
  return VFS_OK;
}

int vfs_set_scalar(vfs_ctx *ctx, int which, double value) {
  Ctx *c = (Ctx *)ctx;
  if (!c || which < 0 || which >= VFS_NSCALARS) return set_err(c, VFS_ERR_INVALID, "vfs_set_scalar: bad argument");
  c->scal[which] = value;
  if (which == VFS_S_DT) c->g.dt = value;
  if (which == VFS_S_REN) c->g.ren = value;
  if (which == VFS_S_ST) c->g.st = value;
  // kernel arguments of a captured step change: capture again.  A captured step depends on
  // ti only through the tests ti > 0 (the wall model of the IB-node reconstruction) and
  // ti < 2 (the first LES steps, which are never captured)
  if (which == VFS_S_DT || which == VFS_S_REN || which == VFS_S_ST) c->setup_epoch++;
  if (which == VFS_S_TI) {
    const int ti = (int)value;
    if ((ti > 0) != (c->ti > 0) || (ti < 2) != (c->ti < 2)) c->setup_epoch++;
    c->ti = ti;
  }
  return ds_upload(c);
}

int vfs_get_scalar(vfs_ctx *ctx, int which, double *value) {
  Ctx *c = (Ctx *)ctx;
  if (!c || !value || which < 0 || which >= VFS_NSCALARS) return set_err(c, VFS_ERR_INVALID, "vfs_get_scalar: bad argument");
  if (which == VFS_S_TI) c->scal[VFS_S_TI] = c->ti;
  if (which == VFS_S_IB_UNRESOLVED) c->scal[which] = c->nib_unresolved;
  *value = c->scal[which];
  return VFS_OK;
}

#define VFS_REQUIRE_SETUP(c)                                                                   \
  do {                                                                                         \
    if (!(c)) return set_err(nullptr, VFS_ERR_INVALID, "null context");                       \
    if (!(c)->metrics_set) return set_err((c), VFS_ERR_STATE, "metrics have not been uploaded"); \
    cudaSetDevice((c)->device);                                                                \
  } while (0)

int vfs_contra2cart(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return contra2cart(c); }
int vfs_formfunction2(vfs_ctx *ctx, double scale) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return formfunction2(c, scale, false, 0.0); }
int vfs_pressure_gradient(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return pressure_gradient(c); }
int vfs_calc_k_flux(vfs_ctx *ctx, double *flux) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  double f = 0;
  int rc = calc_k_flux(c, &f);
  if (flux) *flux = f;
  return rc;
}
int vfs_smagorinsky_constant(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return smagorinsky_constant(c); }
int vfs_eddy_viscosity(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return eddy_viscosity(c); }
int vfs_runge_kutta(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return runge_kutta(c); }
int vfs_poisson_lhs(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return poisson_lhs(c); }
int vfs_poisson_rhs(vfs_ctx *ctx) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  if (!c->ps.built) { int rc = poisson_lhs(c); if (rc) return rc; }
  return poisson_rhs(c);
}
int vfs_poisson_solve(vfs_ctx *ctx, const vfs_solve_opts *o, vfs_solve_stats *st) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  if (!c->ps.built) { int rc = poisson_lhs(c); if (rc) return rc; }
  return poisson_solve(c, o, st);
}
int vfs_poisson_apply(vfs_ctx *ctx, const double *xh, double *yh) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  if (!xh || !yh) return set_err(c, VFS_ERR_INVALID, "vfs_poisson_apply: null array");
  if (!c->ps.built) { int rc = poisson_lhs(c); if (rc) return rc; }
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  double *dx = nullptr, *dy = nullptr;
  if (cudaMallocAsync(&dx, bytes, c->stream) != cudaSuccess || cudaMallocAsync(&dy, bytes, c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "vfs_poisson_apply: allocation failed");
  cudaMemcpyAsync(dx, xh, bytes, cudaMemcpyHostToDevice, c->stream);
  int rc = poisson_apply_dev(c, dx, dy);
  cudaMemcpyAsync(yh, dy, bytes, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(dx, c->stream);
  cudaFreeAsync(dy, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_poisson_apply: failed");
  return rc;
}
int vfs_update_pressure(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return update_pressure(c); }
int vfs_projection(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return projection(c); }
int vfs_divergence(vfs_ctx *ctx, double *maxdiv) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  double m = 0;
  int rc = divergence(c, &m);
  if (maxdiv) *maxdiv = m;
  return rc;
}

int vfs_calc_inlet_area(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return calc_inlet_area(c); }
int vfs_form_bcs(vfs_ctx *ctx, int outflow_scale) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return form_bcs(c, outflow_scale != 0);
}
int vfs_inflow_flux(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return inflow_flux(c); }
int vfs_set_inflow_plane(vfs_ctx *ctx, const double *plane) {
  Ctx *c = (Ctx *)ctx;
  if (!c || !plane) return set_err(c, VFS_ERR_INVALID, "vfs_set_inflow_plane: null argument");
  cudaSetDevice(c->device);
  const size_t bytes = sizeof(double) * 3 * (size_t)c->g.mx * c->g.my;
  if (!c->inflow_plane && cudaMalloc(&c->inflow_plane, bytes) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "vfs_set_inflow_plane: allocation failed");
  cudaMemcpyAsync(c->inflow_plane, plane, bytes, cudaMemcpyHostToDevice, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_set_inflow_plane: copy failed");
  return VFS_OK;
}
int vfs_volume_flux(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return volume_flux(c); }
int vfs_ib_bc(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return ib_bc(c); }
int vfs_ibm_interpolation(vfs_ctx *ctx) { Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c); return ibm_interpolation(c); }
int vfs_ibm_list(vfs_ctx *ctx, int *ints, double *dbls, int cap) {
  Ctx *c = (Ctx *)ctx;
  if (!c) return -VFS_ERR_INVALID;
  cudaSetDevice(c->device);
  if (ints && dbls && c->nib > 0) {
    std::vector<IbNode> h(c->nib);
    if (cudaMemcpy(h.data(), c->ibn, sizeof(IbNode) * c->nib, cudaMemcpyDeviceToHost) != cudaSuccess)
      return -set_err(c, VFS_ERR_CUDA, "vfs_ibm_list: copy failed");
    for (int q = 0; q < c->nib && q < cap; q++) {
      const IbNode &n = h[q];
      int *o = ints + 14 * (size_t)q;
      o[0] = n.i; o[1] = n.j; o[2] = n.k; o[3] = n.cell; o[4] = n.imode;
      for (int v = 0; v < 9; v++) o[5 + v] = n.st[v];
      double *d = dbls + 8 * (size_t)q;
      d[0] = n.cr[0]; d[1] = n.cr[1]; d[2] = n.cr[2]; d[3] = n.cs[0]; d[4] = n.cs[1]; d[5] = n.cs[2];
      d[6] = n.ds; d[7] = n.di;
    }
  }
  return c->nib;
}

int vfs_step(vfs_ctx *ctx, const vfs_solve_opts *opts, vfs_step_stats *st) {
  Ctx *c = (Ctx *)ctx; VFS_REQUIRE_SETUP(c);
  if (opts && opts->graph) return step_graph(c, opts, st);
  return step_core(c, opts, st);
}

}  // extern "C"

namespace vfs {
// One time step (vfs_step); with c->tape set it also records the stage states the
// tangent and adjoint steps need.
// The kernels of one time step after its set-up (Flow_Solver for implicit = 0,
// solvers.c:644-1385, and the old-value copies of the time loop): launched one by one, or
// captured into the step graph (c->capturing), where nothing waits for the host.
static int step_body(Ctx *c, const vfs_solve_opts *opts, vfs_step_stats *s, int *solve_rc) {
  int rc;
  if ((rc = calc_k_flux(c, &s->mean_k_flux))) return rc;
  if (c->g.les) {  // solvers.c:648-654
    if ((rc = contra2cart(c))) return rc;
    if ((c->ti % c->dynamic_freq == 0 || c->ti == c->tistart) && (rc = smagorinsky_constant(c))) return rc;
    if ((rc = eddy_viscosity(c))) return rc;
  }
  if ((rc = pressure_gradient(c))) return rc;
  if (c->cfg.implicit == 4) {  // solvers.c:1282-1289
    if ((rc = implicit_rhs_o(c))) return rc;
    // a Newton solve that stops at its iteration cap leaves the step going on, as the
    // reference's SNESSolve does
    if ((rc = implicit_momentum(c, nullptr)) && rc != VFS_ERR_NOT_CONVERGED) return rc;
  } else if ((rc = runge_kutta(c))) {
    return rc;
  }
  if ((rc = volume_flux(c))) return rc;  // poisson_hypre.c:566
  if ((rc = poisson_rhs(c))) return rc;
  rc = poisson_solve(c, opts, &s->poisson);
  if (rc && rc != VFS_ERR_NOT_CONVERGED) return rc;
  *solve_rc = rc;
  // UpdatePressure + Projection (solvers.c:1341-1342), with Divergence (solvers.c:1378)
  // formed in Projection's Contra2Cart when no IB-node reconstruction comes between
  const bool fuse_div = !c->g.immersed;
  if ((rc = correction(c, fuse_div))) return rc;
  if (c->g.immersed && (rc = ibm_interpolation(c))) return rc;  // solvers.c:1366-1370
  if ((rc = fuse_div ? divergence_finish(c, &s->max_div) : divergence(c, &s->max_div))) return rc;
  if ((rc = ib_bc(c))) return rc;
  if ((rc = contra2cart(c))) return rc;
  // end of the time step: keep Ucont and Ucat of this step (main.c:3584-3602), and with
  // immersed bodies the flags as Nvert_o (main.c:3571-3573)
  const size_t bytes = sizeof(double) * (size_t)c->g.N;
  if (c->g.immersed) {
    if (!c->nvo) {
      if (c->capturing) return set_err(c, VFS_ERR_STATE, "vfs_step: Nvert_o not allocated before capture");
      if (cudaMalloc(&c->nvo, (size_t)c->g.N) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_step: allocation failed");
    }
    cudaMemcpyAsync(c->nvo, c->nv, (size_t)c->g.N, cudaMemcpyDeviceToDevice, c->stream);
  }
  for (int q = 0; q < 3; q++) {
    cudaMemcpyAsync(c->f[VFS_UCONT_O][q], c->f[VFS_UCONT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->f[VFS_UCAT_O][q], c->f[VFS_UCAT][q], bytes, cudaMemcpyDeviceToDevice, c->stream);
  }
  return VFS_OK;
}

// One time step (vfs_step), its kernels launched one by one; with c->tape set it also
// records the stage states the tangent and adjoint steps need.
int step_core(Ctx *c, const vfs_solve_opts *opts, vfs_step_stats *st) {
  int rc;
  vfs_step_stats s;
  memset(&s, 0, sizeof(s));
  cudaEventRecord(c->ev0, c->stream);
  if (c->tape) c->tape->first_step = c->first_step;
  if (c->first_step) {
    // first time step: Calc_Inlet_Area (main.c:3488), PoissonLHSNew (poisson_hypre.c:527),
    // IB_BC (solvers.c:603-611)
    if ((rc = calc_inlet_area(c))) return rc;
    if ((rc = poisson_lhs(c))) return rc;
    if (c->g.immersed && (rc = ibm_interpolation(c))) return rc;
    if ((rc = ib_bc(c))) return rc;
    c->first_step = false;
  } else if (!c->ps.built && (rc = poisson_lhs(c))) {
    return rc;
  }
  int solve_rc = VFS_OK;
  if ((rc = step_body(c, opts, &s, &solve_rc))) return rc;
  c->ti++;
  cudaEventRecord(c->ev1, c->stream);
  cudaEventSynchronize(c->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  s.ms = ms;
  if (st) *st = s;
  return solve_rc;
}

void step_graph_free(Ctx *c) {
  if (c->sg.exec) cudaGraphExecDestroy(c->sg.exec);
  if (c->sg.graph) cudaGraphDestroy(c->sg.graph);
  c->sg.exec = nullptr;
  c->sg.graph = nullptr;
  c->sg.key = -1;
}

// Whether the next step is the same sequence of kernels as the last: no set-up work and no
// decision that changes from step to step.
static bool graph_eligible(const Ctx *c) {
  if (c->first_step || c->tape || !c->ps.built || c->g.moving || c->nsolid < 0 || c->cfg.implicit) return false;
  if (c->g.les && (c->dynamic_freq != 1 || (c->ti < 2 && c->tistart == 0 && !c->rstart))) return false;
  return true;
}

// The step as one CUDA graph: captured when it is missing or stale, then replayed.  The
// host reads back the device scalars and the solve's state after the replay.
int step_graph(Ctx *c, const vfs_solve_opts *opts, vfs_step_stats *st) {
  if (!graph_eligible(c)) return step_core(c, opts, st);
  int rc;
  if ((rc = ensure_gab(c))) return rc;   // set-up work stays outside the graph
  if ((rc = poisson_prepare(c, opts))) return rc;
  const bool fresh = c->sg.exec && c->sg.key == c->setup_epoch && !memcmp(&c->sg.opts, opts, sizeof(*opts));
  if (!fresh) {
    step_graph_free(c);
    const long long l0 = c->launches;
    vfs_step_stats s;
    memset(&s, 0, sizeof(s));
    int solve_rc = VFS_OK;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return set_err(c, VFS_ERR_CUDA, "vfs_step: stream capture failed to start");
    c->capturing = true;
    rc = step_body(c, opts, &s, &solve_rc);
    c->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      c->launches = l0;
      return rc ? rc : set_err(c, VFS_ERR_CUDA, std::string("vfs_step: capture failed: ") + cudaGetErrorString(e));
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      cudaGetLastError();
      c->launches = l0;
      return set_err(c, VFS_ERR_CUDA, "vfs_step: graph instantiation failed");
    }
    c->sg.graph = graph;
    c->sg.exec = exec;
    c->sg.opts = *opts;
    c->sg.key = c->setup_epoch;
    c->sg.launches = c->launches - l0;   // kernels of a step with one Krylov cycle and iteration
    c->launches = l0;
  }
  cudaEventRecord(c->ev0, c->stream);
  if (cudaGraphLaunch(c->sg.exec, c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_step: graph launch failed");
  cudaEventRecord(c->ev1, c->stream);
  cudaMemcpyAsync(c->ds_out, c->ds, sizeof(double) * DS_COUNT, cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(c->kd_host, c->kd, sizeof(KryDev), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_step: graph replay failed");
  const KryDev &k = *c->kd_host;
  c->launches += c->sg.launches + (long long)(k.it > 0 ? k.it - 1 : 0) * c->sg.body_launches +
                 (long long)(k.cycles > 0 ? k.cycles - 1 : 0) * c->sg.cycle_launches;
  c->scal[VFS_S_MEAN_K_FLUX] = c->ds_out[DS_MEAN_K_FLUX];
  c->scal[VFS_S_FLUX_IN] = c->ds_out[DS_FLUX_IN];
  c->scal[VFS_S_FLUX_OUT] = c->ds_out[DS_FLUX_OUT];
  vfs_step_stats s;
  memset(&s, 0, sizeof(s));
  s.mean_k_flux = c->ds_out[DS_MEAN_K_FLUX];
  s.max_div = c->ds_out[DS_MAXDIV];
  s.poisson.iterations = k.it;
  s.poisson.converged = k.conv ? 1 : 0;
  s.poisson.r0 = k.r0;
  s.poisson.rfinal = k.rnorm;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  s.ms = ms;
  s.poisson.ms = 0;  // not timed apart inside the graph
  c->ti++;
  if (st) *st = s;
  return s.poisson.converged ? VFS_OK : set_err(c, VFS_ERR_NOT_CONVERGED, "poisson_solve: iteration cap reached");
}
}  // namespace vfs
