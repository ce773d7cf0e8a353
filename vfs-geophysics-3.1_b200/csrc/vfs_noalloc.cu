// Contra2Cart for callers that cannot allocate device memory.
//
// Some host codes that would call this library run where cudaMalloc is not available to
// them: a solver embedded in a framework that owns every device allocation through its
// own pool, or a process whose memory budget is fixed before the solver starts.  They
// can hand over device buffers they already own, but the library must not allocate on
// their behalf.  vfs_contra2cart_noalloc serves them: it runs the same kernels as
// vfs_contra2cart on caller-owned buffers and keeps its scratch (the two-phase boundary
// buffer, the point flags and the byte copy of nvert) in one file-scope device array.
//
// The array is VFS_NOALLOC_SCRATCH_BYTES per GPU that loads the library and stays
// resident until the process exits.  Every call on a device shares it and it keeps the
// last call's contents; calls that overlap on the GPU (two streams, or two host threads)
// race on it.  Calls in order on one stream are safe.
#include <cstdio>
#include <string>

#include "vfs_internal.cuh"

// Kernels of the Contra2Cart path, defined in vfs_momentum.cu / vfs_api.cu.
namespace vfs {
__global__ void k_periodic_copy(Grid g, double *a, double *b, double *c);
__global__ void k_contra2cart_interior(Grid g, CV3 uc, CV3 csi, CV3 eta, CV3 zet, const uint8_t *__restrict__ nv,
                                       V3 ucat);
__global__ void k_contra2cart_bc(Grid g, Metrics m, const uint8_t *__restrict__ nv, CV3 lu, CV3 uo, V3 out,
                                 uint8_t *flag);
__global__ void k_bc_commit(long long n, CV3 in, uint8_t *flag, V3 dst);
}  // namespace vfs
__global__ void k_nvert_to_u8(const double *__restrict__ nvd, long long n, uint8_t *nv, int *bad);

namespace {

constexpr long long kMaxPoints = VFS_NOALLOC_MAX_POINTS;
// layout: boundary buffer 3*max doubles | nvert bytes | flag bytes | error word
constexpr size_t kBufBytes = sizeof(double) * 3 * kMaxPoints;
constexpr size_t kNvOff = kBufBytes;
constexpr size_t kFlagOff = kNvOff + kMaxPoints;
constexpr size_t kBadOff = kFlagOff + kMaxPoints;
constexpr size_t kScratchBytes = kBadOff + 256;
static_assert(kScratchBytes == VFS_NOALLOC_SCRATCH_BYTES, "scratch size must match the header");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch in the current device's context.  In host code the symbol
// names a host-side stand-in, not device memory, so it must never be passed to a kernel;
// the address comes from cudaGetSymbolAddress with the device current.  It is looked up
// on every call (a cheap query next to the launches and the synchronisation that follow),
// so a device reset or another context made current between calls never leaves a stale
// address behind, and no cache is shared between host threads.
int scratch_address(unsigned char **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess || !p)
    return vfs::set_err(nullptr, VFS_ERR_CUDA, std::string("vfs_contra2cart_noalloc: cudaGetSymbolAddress failed: ") +
                                                   cudaGetErrorString(e));
  *out = (unsigned char *)p;
  return VFS_OK;
}

}  // namespace

extern "C" int vfs_contra2cart_noalloc(const vfs_config *cfg, double *ucont, const double *csi, const double *eta,
                                       const double *zet, const double *nvert, const double *ucat_old, double *ucat,
                                       void *stream) {
  using namespace vfs;
  if (!cfg || !ucont || !csi || !eta || !zet || !nvert || !ucat_old || !ucat)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_contra2cart_noalloc: null argument");
  if (cfg->IM < 4 || cfg->JM < 4 || cfg->KM < 4)
    return set_err(nullptr, VFS_ERR_INVALID, "vfs_contra2cart_noalloc: grid needs at least 4 nodes per direction");
  Grid g{};
  g.mx = cfg->IM + 1; g.my = cfg->JM + 1; g.mz = cfg->KM + 1;
  g.N = (long long)g.mx * g.my * g.mz;
  if (g.N > kMaxPoints) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "vfs_contra2cart_noalloc: grid of %lld points exceeds the %lld-point limit of its static scratch",
             g.N, kMaxPoints);
    return set_err(nullptr, VFS_ERR_INVALID, msg);
  }
  g.iper = cfg->i_periodic; g.jper = cfg->j_periodic; g.kper = cfg->k_periodic;
  for (int q = 0; q < 6; q++) g.bc[q] = cfg->bctype[q];
  g.immersed = cfg->immersed; g.les = cfg->les;
  g.ren = cfg->ren; g.dt = cfg->dt; g.st = cfg->st;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_err(nullptr, VFS_ERR_NO_DEVICE, "vfs_contra2cart_noalloc: no CUDA device");
  unsigned char *s = nullptr;
  int rc = scratch_address(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const long long N = g.N;
  double *buf = (double *)s;
  V3 out{buf, buf + kMaxPoints, buf + 2 * kMaxPoints};
  uint8_t *nv = s + kNvOff, *flag = s + kFlagOff;
  int *bad = (int *)(s + kBadOff);
  // flags and the error word must start at zero whatever an earlier call left there
  cudaMemsetAsync(flag, 0, (size_t)N, st);
  cudaMemsetAsync(bad, 0, sizeof(int), st);
  const unsigned nb = nblocks(N, 256);
  k_nvert_to_u8<<<nb, 256, 0, st>>>(nvert, N, nv, bad);
  V3 uc{ucont, ucont + N, ucont + 2 * N};
  V3 u{ucat, ucat + N, ucat + 2 * N};
  CV3 c{csi, csi + N, csi + 2 * N}, e{eta, eta + N, eta + 2 * N}, z{zet, zet + N, zet + 2 * N};
  CV3 uo{ucat_old, ucat_old + N, ucat_old + 2 * N};
  const bool per = g.iper || g.jper || g.kper;
  if (per) k_periodic_copy<<<nb, 256, 0, st>>>(g, uc.x, uc.y, uc.z);
  k_contra2cart_interior<<<nb, 256, 0, st>>>(g, cv(uc), c, e, z, nv, u);
  if (per) k_periodic_copy<<<nb, 256, 0, st>>>(g, u.x, u.y, u.z);
  Metrics m{};
  m.csi = c; m.eta = e; m.zet = z;
  k_contra2cart_bc<<<nb, 256, 0, st>>>(g, m, nv, cv(u), uo, out, flag);
  k_bc_commit<<<nb, 256, 0, st>>>(N, cv(out), flag, u);
  if (per) k_periodic_copy<<<nb, 256, 0, st>>>(g, u.x, u.y, u.z);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess)
    return set_err(nullptr, VFS_ERR_CUDA, std::string("vfs_contra2cart_noalloc: launch failed: ") + cudaGetErrorString(ce));
  int hbad = 0;
  if (cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(nullptr, VFS_ERR_CUDA, "vfs_contra2cart_noalloc: stream synchronisation failed");
  if (hbad) return set_err(nullptr, VFS_ERR_INVALID, "vfs_contra2cart_noalloc: nvert must hold integers 0..255");
  return VFS_OK;
}
