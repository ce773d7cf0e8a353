// Grid metrics on the device: FormMetrics (metrics.c:4-1347, the NEWMETRIC branch) from
// the node coordinates of grid.dat.
//
// Pass order follows the reference so every value, ghost planes included, is the same:
//   1. cell centres and centre metrics csi/eta/zet, aj = 1/J at interior cells
//      (metrics.c:82-252);
//   2. ghost planes of the centre metrics copied from their neighbour plane, i planes
//      first, then j, then k (metrics.c:255-335) - three launches keep that cascade;
//   3. periodic images of the centre metrics (metrics.c:345-375);
//   4. face metrics as the average of the two adjacent centre metrics and the harmonic
//      mean of aj (metrics.c:580-585, 688-693, 796-801), zero outside the face ranges;
//   5. periodic images of every metric array (metrics.c:1240-1270).
#include "vfs_internal.cuh"

namespace vfs {

struct Nodes {
  const double *x, *y, *z;
  int IM, JM, KM;
};

__device__ __forceinline__ long long nidx(const Nodes &n, int i, int j, int k) {
  return ((long long)k * n.JM + j) * n.IM + i;
}

__global__ void k_centre_metrics(Grid g, Nodes n, V3 cent, V3 csi, V3 eta, V3 zet, double *aj) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  const long long a000 = nidx(n, i, j, k), a010 = nidx(n, i, j - 1, k), a100 = nidx(n, i, j, k - 1),
                  a110 = nidx(n, i, j - 1, k - 1), b000 = nidx(n, i - 1, j, k),
                  b010 = nidx(n, i - 1, j - 1, k), b100 = nidx(n, i - 1, j, k - 1),
                  b110 = nidx(n, i - 1, j - 1, k - 1);
  // coor[k][j][i], coor[k][j-1][i], coor[k-1][j][i], coor[k-1][j-1][i], then i-1
  const double *X = n.x, *Y = n.y, *Z = n.z;
  cent.x[p] = 0.125 * (X[a000] + X[a010] + X[a100] + X[a110] + X[b000] + X[b010] + X[b100] + X[b110]);
  cent.y[p] = 0.125 * (Y[a000] + Y[a010] + Y[a100] + Y[a110] + Y[b000] + Y[b010] + Y[b100] + Y[b110]);
  cent.z[p] = 0.125 * (Z[a000] + Z[a010] + Z[a100] + Z[a110] + Z[b000] + Z[b010] + Z[b100] + Z[b110]);
  // d/dcsi: i minus i-1, summed over the four (j,k) corners
  const double dxdc = 0.25 * (X[a000] + X[a010] + X[a100] + X[a110] - X[b000] - X[b010] - X[b100] - X[b110]);
  const double dydc = 0.25 * (Y[a000] + Y[a010] + Y[a100] + Y[a110] - Y[b000] - Y[b010] - Y[b100] - Y[b110]);
  const double dzdc = 0.25 * (Z[a000] + Z[a010] + Z[a100] + Z[a110] - Z[b000] - Z[b010] - Z[b100] - Z[b110]);
  // d/deta: coor[k][j][i] + coor[k][j][i-1] + coor[k-1][j][i] + coor[k-1][j][i-1] - (j-1 ...)
  const double dxde = 0.25 * (X[a000] + X[b000] + X[a100] + X[b100] - X[a010] - X[b010] - X[a110] - X[b110]);
  const double dyde = 0.25 * (Y[a000] + Y[b000] + Y[a100] + Y[b100] - Y[a010] - Y[b010] - Y[a110] - Y[b110]);
  const double dzde = 0.25 * (Z[a000] + Z[b000] + Z[a100] + Z[b100] - Z[a010] - Z[b010] - Z[a110] - Z[b110]);
  // d/dzeta: coor[k][j][i] + coor[k][j-1][i] + coor[k][j][i-1] + coor[k][j-1][i-1] - (k-1 ...)
  const double dxdz = 0.25 * (X[a000] + X[a010] + X[b000] + X[b010] - X[a100] - X[a110] - X[b100] - X[b110]);
  const double dydz = 0.25 * (Y[a000] + Y[a010] + Y[b000] + Y[b010] - Y[a100] - Y[a110] - Y[b100] - Y[b110]);
  const double dzdz = 0.25 * (Z[a000] + Z[a010] + Z[b000] + Z[b010] - Z[a100] - Z[a110] - Z[b100] - Z[b110]);
  double J = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) +
             dzdc * (dxde * dydz - dyde * dxdz);
  aj[p] = 1. / J;
  csi.x[p] = dyde * dzdz - dzde * dydz;
  csi.y[p] = -dxde * dzdz + dzde * dxdz;
  csi.z[p] = dxde * dydz - dyde * dxdz;
  eta.x[p] = dydz * dzdc - dzdz * dydc;
  eta.y[p] = -dxdz * dzdc + dzdz * dxdc;
  eta.z[p] = dxdz * dydc - dydz * dxdc;
  zet.x[p] = dydc * dzde - dzdc * dyde;
  zet.y[p] = -dxdc * dzde + dzdc * dxde;
  zet.z[p] = dxdc * dyde - dydc * dxde;
}

// Ghost plane copy for direction d (0: i, 1: j, 2: k): plane 0 <- plane 1 and plane m-1
// <- plane m-2, over the whole extent of the other two indices.
__global__ void k_ghost_plane(Grid g, int d, V3 csi, V3 eta, V3 zet, double *aj) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  long long s;
  if (d == 0) {
    if (i == 0) s = p + 1; else if (i == g.mx - 1) s = p - 1; else return;
  } else if (d == 1) {
    if (j == 0) s = p + g.mx; else if (j == g.my - 1) s = p - g.mx; else return;
  } else {
    const long long sz = (long long)g.mx * g.my;
    if (k == 0) s = p + sz; else if (k == g.mz - 1) s = p - sz; else return;
  }
  csi.x[p] = csi.x[s]; csi.y[p] = csi.y[s]; csi.z[p] = csi.z[s];
  eta.x[p] = eta.x[s]; eta.y[p] = eta.y[s]; eta.z[p] = eta.z[s];
  zet.x[p] = zet.x[s]; zet.y[p] = zet.y[s]; zet.z[p] = zet.z[s];
  aj[p] = aj[s];
}

// Face metrics (NEWMETRIC): average of the two centre metrics, harmonic mean of aj.
__global__ void k_face_metrics(Grid g, CV3 csi, CV3 eta, CV3 zet, const double *aj, V3 icsi, V3 ieta,
                               V3 izet, double *iaj, V3 jcsi, V3 jeta, V3 jzet, double *jaj, V3 kcsi,
                               V3 keta, V3 kzet, double *kaj) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  const int mx = g.mx, my = g.my, mz = g.mz;
  const bool ii = i >= 1 && i <= mx - 2, jj = j >= 1 && j <= my - 2, kk = k >= 1 && k <= mz - 2;
  // i faces: i = 0..mx-2, interior j and k (metrics.c:488-585)
  if (i <= mx - 2 && jj && kk) {
    const long long e = p + 1;
    icsi.x[p] = 0.5 * csi.x[p] + 0.5 * csi.x[e]; icsi.y[p] = 0.5 * csi.y[p] + 0.5 * csi.y[e];
    icsi.z[p] = 0.5 * csi.z[p] + 0.5 * csi.z[e];
    ieta.x[p] = 0.5 * eta.x[p] + 0.5 * eta.x[e]; ieta.y[p] = 0.5 * eta.y[p] + 0.5 * eta.y[e];
    ieta.z[p] = 0.5 * eta.z[p] + 0.5 * eta.z[e];
    izet.x[p] = 0.5 * zet.x[p] + 0.5 * zet.x[e]; izet.y[p] = 0.5 * zet.y[p] + 0.5 * zet.y[e];
    izet.z[p] = 0.5 * zet.z[p] + 0.5 * zet.z[e];
    iaj[p] = 2. / (1. / aj[p] + 1. / aj[e]);
  } else {
    icsi.x[p] = icsi.y[p] = icsi.z[p] = 0; ieta.x[p] = ieta.y[p] = ieta.z[p] = 0;
    izet.x[p] = izet.y[p] = izet.z[p] = 0; iaj[p] = 0;
  }
  // j faces: j = 0..my-2, interior i and k (metrics.c:600-693)
  if (j <= my - 2 && ii && kk) {
    const long long e = p + mx;
    jcsi.x[p] = 0.5 * csi.x[p] + 0.5 * csi.x[e]; jcsi.y[p] = 0.5 * csi.y[p] + 0.5 * csi.y[e];
    jcsi.z[p] = 0.5 * csi.z[p] + 0.5 * csi.z[e];
    jeta.x[p] = 0.5 * eta.x[p] + 0.5 * eta.x[e]; jeta.y[p] = 0.5 * eta.y[p] + 0.5 * eta.y[e];
    jeta.z[p] = 0.5 * eta.z[p] + 0.5 * eta.z[e];
    jzet.x[p] = 0.5 * zet.x[p] + 0.5 * zet.x[e]; jzet.y[p] = 0.5 * zet.y[p] + 0.5 * zet.y[e];
    jzet.z[p] = 0.5 * zet.z[p] + 0.5 * zet.z[e];
    jaj[p] = 2. / (1. / aj[p] + 1. / aj[e]);
  } else {
    jcsi.x[p] = jcsi.y[p] = jcsi.z[p] = 0; jeta.x[p] = jeta.y[p] = jeta.z[p] = 0;
    jzet.x[p] = jzet.y[p] = jzet.z[p] = 0; jaj[p] = 0;
  }
  // k faces: k = 0..mz-2, interior i and j (metrics.c:708-801)
  if (k <= mz - 2 && ii && jj) {
    const long long e = p + (long long)mx * my;
    kcsi.x[p] = 0.5 * csi.x[p] + 0.5 * csi.x[e]; kcsi.y[p] = 0.5 * csi.y[p] + 0.5 * csi.y[e];
    kcsi.z[p] = 0.5 * csi.z[p] + 0.5 * csi.z[e];
    keta.x[p] = 0.5 * eta.x[p] + 0.5 * eta.x[e]; keta.y[p] = 0.5 * eta.y[p] + 0.5 * eta.y[e];
    keta.z[p] = 0.5 * eta.z[p] + 0.5 * eta.z[e];
    kzet.x[p] = 0.5 * zet.x[p] + 0.5 * zet.x[e]; kzet.y[p] = 0.5 * zet.y[p] + 0.5 * zet.y[e];
    kzet.z[p] = 0.5 * zet.z[p] + 0.5 * zet.z[e];
    kaj[p] = 2. / (1 / aj[p] + 1 / aj[e]);
  } else {
    kcsi.x[p] = kcsi.y[p] = kcsi.z[p] = 0; keta.x[p] = keta.y[p] = keta.z[p] = 0;
    kzet.x[p] = kzet.y[p] = kzet.z[p] = 0; kaj[p] = 0;
  }
}

int form_metrics(Ctx *c, const double *x, const double *y, const double *z) {
  const Grid &g = c->g;
  int rc;
  const int IM = c->cfg.IM, JM = c->cfg.JM, KM = c->cfg.KM;
  const size_t nn = (size_t)IM * JM * KM;
  double *d = nullptr;
  if (cudaMallocAsync(&d, sizeof(double) * nn * 3, c->stream) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "form_metrics: staging allocation failed");
  cudaMemcpyAsync(d, x, sizeof(double) * nn, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(d + nn, y, sizeof(double) * nn, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(d + 2 * nn, z, sizeof(double) * nn, cudaMemcpyHostToDevice, c->stream);
  Nodes n{d, d + nn, d + 2 * nn, IM, JM, KM};
  // every metric array starts at zero, as the reference's freshly created Vecs do
  for (int f = VFS_CENT; f <= VFS_KAJ; f++)
    for (int q = 0; q < c->dof[f]; q++)
      cudaMemsetAsync(c->f[f][q], 0, sizeof(double) * (size_t)g.N, c->stream);
  V3 csi = field3(c, VFS_CSI), eta = field3(c, VFS_ETA), zet = field3(c, VFS_ZET);
  double *aj = c->f[VFS_AJ][0];
  c->launches++, k_centre_metrics<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, n, field3(c, VFS_CENT), csi, eta, zet, aj);
  if ((rc = check_launch(c, "k_centre_metrics"))) return rc;
  for (int dd = 0; dd < 3; dd++) {
    c->launches++, k_ghost_plane<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, dd, csi, eta, zet, aj);
    if ((rc = check_launch(c, "k_ghost_plane"))) return rc;
  }
  const int fields_c[4] = {VFS_CSI, VFS_ETA, VFS_ZET, VFS_AJ};
  for (int f : fields_c) {
    if (c->dof[f] == 3) rc = periodic_copy3(c, field3(c, f));
    else rc = periodic_copy1(c, c->f[f][0]);
    if (rc) return rc;
  }
  c->launches++, k_face_metrics<<<nblocks(g.N, 256), 256, 0, c->stream>>>(
      g, cv(csi), cv(eta), cv(zet), aj, field3(c, VFS_ICSI), field3(c, VFS_IETA), field3(c, VFS_IZET),
      c->f[VFS_IAJ][0], field3(c, VFS_JCSI), field3(c, VFS_JETA), field3(c, VFS_JZET), c->f[VFS_JAJ][0],
      field3(c, VFS_KCSI), field3(c, VFS_KETA), field3(c, VFS_KZET), c->f[VFS_KAJ][0]);
  if ((rc = check_launch(c, "k_face_metrics"))) return rc;
  for (int f = VFS_ICSI; f <= VFS_KAJ; f++) {
    if (c->dof[f] == 3) rc = periodic_copy3(c, field3(c, f));
    else rc = periodic_copy1(c, c->f[f][0]);
    if (rc) return rc;
  }
  // the node plane k = 1 (x, y, z blocks), for inlet profiles given in node coordinates
  const size_t plane = (size_t)IM * JM;
  if (!c->inlet_nodes && cudaMalloc(&c->inlet_nodes, sizeof(double) * plane * 3) != cudaSuccess)
    return set_err(c, VFS_ERR_CUDA, "form_metrics: node-plane allocation failed");
  for (int q = 0; q < 3; q++)
    cudaMemcpyAsync(c->inlet_nodes + q * plane, d + q * nn + plane, sizeof(double) * plane, cudaMemcpyDeviceToDevice,
                    c->stream);
  cudaFreeAsync(d, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "form_metrics failed");
  c->metrics_set = true;
  c->gab_valid = false;
  c->ps.built = false;
  return VFS_OK;
}

}  // namespace vfs

extern "C" int vfs_form_metrics(vfs_ctx *ctx, const double *x, const double *y, const double *z) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !x || !y || !z) return vfs::set_err(c, VFS_ERR_INVALID, "vfs_form_metrics: null argument");
  cudaSetDevice(c->device);
  return vfs::form_metrics(c, x, y, z);
}
