// Immersed-body classification for sm_100a: the nvert flags of ibm_search_advanced
// (ibm.c:85-587) for a closed triangulated surface, bit for bit.
//
//   * host: the surface bounding box widened by 0.05, the 40 x 40 x 40 bins and each
//     triangle's bin range (ibm.c:132-198), the unit normals as the surface reader forms
//     them (ibm_io.c:869-880), and the ray-direction draws of randomdirection (ibm.c:52-84):
//     srand(n) then rand() for attempt n, reproduced with glibc's random_r on a private
//     state, so the caller's rand() sequence is left alone;
//   * k_ibm_cast: one thread per interior cell centre inside the box casts the ray of
//     point_cell_advanced (ibm.c:1068-1193) through the triangles of its bin column with the
//     Moller-Trumbore test of intsect_triangle (compgeom.c:17-53), retrying with the next
//     draw when two hits coincide (|t1 - t2| < 1e-8 with normals not opposite); an odd
//     number of hits marks the cell inside (4);
//   * k_ibm_near: every DA point (ghosts included) that is not inside but has an inside
//     point in its 3x3x3 neighbourhood becomes 2 (ibm.c:322-345);
//   * k_ibm_remap: interior 2 -> 1 and 4 -> 3 (ibm.c:507-514); ghost points keep a 2.
// The bin column of a cell holds every triangle whose bin range covers it; a triangle is
// tested once per ray, which is what the reference's Element_Searched bookkeeping does,
// and the hit count and the coincidence test do not depend on the order of the tests.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vfs_internal.cuh"

namespace vfs {

constexpr int kIbmBins = 40;       // ncx = ncy = ncz (ibm.c:103)
constexpr int kIbmAttempts = 256;  // ray directions tried before a cell is reported
constexpr int kIbmMaxHits = 64;    // crossings recorded per ray

struct IbmSurface {
  const double *x, *y, *z;         // vertices
  const int *n1, *n2, *n3;         // triangle vertex indices
  const double *nx, *ny, *nz;      // unit normals
  const int *col_start;            // bin column (i + j*40) -> first entry
  const int *col_tri;              // triangle of each entry
  const int *col_kmax;             // its bin range end in k
  const double *draw;              // s of attempt n (1-based) = rand()/(RAND_MAX+1) - 0.5
  double xmin, xmax, ymin, ymax, zmin, zmax, dcx, dcy, dcz;
};

// intsect_triangle (compgeom.c:17-53), in its operation order; returns the hit distance
// in *t when the ray hits the triangle.
__device__ __forceinline__ bool ray_triangle(const double o[3], const double d[3], const double v0[3],
                                             const double v1[3], const double v2[3], double *t) {
  const double e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
  const double e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
  const double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
  if (det > -0.00000001 && det < 0.00000001) return false;
  const double inv_det = 1.0 / det;
  const double tv[3] = {o[0] - v0[0], o[1] - v0[1], o[2] - v0[2]};
  const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv_det;
  if (u < 0.0 || u > 1.0) return false;
  const double qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
  const double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv_det;
  if (v < 0.0 || u + v > 1.0) return false;
  *t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv_det;
  return true;
}

// point_cell_advanced (ibm.c:1068-1193): 4 inside, 0 outside, -1 when every attempt hit a
// coincidence, -2 when a ray crossed more than kIbmMaxHits triangles.
__device__ int cast_cell(const IbmSurface &S, const double p[3], int ic, int jc, int kc) {
  double th[kIbmMaxHits];  // hit distances
  int tq[kIbmMaxHits];     // and their triangles
  const int c0 = S.col_start[jc * kIbmBins + ic], c1 = S.col_start[jc * kIbmBins + ic + 1];
  const double xpc = S.dcx * (ic + 0.5) + S.xmin;
  const double ypc = S.dcy * (jc + 0.5) + S.ymin;
  for (int attempt = 1; attempt <= kIbmAttempts; attempt++) {
    // randomdirection (ibm.c:52-84)
    const double s = S.draw[attempt];
    double dir[3] = {xpc + s * S.dcx - p[0], ypc + s * S.dcy - p[1], S.zmax + 0.2 - p[2]};
    const double len = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    dir[0] /= len; dir[1] /= len; dir[2] /= len;
    int nint = 0;
    bool singular = false;
    for (int e = c0; e < c1 && !singular; e++) {
      if (S.col_kmax[e] <= kc) continue;
      const int t = S.col_tri[e];
      const int a = S.n1[t], b = S.n2[t], c = S.n3[t];
      const double v0[3] = {S.x[a], S.y[a], S.z[a]}, v1[3] = {S.x[b], S.y[b], S.z[b]};
      const double v2[3] = {S.x[c], S.y[c], S.z[c]};
      double th_new;
      if (!ray_triangle(p, dir, v0, v1, v2, &th_new) || !(th_new > 0)) continue;
      const double nx = S.nx[t], ny = S.ny[t], nz = S.nz[t];
      if (nint >= kIbmMaxHits) return -2;
      // coincident crossings (ibm.c:1138-1152)
      for (int q = 0; q < nint; q++) {
        const double ndotn = S.nx[tq[q]] * nx + S.ny[tq[q]] * ny + S.nz[tq[q]] * nz;
        if (fabs(th_new - th[q]) < 1.e-8 && ndotn > -0.97) singular = true;
      }
      th[nint] = th_new;
      tq[nint] = t;
      nint++;
    }
    if (!singular) return (nint % 2) ? 4 : 0;
  }
  return -1;
}

__global__ void k_ibm_cast(Grid g, IbmSurface S, CV3 cent, uint8_t *nv, int reset, int *err) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int i = (int)(p % g.mx);
  const long long r = p / g.mx;
  const int j = (int)(r % g.my), k = (int)(r / g.my);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  int v = nv[p];
  if (reset && v < 5) v = 0;  // a new search starts from zero (ibm.c:233)
  const double px = cent.x[p], py = cent.y[p], pz = cent.z[p];
  if (px > S.xmin && px < S.xmax && py > S.ymin && py < S.ymax && pz > S.zmin && pz < S.zmax) {
    const int ic = (int)floor((px - S.xmin) / S.dcx);
    const int jc = (int)floor((py - S.ymin) / S.dcy);
    const int kc = (int)floor((pz - S.zmin) / S.dcz);
    const double pt[3] = {px, py, pz};
    const int val = cast_cell(S, pt, ic, jc, kc);
    if (val < 0) { atomicExch(err, val); return; }
    v = v > val ? v : val;
  }
  nv[p] = (uint8_t)v;
}

// Near-boundary marking (ibm.c:322-345) over every DA point, into out.
__global__ void k_ibm_near(Grid g, const uint8_t *__restrict__ nv, uint8_t *out) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int i = (int)(p % g.mx);
  const long long r = p / g.mx;
  const int j = (int)(r % g.my), k = (int)(r / g.my);
  int v = nv[p];
  if (v != 4) {
    const int ip = i < g.mx - 1 ? i + 1 : i, im = i > 0 ? i - 1 : i;
    const int jp = j < g.my - 1 ? j + 1 : j, jm = j > 0 ? j - 1 : j;
    const int kp = k < g.mz - 1 ? k + 1 : k, km = k > 0 ? k - 1 : k;
    bool near = false;
    for (int kk = km; kk <= kp; kk++)
      for (int jj = jm; jj <= jp; jj++)
        for (int ii = im; ii <= ip; ii++) near |= nv[lidx(g, ii, jj, kk)] == 4;
    if (near) v = v > 2 ? v : 2;
  }
  out[p] = (uint8_t)v;
}

// Back to 1 and 3 on the interior (ibm.c:507-514); the double field follows.
__global__ void k_ibm_remap(Grid g, const uint8_t *__restrict__ in, uint8_t *nv, double *nvd) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  const int i = (int)(p % g.mx);
  const long long r = p / g.mx;
  const int j = (int)(r % g.my), k = (int)(r / g.my);
  int v = in[p];
  if (i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2) {
    if (v == 2) v = 1;
    if (v == 4) v = 3;
  }
  nv[p] = (uint8_t)v;
  nvd[p] = (double)v;
}

int ibm_search(Ctx *c, int ibi, int n_v, const double *x, const double *y, const double *z, int n_elmt,
               const int *n1, const int *n2, const int *n3) {
  const Grid &g = c->g;
  if (n_v < 3 || n_elmt < 1) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: empty surface");
  for (int e = 0; e < n_elmt; e++)
    if (n1[e] < 0 || n1[e] >= n_v || n2[e] < 0 || n2[e] >= n_v || n3[e] < 0 || n3[e] >= n_v)
      return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: triangle vertex index out of range");
  // bounding box (ibm.c:132-149)
  double xmin = 1.e23, xmax = -1.e23, ymin = 1.e23, ymax = -1.e23, zmin = 1.e23, zmax = -1.e23;
  for (int q = 0; q < n_v; q++) {
    xmin = xmin < x[q] ? xmin : x[q]; xmax = xmax < x[q] ? x[q] : xmax;
    ymin = ymin < y[q] ? ymin : y[q]; ymax = ymax < y[q] ? y[q] : ymax;
    zmin = zmin < z[q] ? zmin : z[q]; zmax = zmax < z[q] ? z[q] : zmax;
  }
  xmin -= 0.05; xmax += 0.05; ymin -= 0.05; ymax += 0.05; zmin -= 0.05; zmax += 0.05;
  const int nb = kIbmBins;
  const double dcx = (xmax - xmin) / (nb - 1.), dcy = (ymax - ymin) / (nb - 1.), dcz = (zmax - zmin) / (nb - 1.);
  // bin ranges of the triangles (ibm.c:160-198) -> per (i, j) column lists
  std::vector<std::vector<std::pair<int, int>>> cols((size_t)nb * nb);
  std::vector<double> nf(3 * (size_t)n_elmt);
  for (int e = 0; e < n_elmt; e++) {
    const int a = n1[e], b = n2[e], cc = n3[e];
    auto mn = [](double p, double q, double r) { double m = p < q ? p : q; return m < r ? m : r; };
    auto mxf = [](double p, double q, double r) { double m = p < q ? q : p; return m < r ? r : m; };
    const double xv0 = mn(x[a], x[b], x[cc]), xv1 = mxf(x[a], x[b], x[cc]);
    const double yv0 = mn(y[a], y[b], y[cc]), yv1 = mxf(y[a], y[b], y[cc]);
    const double zv0 = mn(z[a], z[b], z[cc]), zv1 = mxf(z[a], z[b], z[cc]);
    int iv0 = (int)floor((xv0 - xmin) / dcx), iv1 = (int)(floor((xv1 - xmin) / dcx) + 1);
    int jv0 = (int)floor((yv0 - ymin) / dcy), jv1 = (int)(floor((yv1 - ymin) / dcy) + 1);
    int kv0 = (int)floor((zv0 - zmin) / dcz), kv1 = (int)(floor((zv1 - zmin) / dcz) + 1);
    iv0 = iv0 < 0 ? 0 : iv0; iv1 = iv1 > nb ? nb : iv1;
    jv0 = jv0 < 0 ? 0 : jv0; jv1 = jv1 > nb ? nb : jv1;
    kv0 = kv0 < 0 ? 0 : kv0; kv1 = kv1 > nb ? nb : kv1;
    if (kv0 < kv1)
      for (int jj = jv0; jj < jv1; jj++)
        for (int ii = iv0; ii < iv1; ii++) cols[(size_t)jj * nb + ii].push_back({e, kv1});
    // unit normal as the surface reader forms it (ibm_io.c:869-880)
    const double dx12 = x[b] - x[a], dy12 = y[b] - y[a], dz12 = z[b] - z[a];
    const double dx13 = x[cc] - x[a], dy13 = y[cc] - y[a], dz13 = z[cc] - z[a];
    double fx = dy12 * dz13 - dz12 * dy13, fy = -dx12 * dz13 + dz12 * dx13, fz = dx12 * dy13 - dy12 * dx13;
    const double dr = sqrt(fx * fx + fy * fy + fz * fz);
    nf[3 * (size_t)e] = fx / dr; nf[3 * (size_t)e + 1] = fy / dr; nf[3 * (size_t)e + 2] = fz / dr;
  }
  std::vector<int> col_start((size_t)nb * nb + 1, 0), col_tri, col_kmax;
  for (size_t q = 0; q < cols.size(); q++) {
    col_start[q] = (int)col_tri.size();
    for (auto &pr : cols[q]) { col_tri.push_back(pr.first); col_kmax.push_back(pr.second); }
  }
  col_start[cols.size()] = (int)col_tri.size();
  // ray draws: srand(n); rand() for n = 1..kIbmAttempts, on a private generator state
  std::vector<double> draw(kIbmAttempts + 1, 0.0);
  for (int n = 1; n <= kIbmAttempts; n++) {
    struct random_data rd;
    char state[128];
    memset(&rd, 0, sizeof(rd));
    memset(state, 0, sizeof(state));
    initstate_r((unsigned)n, state, sizeof(state), &rd);
    srandom_r((unsigned)n, &rd);
    int32_t rv = 0;
    random_r(&rd, &rv);
    draw[n] = rv / ((double)RAND_MAX + 1) - 0.5;
  }
  // device copies (set-up only)
  std::vector<double> nx(n_elmt), ny(n_elmt), nz(n_elmt);
  for (int e = 0; e < n_elmt; e++) { nx[e] = nf[3 * (size_t)e]; ny[e] = nf[3 * (size_t)e + 1]; nz[e] = nf[3 * (size_t)e + 2]; }
  const size_t nt = col_tri.size() > 0 ? col_tri.size() : 1;
  const size_t bytes = sizeof(double) * (3 * (size_t)n_v + 3 * (size_t)n_elmt + kIbmAttempts + 1) +
                       sizeof(int) * (3 * (size_t)n_elmt + col_start.size() + 2 * nt) + sizeof(int) + 256;
  char *buf = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: allocation failed");
  size_t off = 0;
  auto put = [&](const void *src, size_t n) {
    void *dst = buf + off;
    if (n) cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, c->stream);
    off += (n + 15) & ~(size_t)15;
    return dst;
  };
  IbmSurface S;
  S.x = (const double *)put(x, sizeof(double) * n_v);
  S.y = (const double *)put(y, sizeof(double) * n_v);
  S.z = (const double *)put(z, sizeof(double) * n_v);
  S.nx = (const double *)put(nx.data(), sizeof(double) * n_elmt);
  S.ny = (const double *)put(ny.data(), sizeof(double) * n_elmt);
  S.nz = (const double *)put(nz.data(), sizeof(double) * n_elmt);
  S.draw = (const double *)put(draw.data(), sizeof(double) * draw.size());
  S.n1 = (const int *)put(n1, sizeof(int) * n_elmt);
  S.n2 = (const int *)put(n2, sizeof(int) * n_elmt);
  S.n3 = (const int *)put(n3, sizeof(int) * n_elmt);
  S.col_start = (const int *)put(col_start.data(), sizeof(int) * col_start.size());
  S.col_tri = (const int *)put(col_tri.data(), sizeof(int) * col_tri.size());
  S.col_kmax = (const int *)put(col_kmax.data(), sizeof(int) * col_kmax.size());
  int *err = (int *)(buf + off);
  cudaMemsetAsync(err, 0, sizeof(int), c->stream);
  S.xmin = xmin; S.xmax = xmax; S.ymin = ymin; S.ymax = ymax; S.zmin = zmin; S.zmax = zmax;
  S.dcx = dcx; S.dcy = dcy; S.dcz = dcz;
  int rc;
  k_ibm_cast<<<nblocks(g.N, 128), 128, 0, c->stream>>>(g, S, cv(field3(c, VFS_CENT)), c->nv, ibi == 0 ? 1 : 0, err);
  if ((rc = check_launch(c, "k_ibm_cast"))) { cudaFree(buf); return rc; }
  k_ibm_near<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nv, c->bcflag);
  if ((rc = check_launch(c, "k_ibm_near"))) { cudaFree(buf); return rc; }
  k_ibm_remap<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->bcflag, c->nv, c->f[VFS_NVERT][0]);
  if ((rc = check_launch(c, "k_ibm_remap"))) { cudaFree(buf); return rc; }
  cudaMemsetAsync(c->bcflag, 0, (size_t)g.N, c->stream);  // Contra2Cart's flag buffer, clear again
  int herr = 0;
  cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    cudaFree(buf);
    return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: kernel failed");
  }
  cudaFree(buf);
  if (herr == -1) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: a cell's rays kept hitting coincident crossings");
  if (herr == -2) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: a ray crossed too many triangles");
  c->nvert_set = true;
  c->nsolid = -1;
  c->ps.built = false;
  return VFS_OK;
}

}  // namespace vfs

extern "C" int vfs_ibm_search(vfs_ctx *ctx, int ibi, int n_v, const double *x, const double *y, const double *z,
                              int n_elmt, const int *nv1, const int *nv2, const int *nv3) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !x || !y || !z || !nv1 || !nv2 || !nv3 || ibi < 0)
    return vfs::set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: bad argument");
  if (!c->metrics_set) return vfs::set_err(c, VFS_ERR_STATE, "vfs_ibm_search: metrics (cell centres) not set");
  cudaSetDevice(c->device);
  return vfs::ibm_search(c, ibi, n_v, x, y, z, n_elmt, nv1, nv2, nv3);
}
