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
#include <algorithm>
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
  int nelmt;
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
  int i, j, k;
  dijk(g, p, i, j, k);
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
  int i, j, k;
  dijk(g, p, i, j, k);
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

// Cells that were inside a body at the end of the last step (Nvert_o > 2.5) and are
// now plain fluid become IB nodes (ibm.c:346-357, the search of the last body).
__global__ void k_ibm_phase(Grid g, const uint8_t *__restrict__ nvo, uint8_t *fl) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  if (nvo[p] >= 3 && fl[p] == 0) fl[p] = 2;
}

// Back to 1 and 3 on the interior (ibm.c:507-514); the double field follows.
__global__ void k_ibm_remap(Grid g, const uint8_t *__restrict__ in, uint8_t *nv, double *nvd) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  int v = in[p];
  if (i >= 1 && i <= g.mx - 2 && j >= 1 && j <= g.my - 2 && k >= 1 && k <= g.mz - 2) {
    if (v == 2) v = 1;
    if (v == 4) v = 3;
  }
  nv[p] = (uint8_t)v;
  nvd[p] = (double)v;
}

// ------------------------------------------------------------------ IB-node list
// The list ibm_search_advanced builds for the cells it marks 2 (ibm.c:347-505): the nearest
// surface point (nearestcell1, ibm.c:1366; BoundingSphere ibm.c:1276 prunes the search),
// the interception of the surface normal through the node with the cell-centre triangles
// of the six neighbouring faces (InterceptionPoint ibm.c:1759 with ICP ibm.c:1659), and the
// two boundary fallbacks.  Geometry helpers of compgeom.c in their operation order.
struct P2 { double x, y; };
struct P3 { double x, y, z; };

__device__ __forceinline__ double dist3(const P3 &a, const P3 &b) {
  return sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z));
}

// ISSameSide2D (compgeom.c:55-106); its first pair of t1/t2 is recomputed unconditionally
// in the reference, so only the second form is evaluated here.
__device__ int same_side2d(P2 p, P2 p1, P2 p2, P2 p3) {
  const double t1 = (p.x - p1.x) * (p2.y - p1.y) - (p.y - p1.y) * (p2.x - p1.x);
  const double t2 = (p3.x - p1.x) * (p2.y - p1.y) - (p3.y - p1.y) * (p2.x - p1.x);
  const double lt = sqrt((p1.x - p2.x) * (p1.x - p2.x) + (p1.y - p2.y) * (p1.y - p2.y));
  if (fabs(t1 / lt) < 1.e-10) return 1;
  if (t1 > 0) return t2 > 0 ? 1 : -1;
  return t2 < 0 ? 1 : -1;
}

// ISInsideTriangle2D (compgeom.c:108-129)
__device__ int inside_triangle2d(P2 p, P2 a, P2 b, P2 c) {
  int ls = same_side2d(p, a, b, c);
  if (ls < 0) return ls;
  ls = same_side2d(p, b, c, a);
  if (ls < 0) return ls;
  return same_side2d(p, c, a, b);
}

// ISPointInTriangle (compgeom.c:131-158): the test in the plane the normal dominates.
__device__ int point_in_triangle(P3 p, P3 p1, P3 p2, P3 p3, double nfx, double nfy, double nfz) {
  P2 q, q1, q2, q3;
  if (fabs(nfz) >= fabs(nfx) && fabs(nfz) >= fabs(nfy)) {
    q = {p.x, p.y}; q1 = {p1.x, p1.y}; q2 = {p2.x, p2.y}; q3 = {p3.x, p3.y};
  } else if (fabs(nfx) >= fabs(nfy) && fabs(nfx) >= fabs(nfz)) {
    q = {p.z, p.y}; q1 = {p1.z, p1.y}; q2 = {p2.z, p2.y}; q3 = {p3.z, p3.y};
  } else {
    q = {p.x, p.z}; q1 = {p1.x, p1.z}; q2 = {p2.x, p2.z}; q3 = {p3.x, p3.z};
  }
  return inside_triangle2d(q, q1, q2, q3);
}

// Dis_P_Line (compgeom.c:160-186): nearest point of segment p1p2 to p, and its distance.
__device__ void dist_point_segment(P3 p, P3 p1, P3 p2, P3 *po, double *d) {
  const double dx21 = p2.x - p1.x, dy21 = p2.y - p1.y, dz21 = p2.z - p1.z;
  const double dx31 = p.x - p1.x, dy31 = p.y - p1.y, dz31 = p.z - p1.z;
  const double t = (dx31 * dx21 + dy31 * dy21 + dz31 * dz21) / (dx21 * dx21 + dy21 * dy21 + dz21 * dz21);
  if (t < 0) {
    *po = p1;
    *d = sqrt(dx31 * dx31 + dy31 * dy31 + dz31 * dz31);
  } else if (t > 1) {
    *po = p2;
    *d = sqrt((p.x - po->x) * (p.x - po->x) + (p.y - po->y) * (p.y - po->y) + (p.z - po->z) * (p.z - po->z));
  } else {
    po->x = p1.x + t * dx21; po->y = p1.y + t * dy21; po->z = p1.z + t * dz21;
    *d = sqrt((p.x - po->x) * (p.x - po->x) + (p.y - po->y) * (p.y - po->y) + (p.z - po->z) * (p.z - po->z));
  }
}

// triangle_intp / triangle_intp2 (compgeom.c:188-226): barycentric weights in 2-D.
__device__ void bary2d(P2 p, P2 p1, P2 p2, P2 p3, double w[3]) {
  const double x13 = p1.x - p3.x, y13 = p1.y - p3.y;
  const double x23 = p2.x - p3.x, y23 = p2.y - p3.y;
  const double xp3 = p.x - p3.x, yp3 = p.y - p3.y;
  const double a = x13 * y23 - x23 * y13;
  w[0] = (y23 * xp3 - x23 * yp3) / a;
  w[1] = (-y13 * xp3 + x13 * yp3) / a;
  w[2] = 1. - w[0] - w[1];
}

// Weights of point q in triangle (t1, t2, t3) projected on the plane the normal n
// dominates, with the reference's coordinate choice (ibm.c:1481-1505, ibm.c:1717-1737).
__device__ bool bary_by_normal(P3 q, P3 t1, P3 t2, P3 t3, double nx, double ny, double nz, double w[3]) {
  if (fabs(nx) >= fabs(ny) && fabs(nx) >= fabs(nz)) {
    bary2d({q.y, q.z}, {t1.y, t1.z}, {t2.y, t2.z}, {t3.y, t3.z}, w);
  } else if (fabs(ny) >= fabs(nx) && fabs(ny) >= fabs(nz)) {
    bary2d({q.x, q.z}, {t1.x, t1.z}, {t2.x, t2.z}, {t3.x, t3.z}, w);
  } else if (fabs(nz) >= fabs(ny) && fabs(nz) >= fabs(nx)) {
    bary2d({q.y, q.x}, {t1.y, t1.x}, {t2.y, t2.x}, {t3.y, t3.x}, w);
  } else {
    return false;
  }
  return true;
}

// Doubles per IB node in the reconstruction buffer: velocity (3), pressure, ustar.
constexpr int kIbOut = 5;

struct IbmGeom {
  IbmSurface S;
  const double *qx, *qy, *qz, *rad;  // bounding spheres (BoundingSphere)
  CV3 cent;
  const long long *cells;            // node cells (linear DA index), ascending
  int n;
  int vbase;                         // first vertex of this body in the surface-velocity array
};

// The triangle data the reconstruction reads: its vertices (for the surface velocity,
// ibm.c:3430-3433) and its unit normal (the wall models' n).
__device__ __forceinline__ void node_triangle(const IbmGeom &G, IbNode &N) {
  const int e = N.cell;
  N.vtx[0] = G.vbase + G.S.n1[e]; N.vtx[1] = G.vbase + G.S.n2[e]; N.vtx[2] = G.vbase + G.S.n3[e];
  N.nf[0] = G.S.nx[e]; N.nf[1] = G.S.ny[e]; N.nf[2] = G.S.nz[e];
}

__device__ __forceinline__ P3 vtx(const IbmSurface &S, int v) { return {S.x[v], S.y[v], S.z[v]}; }

// ICP (ibm.c:1659-1757): interception of the ray p + d n (d > 0) with the eight triangles
// of the nine face cell centres pc; returns the triangle (0..7) or -100.
__device__ int icp(P3 p, const P3 pc[9], double nfx, double nfy, double nfz, double cr[3], double *d_i) {
  const int tri[3][8] = {{0, 1, 2, 4, 4, 4, 3, 3}, {1, 2, 4, 5, 7, 6, 4, 4}, {4, 4, 5, 8, 8, 7, 6, 0}};
  for (int t = 0; t < 8; t++) {
    const P3 p1 = pc[tri[0][t]], p2 = pc[tri[1][t]], p3 = pc[tri[2][t]];
    const double dx1 = p.x - p1.x, dy1 = p.y - p1.y, dz1 = p.z - p1.z;
    const double dx2 = p2.x - p1.x, dy2 = p2.y - p1.y, dz2 = p2.z - p1.z;
    const double dx3 = p3.x - p1.x, dy3 = p3.y - p1.y, dz3 = p3.z - p1.z;
    double d = (nfx * (dy2 * dz3 - dz2 * dy3) - nfy * (dx2 * dz3 - dz2 * dx3) + nfz * (dx2 * dy3 - dy2 * dx3));
    if (!(fabs(d) > 1.e-10)) continue;
    d = -(dx1 * (dy2 * dz3 - dz2 * dy3) - dy1 * (dx2 * dz3 - dz2 * dx3) + dz1 * (dx2 * dy3 - dy2 * dx3)) / d;
    if (!(d > 0)) continue;
    const P3 pint = {p.x + d * nfx, p.y + d * nfy, p.z + d * nfz};
    const double rx1 = p2.x - p1.x, ry1 = p2.y - p1.y, rz1 = p2.z - p1.z;
    const double rx2 = p3.x - p1.x, ry2 = p3.y - p1.y, rz2 = p3.z - p1.z;
    const double nxt = ry1 * rz2 - rz1 * ry2, nyt = -rx1 * rz2 + rz1 * rx2, nzt = rx1 * ry2 - ry1 * rx2;
    if (point_in_triangle(pint, p1, p2, p3, nxt, nyt, nzt) < 0) continue;
    bary_by_normal(pint, p1, p2, p3, nxt, nyt, nzt, cr);
    *d_i = sqrt((pint.x - p.x) * (pint.x - p.x) + (pint.y - p.y) * (pint.y - p.y) + (pint.z - p.z) * (pint.z - p.z));
    return t;
  }
  return -100;
}

__global__ void k_ibm_nodes(Grid g, IbmGeom G, IbNode *out, int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G.n) return;
  const IbmSurface &S = G.S;
  const long long pos = G.cells[q];
  const int i = (int)(pos % g.mx);
  const long long r = pos / g.mx;
  const int j = (int)(r % g.my), k = (int)(r / g.my);
  IbNode N;
  N.i = i; N.j = j; N.k = k;
  const P3 p = {G.cent.x[pos], G.cent.y[pos], G.cent.z[pos]};
  // nearestcell1 (ibm.c:1366-1512)
  double dmin = 1.e20;
  int cmin = -100;
  P3 pmin = {0, 0, 0};
  for (int e = 0; e < S.nelmt; e++) {
    const P3 qc = {G.qx[e], G.qy[e], G.qz[e]};
    if (!(dist3(p, qc) - G.rad[e] < dmin)) continue;
    const int a = S.n1[e], b = S.n2[e], c = S.n3[e];
    const double nfx = S.nx[e], nfy = S.ny[e], nfz = S.nz[e];
    const P3 p1 = vtx(S, a), p2 = vtx(S, b), p3 = vtx(S, c);
    double tf = ((p.x - S.x[a]) * nfx + (p.y - S.y[a]) * nfy + (p.z - S.z[a]) * nfz);
    if (fabs(tf) < 1.e-10) tf = 1.e-10;
    if (!(tf >= 0)) continue;
    const P3 pj = {p.x - tf * nfx, p.y - tf * nfy, p.z - tf * nfz};
    if (point_in_triangle(pj, p1, p2, p3, nfx, nfy, nfz) == 1) {
      if (tf < dmin) { dmin = tf; pmin = pj; cmin = e; }
    } else {
      P3 po;
      double d;
      dist_point_segment(p, p1, p2, &po, &d);
      if (d < dmin) { dmin = d; pmin = po; cmin = e; }
      dist_point_segment(p, p2, p3, &po, &d);
      if (d < dmin) { dmin = d; pmin = po; cmin = e; }
      dist_point_segment(p, p3, p1, &po, &d);
      if (d < dmin) { dmin = d; pmin = po; cmin = e; }
    }
  }
  if (cmin < 0) {  // "Nearest Cell Searching Error!": flagged; the node stays a harmless self-stencil
    atomicExch(err, 1);
    N.cell = 0; N.imode = -2; N.ds = N.di = 0;
    for (int v = 0; v < 3; v++) { N.st[3 * v] = i; N.st[3 * v + 1] = j; N.st[3 * v + 2] = k; N.cr[v] = N.cs[v] = 0; }
    node_triangle(G, N);
    out[q] = N;
    return;
  }
  N.cell = cmin;
  N.ds = dmin;
  N.cs[0] = N.cs[1] = N.cs[2] = 0;
  bary_by_normal(pmin, vtx(S, S.n1[cmin]), vtx(S, S.n2[cmin]), vtx(S, S.n3[cmin]), S.nx[cmin], S.ny[cmin],
                 S.nz[cmin], N.cs);
  // InterceptionPoint (ibm.c:1759-2250): the faces i-1, i+1, j-1, j+1, k-1, k+1 in turn
  double nfx = p.x - pmin.x, nfy = p.y - pmin.y, nfz = p.z - pmin.z;
  const double dr = sqrt(nfx * nfx + nfy * nfy + nfz * nfz);
  nfx /= dr; nfy /= dr; nfz /= dr;
  const int pick[8][3] = {{0, 1, 4}, {1, 2, 4}, {2, 4, 5}, {4, 5, 8}, {4, 7, 8}, {4, 6, 7}, {3, 4, 6}, {3, 4, 0}};
  N.imode = -100;
  for (int f = 0; f < 6 && N.imode < 0; f++) {
    int ip[9], jp[9], kp[9];
    for (int n = 0; n < 9; n++) {
      const int a = n % 3 - 1, b = n / 3 - 1;
      if (f < 2) { ip[n] = i + (f == 0 ? -1 : 1); jp[n] = j + a; kp[n] = k + b; }
      else if (f < 4) { ip[n] = i + a; jp[n] = j + (f == 2 ? -1 : 1); kp[n] = k + b; }
      else { ip[n] = i + a; jp[n] = j + b; kp[n] = k + (f == 4 ? -1 : 1); }
    }
    P3 pc[9];
    for (int n = 0; n < 9; n++) {
      const long long c = lidx(g, ip[n], jp[n], kp[n]);
      pc[n] = {G.cent.x[c], G.cent.y[c], G.cent.z[c]};
    }
    const int t = icp(p, pc, nfx, nfy, nfz, N.cr, &N.di);
    if (t >= 0) {
      N.imode = t;
      for (int v = 0; v < 3; v++) {
        N.st[3 * v] = ip[pick[t][v]]; N.st[3 * v + 1] = jp[pick[t][v]]; N.st[3 * v + 2] = kp[pick[t][v]];
      }
    }
  }
  if (N.imode < 0) {  // ibm.c:400-498
    int dj = 0, dk = 0;
    if (i == 1 || i == g.mx - 2 || j == 1 || j == g.my - 2) dk = S.nz[cmin] > 0 ? 1 : -1;
    else if (k == 1 || k == g.mz - 2) dj = 1;
    if (dj || dk) {
      const long long c = lidx(g, i, j + dj, k + dk);
      const P3 pt = {G.cent.x[c], G.cent.y[c], G.cent.z[c]};
      N.di = sqrt((p.x - pt.x) * (p.x - pt.x) + (p.y - pt.y) * (p.y - pt.y) + (p.z - pt.z) * (p.z - pt.z));
      N.cr[0] = 1.; N.cr[1] = 0.; N.cr[2] = 0.;
      for (int v = 0; v < 3; v++) { N.st[3 * v] = i; N.st[3 * v + 1] = j + dj; N.st[3 * v + 2] = k + dk; }
      N.imode = -1;
    } else {
      // "IBM Searching Fail!": the reference keeps undefined stencil data; this node
      // interpolates nothing (its velocity becomes the surface velocity)
      for (int v = 0; v < 3; v++) { N.st[3 * v] = i; N.st[3 * v + 1] = j; N.st[3 * v + 2] = k; }
      N.cr[0] = N.cr[1] = N.cr[2] = 0;
      N.di = 0;
      N.imode = -2;
    }
  }
  node_triangle(G, N);
  out[q] = N;
}

__global__ void k_ibm_collect(Grid g, const uint8_t *__restrict__ fl, long long *cells, int *count, int cap) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2 || fl[p] != 2) return;
  const int slot = atomicAdd(count, 1);
  if (slot < cap) cells[slot] = p;
}

// BoundingSphere (ibm.c:1276-1364): a sphere around each triangle that bounds the
// nearest-point search.
static void bounding_spheres(int n_elmt, const double *x, const double *y, const double *z, const int *n1,
                             const int *n2, const int *n3, std::vector<double> &qx, std::vector<double> &qy,
                             std::vector<double> &qz, std::vector<double> &rad) {
  struct H { double x, y, z; };
  auto dist = [](const H &a, const H &b) {
    return sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z));
  };
  qx.resize(n_elmt); qy.resize(n_elmt); qz.resize(n_elmt); rad.resize(n_elmt);
  const H p0 = {0, 0, 0};
  for (int e = 0; e < n_elmt; e++) {
    const H p1 = {x[n1[e]], y[n1[e]], z[n1[e]]}, p2 = {x[n2[e]], y[n2[e]], z[n2[e]]}, p3 = {x[n3[e]], y[n3[e]], z[n3[e]]};
    const double l12 = dist(p1, p2), l23 = dist(p2, p3), l31 = dist(p3, p1);
    H pa, pb, pc;
    if (l12 > l23) {
      if (l12 > l31) { pa = p1; pb = p2; pc = p3; }
      else { pa = p3; pb = p1; pc = p2; }
    } else {
      if (l31 < l23) { pa = p2; pb = p3; pc = p1; }
      else { pa = p3; pb = p1; pc = p2; }
    }
    const H pf = {0.5 * (pa.x + pb.x), 0.5 * (pa.y + pb.y), 0.5 * (pa.z + pb.z)};
    const H pu = {pa.x - pf.x, pa.y - pf.y, pa.z - pf.z}, pv = {pc.x - pf.x, pc.y - pf.y, pc.z - pf.z};
    const H pt = {pu.y * pv.z - pu.z * pv.y, pu.z * pv.x - pu.x * pv.z, pu.x * pv.y - pu.y * pv.x};
    const H pd = {pt.y * pu.z - pt.z * pu.y, pt.z * pu.x - pt.x * pu.z, pt.x * pu.y - pt.y * pu.x};
    double gama = -(dist(pu, p0) * dist(pu, p0) - dist(pv, p0) * dist(pv, p0));
    const H pw = {pv.x - pu.x, pv.y - pu.y, pv.z - pu.z};
    double lamda = 2 * (pd.x * pw.x + pd.y * pw.y + pd.z * pw.z);
    gama /= lamda;
    lamda = (gama < 0) ? 0 : gama;
    const H q = {pf.x + lamda * pd.x, pf.y + lamda * pd.y, pf.z + lamda * pd.z};
    qx[e] = q.x; qy[e] = q.y; qz[e] = q.z;
    rad[e] = dist(q, pa);
  }
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
                       sizeof(int) * (3 * (size_t)n_elmt + col_start.size() + 2 * nt) + 2 * sizeof(int) + 256;
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
  S.nelmt = n_elmt;
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
  int *err = (int *)(buf + off);  // err[0]: search status, err[1]: node count
  cudaMemsetAsync(err, 0, 2 * sizeof(int), c->stream);
  S.xmin = xmin; S.xmax = xmax; S.ymin = ymin; S.ymax = ymax; S.zmin = zmin; S.zmax = zmax;
  S.dcx = dcx; S.dcy = dcy; S.dcz = dcz;
  int rc;
  c->launches++, k_ibm_cast<<<nblocks(g.N, 128), 128, 0, c->stream>>>(g, S, cv(field3(c, VFS_CENT)), c->nv, ibi == 0 ? 1 : 0, err);
  if ((rc = check_launch(c, "k_ibm_cast"))) { cudaFree(buf); return rc; }
  c->launches++, k_ibm_near<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nv, c->bcflag);
  if ((rc = check_launch(c, "k_ibm_near"))) { cudaFree(buf); return rc; }
  if (c->nvo && ibi == (int)c->scal[VFS_S_NBODIES] - 1) {
    c->launches++, k_ibm_phase<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->nvo, c->bcflag);
    if ((rc = check_launch(c, "k_ibm_phase"))) { cudaFree(buf); return rc; }
  }
  // the IB-node list of this body (ibm.c:347-505): cells marked 2, ascending
  {
    int *cnt = err + 1;
    cudaMemsetAsync(cnt, 0, sizeof(int), c->stream);
    const int cap = 1 << 22;
    long long *cells = nullptr;
    if (cudaMallocAsync((void **)&cells, sizeof(long long) * cap, c->stream) != cudaSuccess) {
      cudaFree(buf);
      return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: allocation failed");
    }
    c->launches++, k_ibm_collect<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->bcflag, cells, cnt, cap);
    int hn = 0;
    cudaMemcpyAsync(&hn, cnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    if (hn > cap) { cudaFreeAsync(cells, c->stream); cudaFree(buf); return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: too many IB nodes"); }
    std::vector<long long> hc(hn);
    if (hn) cudaMemcpy(hc.data(), cells, sizeof(long long) * hn, cudaMemcpyDeviceToHost);
    std::sort(hc.begin(), hc.end());
    if (hn) cudaMemcpy(cells, hc.data(), sizeof(long long) * hn, cudaMemcpyHostToDevice);
    std::vector<double> qx, qy, qz, rad;
    bounding_spheres(n_elmt, x, y, z, n1, n2, n3, qx, qy, qz, rad);
    double *qd = nullptr;
    IbNode *nodes = nullptr;
    const int base = (ibi == 0) ? 0 : c->nib;
    bool ok = cudaMalloc(&qd, sizeof(double) * 4 * (size_t)n_elmt) == cudaSuccess;
    ok = ok && cudaMalloc(&nodes, sizeof(IbNode) * (size_t)(base + hn + 1)) == cudaSuccess;
    if (!ok) { cudaFree(qd); cudaFree(nodes); cudaFreeAsync(cells, c->stream); cudaFree(buf); return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: allocation failed"); }
    cudaMemcpyAsync(qd, qx.data(), sizeof(double) * n_elmt, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(qd + n_elmt, qy.data(), sizeof(double) * n_elmt, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(qd + 2 * (size_t)n_elmt, qz.data(), sizeof(double) * n_elmt, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(qd + 3 * (size_t)n_elmt, rad.data(), sizeof(double) * n_elmt, cudaMemcpyHostToDevice, c->stream);
    if (base) cudaMemcpyAsync(nodes, c->ibn, sizeof(IbNode) * base, cudaMemcpyDeviceToDevice, c->stream);
    IbmGeom G;
    G.S = S;
    G.qx = qd; G.qy = qd + n_elmt; G.qz = qd + 2 * (size_t)n_elmt; G.rad = qd + 3 * (size_t)n_elmt;
    G.cent = cv(field3(c, VFS_CENT));
    G.cells = cells;
    G.n = hn;
    // this body's vertices in the surface-velocity array (zero: a fixed body)
    if ((int)c->vtx_base.size() <= ibi) c->vtx_base.resize(ibi + 1, -1);
    if (ibi == 0) c->nvtx = 0;
    for (size_t b = ibi + 1; b < c->vtx_base.size(); b++) c->vtx_base[b] = -1;
    c->vtx_base[ibi] = c->nvtx;
    G.vbase = c->nvtx;
    {
      double *nvb = nullptr;
      const int ntot = c->nvtx + n_v;
      if (cudaMalloc(&nvb, sizeof(double) * 3 * (size_t)ntot) != cudaSuccess) {
        cudaFree(qd); cudaFree(nodes); cudaFreeAsync(cells, c->stream); cudaFree(buf);
        return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: allocation failed");
      }
      cudaMemsetAsync(nvb, 0, sizeof(double) * 3 * (size_t)ntot, c->stream);
      if (c->ibv && c->nvtx)
        for (int d = 0; d < 3; d++)
          cudaMemcpyAsync(nvb + (size_t)d * ntot, c->ibv + (size_t)d * c->nvtx, sizeof(double) * c->nvtx,
                          cudaMemcpyDeviceToDevice, c->stream);
      cudaStreamSynchronize(c->stream);
      if (c->ibv) cudaFree(c->ibv);
      c->ibv = nvb;
      c->nvtx = ntot;
    }
    if (hn) c->launches++, k_ibm_nodes<<<nblocks(hn, 64), 64, 0, c->stream>>>(g, G, nodes + base, err);
    if ((rc = check_launch(c, "k_ibm_nodes"))) { cudaFree(qd); cudaFree(nodes); cudaFree(buf); return rc; }
    cudaFreeAsync(cells, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(qd);
    if (c->ibn) cudaFree(c->ibn);
    if (c->ibbuf) cudaFree(c->ibbuf);
    c->ibn = nodes;
    c->nib = base + hn;
    if (ibi == 0) c->nib_body0 = hn;
    c->ibbuf = nullptr;
    if (c->nib && cudaMalloc(&c->ibbuf, sizeof(double) * kIbOut * (size_t)c->nib) != cudaSuccess) {
      cudaFree(buf);
      return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: allocation failed");
    }
    std::vector<IbNode> hnodes(hn);
    if (hn) cudaMemcpy(hnodes.data(), nodes + base, sizeof(IbNode) * hn, cudaMemcpyDeviceToHost);
    if (ibi == 0) c->nib_unresolved = 0;
    for (const IbNode &nd : hnodes) c->nib_unresolved += nd.imode == -2;
  }
  c->launches++, k_ibm_remap<<<nblocks(g.N, 256), 256, 0, c->stream>>>(g, c->bcflag, c->nv, c->f[VFS_NVERT][0]);
  if ((rc = check_launch(c, "k_ibm_remap"))) { cudaFree(buf); return rc; }
  cudaMemsetAsync(c->bcflag, 0, (size_t)g.N, c->stream);  // Contra2Cart's flag buffer, clear again
  int herr = 0;
  cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    cudaFree(buf);
    return set_err(c, VFS_ERR_CUDA, "vfs_ibm_search: kernel failed");
  }
  cudaFree(buf);
  if (herr == 1) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: no nearest surface point for an IB node");
  if (herr == -1) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: a cell's rays kept hitting coincident crossings");
  if (herr == -2) return set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: a ray crossed too many triangles");
  c->nvert_set = true;
  c->nsolid = -1;
  c->ps.built = false;
  c->setup_epoch++;
  return VFS_OK;
}

// ------------------------------------------------------------------ per-step IB work
// ibm_interpolation_advanced (ibm.c:3294-3700) for fixed bodies with the no-slip
// reconstruction (noslip, wallfunction.c:134-150): each IB node takes
// Ub = (sb/sc)(Uc - Ua) + Ua from the velocity Uc interpolated at its three stencil cells
// (sc = sb + d_i), zero when a stencil cell is not fluid or the node is solid, and the
// pressure interpolated the same way.  All nodes read the fields as they were before the
// pass (the reference reads the local copies lUcat and lP), then write.
// The wall model of the reconstruction, wall_function_roughness_a (sediment_transport-Y.c:
// 68-91) with its helpers E_coeff, u_hydset_roughness, f_hydset, df_hydset and
// find_utau_hydset (sediment_transport-Y.c:16-66): a log law with a roughness shift for
// the tangential velocity, solved for the friction velocity by Newton's method with a
// central-difference derivative, in the reference's operation order.
__device__ __forceinline__ double wf_e_coeff(double utau, double ks, double nu) {
  const double kplus = utau * ks / nu;
  const double kappa = 0.41, B = 5.5;
  double dB = 0.0;
  if (kplus <= 2.25) dB = 0.0;
  else if (kplus > 2.25 && kplus < 90.) dB = (B - 8.5 + 1. / kappa * log(kplus)) * sin(0.4258 * (log(kplus) - 0.811));
  else if (kplus >= 90.) dB = B - 8.5 + 1. / kappa * log(kplus);
  return exp(kappa * (B - dB));
}
__device__ __forceinline__ double wf_u_hydset(double nu, double y, double utau, double ks) {
  const double y0plus = 11.53, kappa = 0.41;
  const double yplus = utau * y / nu;
  if (yplus <= y0plus) return utau * yplus;
  return utau / kappa * log(wf_e_coeff(utau, ks, nu) * yplus);
}
__device__ __forceinline__ double wf_f_hydset(double nu, double u, double y, double utau0, double ks) {
  const double y0plus = 11.53, kappa = 0.41;
  const double yplus = utau0 * y / nu;
  if (yplus <= y0plus) return utau0 * yplus - u;
  return utau0 * (1. / kappa * log(wf_e_coeff(utau0, ks, nu) * yplus)) - u;
}
// The rough-wall log law of wall_function_roughness_loglaw (wallfunction.c:71-98,
// 221-250, 423-437): u = utau (ln(y/ks)/kappa + 8.5), solved for utau by Newton's method
// with a central-difference derivative (step 1e-7), at most 30 steps, stopping when a step
// moves utau by less than 1e-10.
__device__ __forceinline__ double wf_u_loglaw(double y, double utau, double ks) {
  const double kappa = 0.41;
  return utau * (1. / kappa * log(y / ks) + 8.5);
}
__device__ __forceinline__ double wf_find_utau_loglaw(double u, double y, double guess, double ks) {
  double x = guess, x0 = guess;
  const double eps = 1.e-7;
  for (int i = 0; i < 30; i++) {
    const double df = ((wf_u_loglaw(y, x0 + eps, ks) - u) - (wf_u_loglaw(y, x0 - eps, ks) - u)) / (2 * eps);
    x = x0 - (wf_u_loglaw(y, x0, ks) - u) / df;
    if (fabs(x0 - x) < 1.e-10) break;
    x0 = x;
  }
  return x;
}
__device__ __forceinline__ double wf_find_utau(double nu, double u, double y, double guess, double ks) {
  double utau = guess, utau0 = guess;
  const double eps = 1.e-7;
  for (int ii = 0; ii < 30; ii++) {
    const double df = (wf_f_hydset(nu, u, y, utau0 + eps, ks) - wf_f_hydset(nu, u, y, utau0 - eps, ks)) / (2. * eps);
    utau = utau0 - wf_f_hydset(nu, u, y, utau0, ks) / df;
    if (fabs(utau - utau0) < 1.e-7) break;
    utau0 = utau;
  }
  return utau;
}

// One IB node of ibm_interpolation_advanced (ibm.c:3405-3530): the surface velocity Ua
// from the triangle's vertex velocities (zero for a fixed body), Uc interpolated at the
// node's three stencil cells; the node's velocity is 0 next to a solid stencil cell
// (fixed bodies) or inside a body, the wall model's (wallfunction, from ti > 0), or
// Ub = (sb/sc)(Uc - Ua) + Ua (noslip, wallfunction.c:134-150); the friction velocity of
// either goes to ustar.  All nodes read the fields as they were before the pass (the
// reference reads the local copies lUcat and lP), then write.
__global__ void k_ibm_gather(Grid g, const IbNode *__restrict__ nodes, int n, CV3 ucat, const double *__restrict__ p,
                             const uint8_t *__restrict__ nv, const double *__restrict__ ibv, int nvtx, int ti,
                             int nbody0, double *out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const IbNode N = nodes[q];
  const long long s1 = lidx(g, N.st[0], N.st[1], N.st[2]), s2 = lidx(g, N.st[3], N.st[4], N.st[5]);
  const long long s3 = lidx(g, N.st[6], N.st[7], N.st[8]);
  const double sb = N.ds, sc = sb + N.di;
  const double sk1 = N.cr[0], sk2 = N.cr[1], sk3 = N.cr[2];
  const double cs1 = N.cs[0], cs2 = N.cs[1], cs3 = N.cs[2];
  double uax = 0, uay = 0, uaz = 0;
  if (N.cell >= 0) {
    const int a = N.vtx[0], b = N.vtx[1], c = N.vtx[2];
    uax = ibv[a] * cs1 + ibv[b] * cs2 + ibv[c] * cs3;
    uay = ibv[nvtx + a] * cs1 + ibv[nvtx + b] * cs2 + ibv[nvtx + c] * cs3;
    uaz = ibv[2 * nvtx + a] * cs1 + ibv[2 * nvtx + b] * cs2 + ibv[2 * nvtx + c] * cs3;
  }
  const double ucx = (ucat.x[s1] * sk1 + ucat.x[s2] * sk2 + ucat.x[s3] * sk3);
  const double ucy = (ucat.y[s1] * sk1 + ucat.y[s2] * sk2 + ucat.y[s3] * sk3);
  const double ucz = (ucat.z[s1] * sk1 + ucat.z[s2] * sk2 + ucat.z[s3] * sk3);
  const long long pos = lidx(g, N.i, N.j, N.k);
  double ub[3], ustar;
  if ((!g.moving && (double)nv[s1] + (double)nv[s2] + (double)nv[s3] > 0.1) || nv[pos] > 2) {
    ub[0] = ub[1] = ub[2] = 0;
    ustar = 0;
  } else if (g.wallfunction && ti > 0 && g.roughness > 0 && q < nbody0) {
    // rough_set && ibi == 0: the rough-wall log law, tangential velocity only (ibm.c:3468-3470)
    const double nx = N.nf[0], ny = N.nf[1], nz = N.nf[2];
    const double u_c = ucx - uax, v_c = ucy - uay, w_c = ucz - uaz;
    const double un = u_c * nx + v_c * ny + w_c * nz;
    double ut = u_c - un * nx, vt = v_c - un * ny, wt = w_c - un * nz;
    const double ut_mag = sqrt(ut * ut + vt * vt + wt * wt);
    ustar = wf_find_utau_loglaw(ut_mag, sc, 0.01, g.roughness);
    const double ut_mag_modeled = wf_u_loglaw(sb, ustar, g.roughness);
    if (ut_mag > 1.e-10) {
      ut *= ut_mag_modeled / ut_mag;
      vt *= ut_mag_modeled / ut_mag;
      wt *= ut_mag_modeled / ut_mag;
    } else {
      ut = vt = wt = 0;
    }
    ub[0] = ut; ub[1] = vt; ub[2] = wt;
    ub[0] += uax; ub[1] += uay; ub[2] += uaz;
  } else if (g.wallfunction && ti > 0) {
    const double nx = N.nf[0], ny = N.nf[1], nz = N.nf[2];
    const double u_c = ucx - uax, v_c = ucy - uay, w_c = ucz - uaz;
    const double un = u_c * nx + v_c * ny + w_c * nz;
    double ut = u_c - un * nx, vt = v_c - un * ny, wt = w_c - un * nz;
    const double ut_mag = sqrt(ut * ut + vt * vt + wt * wt);
    ustar = wf_find_utau(1. / g.ren, ut_mag, sc, 0.01, 0.0001);
    const double ut_mag_modeled = wf_u_hydset(1. / g.ren, sb, ustar, 0.0001);
    if (ut_mag > 1.e-10) {
      ut *= ut_mag_modeled / ut_mag;
      vt *= ut_mag_modeled / ut_mag;
      wt *= ut_mag_modeled / ut_mag;
    } else {
      ut = vt = wt = 0;
    }
    ub[0] = ut + sb / sc * un * nx;
    ub[1] = vt + sb / sc * un * ny;
    ub[2] = wt + sb / sc * un * nz;
    ub[0] += uax; ub[1] += uay; ub[2] += uaz;
  } else {
    const double nx = N.nf[0], ny = N.nf[1], nz = N.nf[2];
    const double u_c = ucx - uax, v_c = ucy - uay, w_c = ucz - uaz;
    const double un = u_c * nx + v_c * ny + w_c * nz;
    const double ut = u_c - un * nx, vt = v_c - un * ny, wt = w_c - un * nz;
    const double ut_mag = sqrt(ut * ut + vt * vt + wt * wt);
    ustar = sqrt(ut_mag / sc / g.ren);
    ub[0] = sb / sc * u_c; ub[1] = sb / sc * v_c; ub[2] = sb / sc * w_c;
    ub[0] += uax; ub[1] += uay; ub[2] += uaz;
  }
  const double pn = (p[s1] * sk1 + p[s2] * sk2 + p[s3] * sk3);
  double *o = out + (size_t)kIbOut * q;
  o[0] = ub[0]; o[1] = ub[1]; o[2] = ub[2]; o[3] = pn; o[4] = ustar;
}

__global__ void k_ibm_scatter(Grid g, const IbNode *__restrict__ nodes, int n, const double *__restrict__ in, V3 ucat,
                              double *p, double *ustar) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const IbNode N = nodes[q];
  const long long pos = lidx(g, N.i, N.j, N.k);
  const double *v = in + (size_t)kIbOut * q;
  ucat.x[pos] = v[0]; ucat.y[pos] = v[1]; ucat.z[pos] = v[2];
  p[pos] = v[3];
  ustar[pos] = v[4];
}

// Face fluxes next to IB nodes from the averaged Cartesian velocity (ibm.c:3605-3650 and
// the immersed branch of IB_BC, momentum.c:2077-2108): every face of an IB-node cell, and
// the lower faces of cells whose upper neighbour is an IB node.
__global__ void k_ib_faces(Grid g, Metrics m, CV3 u, const uint8_t *__restrict__ nv, V3 uc) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.N) return;
  int i, j, k;
  dijk(g, p, i, j, k);
  if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) return;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  const bool self = nv[p] == 1;
  if (self || nv[p + 1] == 1) {
    const double ucx = (u.x[p] + u.x[p + 1]) * 0.5, ucy = (u.y[p] + u.y[p + 1]) * 0.5, ucz = (u.z[p] + u.z[p + 1]) * 0.5;
    uc.x[p] = (ucx * m.icsi.x[p] + ucy * m.icsi.y[p] + ucz * m.icsi.z[p]) * 1.0;
  }
  if (self || nv[p + sy] == 1) {
    const double ucx = (u.x[p + sy] + u.x[p]) * 0.5, ucy = (u.y[p + sy] + u.y[p]) * 0.5, ucz = (u.z[p + sy] + u.z[p]) * 0.5;
    uc.y[p] = (ucx * m.jeta.x[p] + ucy * m.jeta.y[p] + ucz * m.jeta.z[p]) * 1.0;
  }
  if (self || nv[p + sz] == 1) {
    const double ucx = (u.x[p + sz] + u.x[p]) * 0.5, ucy = (u.y[p + sz] + u.y[p]) * 0.5, ucz = (u.z[p + sz] + u.z[p]) * 0.5;
    uc.z[p] = (ucx * m.kzet.x[p] + ucy * m.kzet.y[p] + ucz * m.kzet.z[p]) * 1.0;
  }
}

int ib_faces(Ctx *c) {
  c->launches++, k_ib_faces<<<nblocks(c->g.N, 256), 256, 0, c->stream>>>(c->g, metrics(c), cv(field3(c, VFS_UCAT)), c->nv,
                                                         field3(c, VFS_UCONT));
  return check_launch(c, "k_ib_faces");
}

int ibm_interpolation(Ctx *c) {
  int rc;
  if (c->nib > 0) {
    const Grid &g = c->g;
    c->launches++, k_ibm_gather<<<nblocks(c->nib, 128), 128, 0, c->stream>>>(g, c->ibn, c->nib, cv(field3(c, VFS_UCAT)),
                                                             c->f[VFS_P][0], c->nv, c->ibv, c->nvtx, c->ti,
                                                             c->nib_body0, c->ibbuf);
    if ((rc = check_launch(c, "k_ibm_gather"))) return rc;
    c->launches++, k_ibm_scatter<<<nblocks(c->nib, 128), 128, 0, c->stream>>>(g, c->ibn, c->nib, c->ibbuf, field3(c, VFS_UCAT),
                                                              c->f[VFS_P][0], c->f[VFS_USTAR][0]);
    if ((rc = check_launch(c, "k_ibm_scatter"))) return rc;
  }
  if ((rc = ib_faces(c))) return rc;
  return contra2cart(c);
}

// VolumeFlux(user, &ibm_Flux, &ibm_Area, 0) (poisson.c:3570-3730): the net flux through the
// faces between fluid cells and IB nodes, faces carrying |Ucont| <= 1e-8 zeroed, is spread
// over those faces in proportion to their area (the centre-metric norm the reference uses).
__device__ __forceinline__ double face_area(CV3 m, long long p) {
  return sqrt(m.x[p] * m.x[p] + m.y[p] * m.y[p] + m.z[p] * m.z[p]);
}

template <int PASS>
__global__ void k_vflux_ibm(Grid g, Metrics m, const uint8_t *__restrict__ nv, V3 uc, const double *__restrict__ ds,
                            double *parts) {
  // pass 1: the net flux of pass 0 spread over the IB faces in proportion to their area
  double correction = 0;
  if (PASS == 1) {
    const double f = ds[DS_VF_FLUX], a = ds[DS_VF_AREA];
    correction = (a > 1.e-15) ? f / a : 0;
  }
  __shared__ double s1[256], s2[256];
  double fsum = 0, asum = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long sy = g.mx, sz = (long long)g.mx * g.my;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N; p += stride) {
    int i, j, k;
    dijk(g, p, i, j, k);
    if (i < 1 || i > g.mx - 2 || j < 1 || j > g.my - 2 || k < 1 || k > g.mz - 2) continue;
    const int v0 = nv[p];
    double *comp[3] = {uc.x, uc.y, uc.z};
    const CV3 *met[3] = {&m.csi, &m.eta, &m.zet};  // centre metrics (lCsi, lEta, lZet)
    const long long off[3] = {1, sy, sz};
    const bool inner[3] = {i < g.mx - 2, j < g.my - 2, k < g.mz - 2};
    for (int d = 0; d < 3; d++) {
      const int vn = nv[p + off[d]];
      double sign = 0;
      if (v0 == 0 && vn == 1 && inner[d]) sign = 1;       // fluid cell, IB node above
      if (v0 == 1 && vn == 0 && inner[d]) sign = -1;      // IB node, fluid cell above
      if (sign == 0) continue;
      double &f = comp[d][p];
      if (PASS == 0) {
        if (fabs(f) > 1.e-8) {
          fsum = sign > 0 ? fsum + f : fsum - f;
          asum += face_area(*met[d], p);
        } else {
          f = 0.;
        }
      } else if (fabs(f) > 1.e-8) {
        f = sign > 0 ? f - face_area(*met[d], p) * correction : f + face_area(*met[d], p) * correction;
      }
    }
  }
  if (PASS == 1) return;
  s1[threadIdx.x] = fsum; s2[threadIdx.x] = asum;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { parts[blockIdx.x] = s1[0]; parts[gridDim.x + blockIdx.x] = s2[0]; }
}

int volume_flux_ibm(Ctx *c, double *flux, double *area) {
  int rc;
  const int nb = 148 * 2;
  if ((rc = ensure_red(c, 2 * nb + 64))) return rc;
  Metrics m = metrics(c);
  c->launches++, k_vflux_ibm<0><<<nb, 256, 0, c->stream>>>(c->g, m, c->nv, field3(c, VFS_UCONT), c->ds, c->red);
  if ((rc = check_launch(c, "k_vflux_ibm"))) return rc;
  if ((rc = reduce_to(c, c->red, nb, c->ds + DS_VF_FLUX))) return rc;
  if ((rc = reduce_to(c, c->red + nb, nb, c->ds + DS_VF_AREA))) return rc;
  c->launches++, k_vflux_ibm<1><<<nb, 256, 0, c->stream>>>(c->g, m, c->nv, field3(c, VFS_UCONT), c->ds, c->red);
  if ((rc = check_launch(c, "k_vflux_ibm"))) return rc;
  if ((flux || area) && !c->capturing) {
    if ((rc = ds_fetch(c))) return rc;
    if (flux) *flux = c->ds_out[DS_VF_FLUX];
    if (area) *area = c->ds_out[DS_VF_AREA];
  }
  return VFS_OK;
}

}  // namespace vfs

extern "C" int vfs_ibm_set_velocity(vfs_ctx *ctx, int ibi, int n_v, const double *u, const double *v,
                                    const double *w) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !u || !v || !w || ibi < 0 || n_v < 1) return vfs::set_err(c, VFS_ERR_INVALID, "vfs_ibm_set_velocity: bad argument");
  if (ibi >= (int)c->vtx_base.size() || c->vtx_base[ibi] < 0 || !c->ibv)
    return vfs::set_err(c, VFS_ERR_STATE, "vfs_ibm_set_velocity: body not searched (vfs_ibm_search first)");
  const int next = ibi + 1 < (int)c->vtx_base.size() && c->vtx_base[ibi + 1] >= 0 ? c->vtx_base[ibi + 1] : c->nvtx;
  if (n_v != next - c->vtx_base[ibi])
    return vfs::set_err(c, VFS_ERR_INVALID, "vfs_ibm_set_velocity: vertex count differs from the body's");
  cudaSetDevice(c->device);
  const double *src[3] = {u, v, w};
  for (int d = 0; d < 3; d++)
    cudaMemcpyAsync(c->ibv + (size_t)d * c->nvtx + c->vtx_base[ibi], src[d], sizeof(double) * n_v,
                    cudaMemcpyHostToDevice, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return vfs::set_err(c, VFS_ERR_CUDA, "vfs_ibm_set_velocity: copy failed");
  return VFS_OK;
}

extern "C" int vfs_ibm_search(vfs_ctx *ctx, int ibi, int n_v, const double *x, const double *y, const double *z,
                              int n_elmt, const int *nv1, const int *nv2, const int *nv3) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !x || !y || !z || !nv1 || !nv2 || !nv3 || ibi < 0)
    return vfs::set_err(c, VFS_ERR_INVALID, "vfs_ibm_search: bad argument");
  if (!c->metrics_set) return vfs::set_err(c, VFS_ERR_STATE, "vfs_ibm_search: metrics (cell centres) not set");
  cudaSetDevice(c->device);
  return vfs::ibm_search(c, ibi, n_v, x, y, z, n_elmt, nv1, nv2, nv3);
}
