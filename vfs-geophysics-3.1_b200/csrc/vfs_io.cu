// Restart files in the reference's format (host code).
//
// The reference writes its flow state with PETSc's binary viewer, one file per vector
// and time step (Ucont_P_Binary_Output, main.c:765-1035) and reads it back at a restart
// (Ucont_P_Binary_Input, main.c:394-760):  <dir>/vfield%06d_%1d.dat (Ucont),
// ufield (Ucat), pfield (P), nvfield (Nvert), and cs_%06d_%1d.dat (the Smagorinsky
// coefficient) when les is on, with the time step and the block number in the names.
// A PETSc 3.1 binary Vec file is the Vec class id 1211214 and the global length as
// 32-bit big-endian integers followed by the entries as big-endian doubles; a DA vector
// is written in the natural ordering, (k, j, i) with i fastest and the components of a
// point together, which is the layout vfs_get_field and vfs_set_field use.  So a GPU run
// can resume from the reference's files and the reference from the library's.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vfs_internal.cuh"

namespace {

constexpr int kVecClassId = 1211214;

void put_be32(unsigned char *b, unsigned v) {
  b[0] = (unsigned char)(v >> 24); b[1] = (unsigned char)(v >> 16);
  b[2] = (unsigned char)(v >> 8); b[3] = (unsigned char)v;
}
unsigned get_be32(const unsigned char *b) {
  return (unsigned)b[0] << 24 | (unsigned)b[1] << 16 | (unsigned)b[2] << 8 | (unsigned)b[3];
}

std::string restart_name(const char *dir, const char *stem, int ti, int block) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%s%06d_%1d.dat", stem, ti, block);
  return std::string(dir) + "/" + buf;
}

}  // namespace

extern "C" int vfs_petsc_vec_write(const char *path, const double *values, long long n) {
  if (!path || (!values && n > 0) || n < 0 || n > 0x7fffffffLL)
    return vfs::set_err(nullptr, VFS_ERR_INVALID, "vfs_petsc_vec_write: bad argument");
  FILE *f = fopen(path, "wb");
  if (!f) return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_write: cannot open ") + path);
  unsigned char head[8];
  put_be32(head, kVecClassId);
  put_be32(head + 4, (unsigned)n);
  bool ok = fwrite(head, 1, 8, f) == 8;
  std::vector<unsigned char> buf(8 * 4096);
  for (long long q0 = 0; ok && q0 < n; q0 += 4096) {
    const long long m = std::min<long long>(4096, n - q0);
    for (long long q = 0; q < m; q++) {
      unsigned long long u;
      memcpy(&u, values + q0 + q, 8);
      for (int t = 0; t < 8; t++) buf[8 * q + t] = (unsigned char)(u >> (56 - 8 * t));
    }
    ok = fwrite(buf.data(), 1, 8 * m, f) == (size_t)(8 * m);
  }
  ok = (fclose(f) == 0) && ok;
  return ok ? VFS_OK : vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_write: write failed: ") + path);
}

extern "C" int vfs_petsc_vec_read(const char *path, double *values, long long n) {
  if (!path || (!values && n > 0) || n < 0)
    return vfs::set_err(nullptr, VFS_ERR_INVALID, "vfs_petsc_vec_read: bad argument");
  FILE *f = fopen(path, "rb");
  if (!f) return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_read: cannot open ") + path);
  unsigned char head[8];
  if (fread(head, 1, 8, f) != 8 || get_be32(head) != (unsigned)kVecClassId) {
    fclose(f);
    return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_read: not a PETSc Vec file: ") + path);
  }
  if ((long long)get_be32(head + 4) != n) {
    fclose(f);
    return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_read: length differs from the grid's: ") + path);
  }
  std::vector<unsigned char> buf(8 * 4096);
  bool ok = true;
  for (long long q0 = 0; ok && q0 < n; q0 += 4096) {
    const long long m = std::min<long long>(4096, n - q0);
    ok = fread(buf.data(), 1, 8 * m, f) == (size_t)(8 * m);
    for (long long q = 0; ok && q < m; q++) {
      unsigned long long u = 0;
      for (int t = 0; t < 8; t++) u = (u << 8) | buf[8 * q + t];
      memcpy(values + q0 + q, &u, 8);
    }
  }
  fclose(f);
  return ok ? VFS_OK : vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_petsc_vec_read: short file: ") + path);
}

extern "C" int vfs_restart_write(vfs_ctx *ctx, const char *dir, int ti, int block) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !dir || ti < 0 || block < 0 || block > 9)
    return vfs::set_err(c, VFS_ERR_INVALID, "vfs_restart_write: bad argument");
  const long long n = c->g.N;
  std::vector<double> h(3 * (size_t)n);
  struct Item { const char *stem; int field; int dof; };
  const Item items[] = {{"vfield", VFS_UCONT, 3}, {"ufield", VFS_UCAT, 3}, {"pfield", VFS_P, 1},
                        {"nvfield", VFS_NVERT, 1}, {"cs_", VFS_CS, 1}};
  for (const Item &it : items) {
    if (it.field == VFS_CS && !c->g.les) continue;
    int rc = vfs_get_field(ctx, it.field, h.data());
    if (rc) return rc;
    if ((rc = vfs_petsc_vec_write(restart_name(dir, it.stem, ti, block).c_str(), h.data(), n * it.dof))) {
      vfs::set_err(c, rc, vfs_last_error(nullptr));
      return rc;
    }
  }
  return VFS_OK;
}

extern "C" int vfs_restart_read(vfs_ctx *ctx, const char *dir, int ti, int block) {
  vfs::Ctx *c = (vfs::Ctx *)ctx;
  if (!c || !dir || ti < 0 || block < 0 || block > 9)
    return vfs::set_err(c, VFS_ERR_INVALID, "vfs_restart_read: bad argument");
  const long long n = c->g.N;
  std::vector<double> h(3 * (size_t)n);
  auto load = [&](const char *stem, int dof) {
    const int rc = vfs_petsc_vec_read(restart_name(dir, stem, ti, block).c_str(), h.data(), n * dof);
    if (rc) vfs::set_err(c, rc, vfs_last_error(nullptr));
    return rc;
  };
  int rc;
  // Ucont, and Ucont_o = Ucont (main.c:401-405, 429-431)
  if ((rc = load("vfield", 3)) || (rc = vfs_set_field(ctx, VFS_UCONT, h.data())) ||
      (rc = vfs_set_field(ctx, VFS_UCONT_O, h.data())))
    return rc;
  if ((rc = load("pfield", 1)) || (rc = vfs_set_field(ctx, VFS_P, h.data()))) return rc;  // main.c:409-412
  // Nvert_o (main.c:414-417); with immersed bodies the flags of the file stand until the
  // caller classifies the bodies again, as the reference's IB search does after a restart
  if (c->g.immersed && ((rc = load("nvfield", 1)) || (rc = vfs_set_field(ctx, VFS_NVERT, h.data())))) return rc;
  // Ucat and lUcat_old = Ucat (main.c:419-422, 433-437)
  if ((rc = load("ufield", 3)) || (rc = vfs_set_field(ctx, VFS_UCAT, h.data())) ||
      (rc = vfs_set_field(ctx, VFS_UCAT_O, h.data())))
    return rc;
  if (c->g.les) {  // main.c:654-676: Cs from its file, 0 when there is none
    FILE *f = fopen(restart_name(dir, "cs_", ti, block).c_str(), "rb");
    if (f) {
      fclose(f);
      if ((rc = load("cs_", 1))) return rc;
    } else {
      std::fill(h.begin(), h.begin() + n, 0.0);
    }
    if ((rc = vfs_set_field(ctx, VFS_CS, h.data()))) return rc;
  }
  // the run continues at time step ti as a restarted run: tistart = ti with the restart
  // flag set (the first step repeats the set-up of ti == tistart, and the Smagorinsky
  // coefficient is computed from the first step on, les.c:69)
  c->ti = ti;
  c->tistart = ti;
  c->rstart = 1;
  c->first_step = true;
  return VFS_OK;
}

// ------------------------------------------------------------------ grid.dat
// The grid reader of MG_Initial (init.c:313-440): grid.dat in ASCII ("nblocks", then per
// block "IM JM KM" and the IM*JM*KM node x coordinates, then y, then z, [k][j][i] with i
// fastest, each scanned with %le), the same in binary (-binary 1: int nblocks, ints IM, JM,
// KM, native doubles), or xyz.dat (-xyz 1: one block, "IM JM KM", then IM lines whose first
// value is x(i), JM lines whose second is y(j), KM lines whose third is z(k): a tensor
// grid).  Each value v is stored as v / cl * L_dim, as the reference stores it.
namespace {

bool skip_doubles(FILE *f, int format, long long n) {
  double v;
  for (long long q = 0; q < n; q++) {
    if (format == 1 ? fread(&v, sizeof(double), 1, f) != 1 : fscanf(f, "%le", &v) != 1) return false;
  }
  return true;
}

}  // namespace

extern "C" int vfs_grid_read(const char *path, int format, int block, double cl, double L_dim, int *IM, int *JM,
                             int *KM, double *x, double *y, double *z) {
  if (!path || !IM || !JM || !KM || format < 0 || format > 2 || block < 0 || cl == 0.0)
    return vfs::set_err(nullptr, VFS_ERR_INVALID, "vfs_grid_read: bad argument");
  FILE *f = fopen(path, format == 1 ? "rb" : "r");
  if (!f) return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_grid_read: cannot open ") + path);
  auto fail = [&](const char *why) {
    fclose(f);
    return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_grid_read: ") + why + " in " + path);
  };
  int nblocks = 1;
  if (format == 1 && fread(&nblocks, sizeof(int), 1, f) != 1) return fail("no block count");
  if (format == 0 && fscanf(f, "%i\n", &nblocks) != 1) return fail("no block count");
  if (block >= nblocks) return fail("no such block");
  int d[3] = {0, 0, 0};
  for (int bi = 0; bi <= block; bi++) {
    if (format == 1) {
      if (fread(d, sizeof(int), 3, f) != 3) return fail("truncated block header");
    } else if (fscanf(f, "%i %i %i\n", &d[0], &d[1], &d[2]) != 3) {
      return fail("truncated block header");
    }
    if (d[0] < 2 || d[1] < 2 || d[2] < 2) return fail("bad node counts");
    const long long n = (long long)d[0] * d[1] * d[2];
    if (bi < block && !skip_doubles(f, format, 3 * n)) return fail("truncated block");
  }
  *IM = d[0]; *JM = d[1]; *KM = d[2];
  if (!x) { fclose(f); return VFS_OK; }
  if (!y || !z) return fail("null coordinate array");
  const long long nI = d[0], nJ = d[1], nK = d[2], n = nI * nJ * nK;
  if (format == 2) {
    std::vector<double> X(nI), Y(nJ), Z(nK);
    double t0, t1;
    for (long long i = 0; i < nI; i++) if (fscanf(f, "%le %le %le\n", &X[i], &t0, &t1) != 3) return fail("truncated x list");
    for (long long j = 0; j < nJ; j++) if (fscanf(f, "%le %le %le\n", &t0, &Y[j], &t1) != 3) return fail("truncated y list");
    for (long long k = 0; k < nK; k++) if (fscanf(f, "%le %le %le\n", &t0, &t1, &Z[k]) != 3) return fail("truncated z list");
    for (long long k = 0; k < nK; k++)
      for (long long j = 0; j < nJ; j++)
        for (long long i = 0; i < nI; i++) {
          const long long p = (k * nJ + j) * nI + i;
          x[p] = X[i] / cl * L_dim;
          y[p] = Y[j] / cl * L_dim;
          z[p] = Z[k] / cl * L_dim;
        }
    fclose(f);
    return VFS_OK;
  }
  double *dst[3] = {x, y, z};
  for (int c = 0; c < 3; c++)
    for (long long p = 0; p < n; p++) {
      double v;
      if (format == 1 ? fread(&v, sizeof(double), 1, f) != 1 : fscanf(f, "%le", &v) != 1) return fail("truncated coordinates");
      dst[c][p] = v / cl * L_dim;
    }
  fclose(f);
  return VFS_OK;
}

extern "C" int vfs_grid_write(const char *path, int format, int IM, int JM, int KM, const double *x, const double *y,
                              const double *z) {
  if (!path || !x || !y || !z || format < 0 || format > 2 || IM < 2 || JM < 2 || KM < 2)
    return vfs::set_err(nullptr, VFS_ERR_INVALID, "vfs_grid_write: bad argument");
  const long long nI = IM, nJ = JM, nK = KM, n = nI * nJ * nK;
  if (format == 2) {  // a tensor grid only
    for (long long k = 0; k < nK; k++)
      for (long long j = 0; j < nJ; j++)
        for (long long i = 0; i < nI; i++) {
          const long long p = (k * nJ + j) * nI + i;
          if (x[p] != x[i] || y[p] != y[j * nI] || z[p] != z[k * nJ * nI])
            return vfs::set_err(nullptr, VFS_ERR_INVALID, "vfs_grid_write: xyz.dat holds tensor-product grids only");
        }
  }
  FILE *f = fopen(path, format == 1 ? "wb" : "w");
  if (!f) return vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_grid_write: cannot create ") + path);
  bool ok = true;
  if (format == 1) {
    const int hdr[4] = {1, IM, JM, KM};
    ok = fwrite(hdr, sizeof(int), 4, f) == 4 && fwrite(x, sizeof(double), n, f) == (size_t)n &&
         fwrite(y, sizeof(double), n, f) == (size_t)n && fwrite(z, sizeof(double), n, f) == (size_t)n;
  } else if (format == 0) {
    ok = fprintf(f, "1\n%d %d %d\n", IM, JM, KM) > 0;
    const double *src[3] = {x, y, z};
    for (int c = 0; c < 3 && ok; c++)
      for (long long p = 0; p < n && ok; p++) ok = fprintf(f, "%.17e\n", src[c][p]) > 0;
  } else {
    ok = fprintf(f, "%d %d %d\n", IM, JM, KM) > 0;
    for (long long i = 0; i < nI && ok; i++) ok = fprintf(f, "%.17e 0 0\n", x[i]) > 0;
    for (long long j = 0; j < nJ && ok; j++) ok = fprintf(f, "0 %.17e 0\n", y[j * nI]) > 0;
    for (long long k = 0; k < nK && ok; k++) ok = fprintf(f, "0 0 %.17e\n", z[k * nJ * nI]) > 0;
  }
  if (fclose(f) != 0) ok = false;
  return ok ? VFS_OK : vfs::set_err(nullptr, VFS_ERR_INVALID, std::string("vfs_grid_write: write failed: ") + path);
}
