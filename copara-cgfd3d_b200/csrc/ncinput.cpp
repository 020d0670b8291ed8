// ncinput.cpp -- the reference's NetCDF model inputs, read from NetCDF
// classic files (ncread.cpp): the volume media file and the finite-fault
// (focal) series file.  Two-call pattern: with the data pointers NULL the
// functions return the sizes only.
#include "../../include/cgfd.h"
#include "abi_guard.h"
#include "ncread.h"

#include <climits>
#include <cstdio>
#include <string>
#include <vector>

namespace cgfd {
void set_global_error(const char *msg);
}
using namespace cgfd;

namespace {

int fail(const std::string &msg) {
  set_global_error(msg.c_str());
  return CGFD_ERR_ARG;
}

}  // namespace

extern "C" {

// mediapar::read_volume_new (src/mediaparas.cpp:1273-1425) with the default
// build's ZWmedia: dimensions x, y, depth (z without ZWmedia); 1-D variables
// x, y, depth; Vp, Vs, rho over [x][y][depth].  The depth axis is compared
// with the grid's z coordinates as stored (the reference does the same).
int cgfd_read_media_volume_nc(const char *path, int *nvx, int *nvy, int *nvz, double *vx,
                              double *vy, double *vz, float *vp, float *vs, float *rho) {
  CGFD_ABI_BEGIN
  if (!path || !nvx || !nvy || !nvz) return fail("cgfd_read_media_volume_nc: null argument");
  nc::File f;
  if (!f.open(path)) return fail(f.err);
  const char *zname = f.dim("depth") >= 0 ? "depth" : "z";
  const long long n[3] = {f.dim("x"), f.dim("y"), f.dim(zname)};
  if (n[0] < 2 || n[1] < 2 || n[2] < 2)
    return fail(std::string(path) + ": dimensions x, y and depth (or z) of at least 2 needed");
  if (n[0] > INT_MAX || n[1] > INT_MAX || n[2] > INT_MAX)
    return fail(std::string(path) + ": a dimension exceeds the int range");
  long long total = 0;
  if (__builtin_mul_overflow(n[0], n[1], &total) || __builtin_mul_overflow(total, n[2], &total))
    return fail(std::string(path) + ": the volume's size overflows");
  const bool query = !vx;
  if (!query && (*nvx != n[0] || *nvy != n[1] || *nvz != n[2]))
    return fail("cgfd_read_media_volume_nc: the arrays' sizes differ from the file's");
  *nvx = (int)n[0];
  *nvy = (int)n[1];
  *nvz = (int)n[2];
  if (query) return CGFD_OK;
  if (!vy || !vz || !vp || !vs || !rho) return fail("cgfd_read_media_volume_nc: null array");
  std::vector<double> v;
  double *axes[3] = {vx, vy, vz};
  const char *anames[3] = {"x", "y", zname};
  for (int a = 0; a < 3; ++a) {
    if (!f.read(anames[a], &v)) return fail(f.err);
    if ((long long)v.size() != n[a]) return fail(std::string(path) + ": axis size of " + anames[a]);
    for (long long q = 0; q < n[a]; ++q) axes[a][q] = v[q];
  }
  float *outs[3] = {vp, vs, rho};
  const char *names[3] = {"Vp", "Vs", "rho"};
  for (int c = 0; c < 3; ++c) {
    std::vector<size_t> sh;
    if (!f.shape(names[c], &sh) || sh.size() != 3 || (long long)sh[0] != n[0] ||
        (long long)sh[1] != n[1] || (long long)sh[2] != n[2])
      return fail(std::string(path) + ": " + names[c] + " must be [x][y][depth]");
    if (!f.read(names[c], &v)) return fail(f.err);
    for (long long q = 0; q < total; ++q) outs[c][q] = (float)v[q];
  }
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

// source::source + readdata for source_type 1 (src/source.cpp:43-56,
// 796-840): dimensions NP (points) and NT (samples), global attribute DT
// (sample interval, s), variables Mxx Myy Mzz Mxy Mxz Myz [NP][NT] and posx,
// posy, posz [NP] (m).  mom receives [6][NP][NT] in that component order;
// the reference's simulate_damp factor is the caller's to apply.
int cgfd_read_focal_nc(const char *path, int *np, int *nt, double *dt, double *posx,
                       double *posy, double *posz, float *mom) {
  CGFD_ABI_BEGIN
  if (!path || !np || !nt || !dt) return fail("cgfd_read_focal_nc: null argument");
  nc::File f;
  if (!f.open(path)) return fail(f.err);
  const long long p = f.dim("NP"), t = f.dim("NT");
  if (p < 1 || t < 1) return fail(std::string(path) + ": dimensions NP and NT needed");
  if (p > INT_MAX || t > INT_MAX)
    return fail(std::string(path) + ": NP or NT exceeds the int range");
  auto it = f.gatts.find("DT");
  if (it == f.gatts.end() || it->second.empty() || !(it->second[0] > 0.0))
    return fail(std::string(path) + ": a positive global attribute DT is needed");
  const bool query = !mom;
  if (!query && (*np != p || *nt != t))
    return fail("cgfd_read_focal_nc: the arrays' sizes differ from the file's");
  *np = (int)p;
  *nt = (int)t;
  *dt = it->second[0];
  if (query) return CGFD_OK;
  if (!posx || !posy || !posz) return fail("cgfd_read_focal_nc: null array");
  std::vector<double> v;
  const char *names[6] = {"Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"};
  for (int c = 0; c < 6; ++c) {
    std::vector<size_t> sh;
    if (!f.shape(names[c], &sh) || sh.size() != 2 || (long long)sh[0] != p ||
        (long long)sh[1] != t)
      return fail(std::string(path) + ": " + names[c] + " must be [NP][NT]");
    if (!f.read(names[c], &v)) return fail(f.err);
    for (long long q = 0; q < p * t; ++q) mom[(size_t)c * p * t + q] = (float)v[q];
  }
  double *pos[3] = {posx, posy, posz};
  const char *pnames[3] = {"posx", "posy", "posz"};
  for (int a = 0; a < 3; ++a) {
    if (!f.read(pnames[a], &v) || (long long)v.size() != p)
      return fail(std::string(path) + ": " + pnames[a] + " must be [NP]");
    for (long long q = 0; q < p; ++q) pos[a][q] = v[q];
  }
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

}  // extern "C"
