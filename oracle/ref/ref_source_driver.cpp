// ref_source_driver.cpp -- runs the reference's own source location and
// smoothing (source::source + readdata + cal_index, src/source.cpp, with its
// SrcSmooth and TypeDouble options) and its point location
// (common::reposition, src/common.cpp:225-270, as seisplot::locpoint calls it
// for receivers), built unmodified from the sources, for the parity fixtures
// of cgfd_locate_points, cgfd_source_smoothing, cgfd_stf and
// cgfd_angle2moment.
//
// TEST INFRASTRUCTURE ONLY (oracle/ref): never linked into the product.
//
// usage: ref_source <dir> <in> <out> [<ftype> <ft0> <ff0> <mtype> <mt0> <mf0> <mech> <start>]
//   <in> (binary, native endian): int32 ni nj nk nf nm np nt; float64 hyp,
//   stept; x, y, z, rho, vs as float64 full arrays (ni+6)(nj+6)(nk+6), z
//   fastest; nf force rows (x y z fx fy fz), nm moment rows (x y z mxx myy
//   mzz mxy mxz myz), np receiver rows (x y z), all float64.
//   The driver writes the par files the reference reads into <dir> (keep it
//   short: the reference keeps paths in 128-byte buffers).  Source time
//   functions: force_stf_type <ftype> with time factor <ft0> and frequency
//   factor <ff0>, moment_stf_type likewise, every source starting at
//   <start>; moment_mech_input <mech> ("moment", or "angle": the first three
//   of a moment row's six values are strike, dip, rake).  Default: Ricker,
//   t0 = 0.6 s, f0 = 2 Hz, "moment", start 0.
//   <out>: per force: int32 loc[3], float64 posz, dnorm[343], stf[2(nt+1)],
//   fx fy fz; per moment the same with mxx myy mzz mxy mxz myz (x mu for
//   "angle"); per receiver: int32 loc[3], float64 posz.
#include "typenew.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace defstruct;

namespace {

Real ***cube(int nx, int ny, int nz, const double *src) {
  Real ***v = new Real **[nx];
  for (int i = 0; i < nx; ++i) {
    v[i] = new Real *[ny];
    for (int j = 0; j < ny; ++j) {
      v[i][j] = new Real[nz];
      for (int k = 0; k < nz; ++k) v[i][j][k] = (Real)src[((size_t)i * ny + j) * nz + k];
    }
  }
  return v;
}

template <class T>
bool get(FILE *f, T *p, size_t n) {
  return std::fread(p, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 4 && argc != 12) {
    std::fprintf(stderr, "usage: ref_source <dir> <in> <out> [ftype ft0 ff0 mtype mt0 mf0 mech "
                         "start]\n");
    return 2;
  }
  const bool opt = argc == 12;
  const char *ftype = opt ? argv[4] : "Ricker", *ft0 = opt ? argv[5] : "0.6",
             *ff0 = opt ? argv[6] : "2.0", *mtype = opt ? argv[7] : "Ricker",
             *mt0 = opt ? argv[8] : "0.6", *mf0 = opt ? argv[9] : "2.0",
             *mech = opt ? argv[10] : "moment", *start = opt ? argv[11] : "0.0";
  const bool angle = std::string(mech) == "angle";
  const char *dir = argv[1];
  FILE *in = std::fopen(argv[2], "rb");
  if (!in) return 3;
  int hdr[7];
  double hyp, stept;
  if (!get(in, hdr, 7) || !get(in, &hyp, 1) || !get(in, &stept, 1)) return 3;
  const int ni = hdr[0], nj = hdr[1], nk = hdr[2], nf = hdr[3], nm = hdr[4], np = hdr[5];
  const int nt = hdr[6];
  const int nx = ni + 6, ny = nj + 6, nz = nk + 6;
  const size_t n = (size_t)nx * ny * nz;
  std::vector<double> arr[5];
  for (auto &a : arr) {
    a.resize(n);
    if (!get(in, a.data(), n)) return 3;
  }
  std::vector<double> fr((size_t)6 * nf), mr((size_t)9 * nm), pr((size_t)3 * np);
  if (!get(in, fr.data(), fr.size()) || !get(in, mr.data(), mr.size()) ||
      !get(in, pr.data(), pr.size()))
    return 3;
  std::fclose(in);

  char conf[256], src[256];
  std::snprintf(conf, sizeof conf, "%s/SeisFD3D.conf", dir);
  std::snprintf(src, sizeof src, "%s/source.dat", dir);
  FILE *f = std::fopen(conf, "w");
  if (!f) return 4;
  std::fprintf(f, "seispath = %s\nsource_filename = source.dat\n", dir);
  std::fclose(f);
  f = std::fopen(src, "w");
  if (!f) return 4;
  std::fprintf(f, "source_type = 2\nnumber_of_force_source = %d\nnumber_of_moment_source = %d\n",
               nf, nm);
  std::fprintf(f, "distance2meter = 1.0\nsource_hyper_height = %.17g\n", hyp);
  std::fprintf(f, "force_stf_window = 1\nforce_stf_type = %s\n", ftype);
  std::fprintf(f, "force_stf_timefactor = %s\nforce_stf_freqfactor = %s\n", ft0, ff0);
  std::fprintf(f, "moment_stf_window = 1\nmoment_mech_input = %s\n", mech);
  std::fprintf(f, "moment_stf_type = %s\nmoment_stf_timefactor = %s\n", mtype, mt0);
  std::fprintf(f, "moment_stf_freqfactor = %s\nsimulate_damp = 1.0\n", mf0);
  std::fprintf(f, "<anchor_force>\n");
  for (int q = 0; q < nf; ++q) {
    const double *r = &fr[(size_t)6 * q];
    std::fprintf(f, "%.17g %.17g %.17g %s 1.0 %.17g %.17g %.17g\n", r[0], r[1], r[2], start,
                 r[3], r[4], r[5]);
  }
  std::fprintf(f, "<anchor_moment>\n");
  for (int q = 0; q < nm; ++q) {
    const double *r = &mr[(size_t)9 * q];
    if (angle)
      std::fprintf(f, "%.17g %.17g %.17g %s 1.0 %.17g %.17g %.17g\n", r[0], r[1], r[2], start,
                   r[3], r[4], r[5]);
    else
      std::fprintf(f, "%.17g %.17g %.17g %s 1.0 %.17g %.17g %.17g %.17g %.17g %.17g\n", r[0],
                   r[1], r[2], start, r[3], r[4], r[5], r[6], r[7], r[8]);
  }
  std::fclose(f);

  cindx cdx;
  cdx.ni = ni; cdx.nj = nj; cdx.nk = nk;
  cdx.nx = nx; cdx.ny = ny; cdx.nz = nz;
  cdx.nx1 = 0; cdx.nx2 = nx; cdx.ny1 = 0; cdx.ny2 = ny; cdx.nz1 = 0; cdx.nz2 = nz;
  cdx.ni1 = 3; cdx.ni2 = ni + 3; cdx.nj1 = 3; cdx.nj2 = nj + 3; cdx.nk1 = 3; cdx.nk2 = nk + 3;
  coord crd;
  crd.x = cube(nx, ny, nz, arr[0].data());
  crd.y = cube(nx, ny, nz, arr[1].data());
  crd.z = cube(nx, ny, nz, arr[2].data());
  mdpar mpa{};
  mpa.rho = cube(nx, ny, nz, arr[3].data());
  mpa.beta = cube(nx, ny, nz, arr[4].data());
  mpa.alpha = mpa.beta;

  source sr(conf, nt, 0, 0, 1);
  sr.readdata((Real)stept);
  sr.cal_index(cdx, crd, mpa);

  FILE *o = std::fopen(argv[3], "wb");
  if (!o) return 4;
  auto put_src = [&](int *lx, int *ly, int *lz, Real *pz, Real ****dn, Real **stf, int cnt,
                     std::vector<Real *> coef) {
    for (int q = 0; q < cnt; ++q) {
      const int l[3] = {lx[q], ly[q], lz[q]};
      std::fwrite(l, sizeof(int), 3, o);
      const double z = (double)pz[q];
      std::fwrite(&z, sizeof z, 1, o);
      for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b)
          for (int c = 0; c < 7; ++c) {
            const double d = (double)dn[q][a][b][c];
            std::fwrite(&d, sizeof d, 1, o);
          }
      for (int t = 0; t < sr.nstf; ++t) {
        const double s = (double)stf[q][t];
        std::fwrite(&s, sizeof s, 1, o);
      }
      for (Real *c : coef) {
        const double v = (double)c[q];
        std::fwrite(&v, sizeof v, 1, o);
      }
    }
  };
  if (nf)
    put_src(sr.frc.locx, sr.frc.locy, sr.frc.locz, sr.frc.posz, sr.frc.dnorm, sr.frc.stf, nf,
            {sr.frc.fx, sr.frc.fy, sr.frc.fz});
  if (nm)
    put_src(sr.mnt.locx, sr.mnt.locy, sr.mnt.locz, sr.mnt.posz, sr.mnt.dnorm, sr.mnt.stf, nm,
            {sr.mnt.mxx, sr.mnt.myy, sr.mnt.mzz, sr.mnt.mxy, sr.mnt.mxz, sr.mnt.myz});
  common com;
  for (int q = 0; q < np; ++q) {
    int l[3] = {0, 0, 0};
    Real z = 0;
    const double *p = &pr[(size_t)3 * q];
    com.reposition((Real)p[0], (Real)p[1], (Real)p[2], cdx, crd, (Real)hyp, &l[0], &l[1], &l[2],
                   &z);
    std::fwrite(l, sizeof(int), 3, o);
    const double zz = (double)z;
    std::fwrite(&zz, sizeof zz, 1, o);
  }
  std::fclose(o);
  return 0;
}
