// ref_grid_driver.cpp -- runs the reference's own vmap grid generation
// (gridmesh::gridmesh + readdata -> read_vmapnew, src/gridmesh.cpp, built
// unmodified from its sources with the reference's TypeDouble option) on a
// vmap file, then its calmetric and absorb::CalCFSfactors on that grid, for
// the parity fixtures of cgfd_grid_vmap, cgfd_metric_from_coords and
// cgfd_cfs_factors.
//
// TEST INFRASTRUCTURE ONLY (oracle/ref): never linked into the product.
//
// usage: ref_grid <dir> <ni> <nj> <nk> <hybrid> <conversion depth> <out>
//                 [<metric out> [<pml out> <n0..n5> <velocity> <bmax> <amax> <stept>]]
//   <dir>/grid.dat must hold the vmap file (vmap_dims / vmap_gridpoints /
//   vmap_equalspacing / <vmap_anchor> block); the driver writes the par
//   files the reference reads next to it (keep <dir> short: the reference
//   keeps paths in 128-byte buffers).  <out>: int32 ConIndex, then x, y, z
//   as float64 full arrays (ni+6)(nj+6)(nk+6), z fastest.  <metric out>:
//   gridmesh::calmetric's xi_x..z, eta_x..z, zeta_x..z and jac for that
//   grid (steph 100, the grid's own), as ten such float64 arrays.  <pml
//   out>: absorb::CalCFSfactors (src/absorb.cpp:346-805) on that metric with
//   abs_number n0..n5 and one velocity, bmax and amax for all six faces:
//   APD, B, DB for x (ni+6), then y (nj+6), then z (nk+6), float64.
#include "typenew.h"

#include <cstdio>
#include <cstdlib>

using namespace defstruct;

int main(int argc, char **argv) {
  if (argc != 8 && argc != 9 && argc != 20) {
    std::fprintf(stderr, "usage: ref_grid <dir> <ni> <nj> <nk> <hybrid> <depth> <out> "
                         "[<metric> [<pml> n0..n5 vel bmax amax stept]]\n");
    return 2;
  }
  const char *dir = argv[1];
  const int ni = std::atoi(argv[2]), nj = std::atoi(argv[3]), nk = std::atoi(argv[4]);
  const int hybrid = std::atoi(argv[5]);
  const double depth = std::atof(argv[6]);
  char conf[256], src[256];
  std::snprintf(conf, sizeof conf, "%s/SeisFD3D.conf", dir);
  std::snprintf(src, sizeof src, "%s/source.dat", dir);
  FILE *f = std::fopen(conf, "w");
  if (!f) return 3;
  std::fprintf(f, "seispath = %s\ngrid_type = vmap\ngrid_filename = grid.dat\n", dir);
  std::fprintf(f, "hybrid_grid = %d\nconversion_interface_depth = %.17g\n", hybrid, depth);
  std::fprintf(f, "source_filename = source.dat\nreference_velocity = 2000.0\n");
  std::fprintf(f, "absorb_filename = absorb.dat\n");
  std::fclose(f);
  f = std::fopen(src, "w");
  if (!f) return 3;
  std::fprintf(f, "number_of_force_source = 0\nnumber_of_moment_source = 1\n");
  std::fprintf(f, "moment_stf_window = 1\nmoment_stf_freqfactor = 2.0\n");
  std::fclose(f);

  cindx cdx;
  cdx.ni = ni; cdx.nj = nj; cdx.nk = nk;
  cdx.nx = ni + 6; cdx.ny = nj + 6; cdx.nz = nk + 6;
  cdx.nx1 = 0; cdx.nx2 = cdx.nx; cdx.ny1 = 0; cdx.ny2 = cdx.ny; cdx.nz1 = 0; cdx.nz2 = cdx.nz;
  cdx.ni1 = 3; cdx.ni2 = ni + 3; cdx.nj1 = 3; cdx.nj2 = nj + 3; cdx.nk1 = 3; cdx.nk2 = nk + 3;
  gridmesh gm(conf, cdx, 0, 0);
  gm.readdata(cdx, conf, 100.0);

  FILE *o = std::fopen(argv[7], "wb");
  if (!o) return 4;
  const int con = gm.ConIndex;
  std::fwrite(&con, sizeof con, 1, o);
  Real ***v[3] = {gm.crd.x, gm.crd.y, gm.crd.z};
  for (int q = 0; q < 3; ++q)
    for (int i = 0; i < cdx.nx; ++i)
      for (int j = 0; j < cdx.ny; ++j)
        for (int k = 0; k < cdx.nz; ++k) {
          const double d = (double)v[q][i][j][k];
          std::fwrite(&d, sizeof d, 1, o);
        }
  std::fclose(o);
  if (argc >= 9) {
    gm.calmetric(100.0, cdx);
    FILE *om = std::fopen(argv[8], "wb");
    if (!om) return 4;
    Real ***d[10] = {gm.drv.xi_x,   gm.drv.xi_y,   gm.drv.xi_z,   gm.drv.eta_x,
                     gm.drv.eta_y,  gm.drv.eta_z,  gm.drv.zeta_x, gm.drv.zeta_y,
                     gm.drv.zeta_z, gm.drv.jac};
    for (int q = 0; q < 10; ++q)
      for (int i = 0; i < cdx.nx; ++i)
        for (int j = 0; j < cdx.ny; ++j)
          for (int k = 0; k < cdx.nz; ++k) {
            const double v = (double)d[q][i][j][k];
            std::fwrite(&v, sizeof v, 1, om);
          }
    std::fclose(om);
  }
  if (argc == 20) {
    char absf[256];
    std::snprintf(absf, sizeof absf, "%s/absorb.dat", dir);
    FILE *fa = std::fopen(absf, "w");
    if (!fa) return 3;
    std::fprintf(fa, "abs_number = %s %s %s %s %s %s\n", argv[10], argv[11], argv[12], argv[13],
                 argv[14], argv[15]);
    const char *keys[3] = {"abs_velocity", "bmax", "amax"};
    for (int q = 0; q < 3; ++q) {
      std::fprintf(fa, "%s =", keys[q]);
      for (int t = 0; t < 6; ++t) std::fprintf(fa, " %s", argv[16 + q]);
      std::fprintf(fa, "\n");
    }
    std::fclose(fa);
    absorb ab(conf, cdx, 0, 0);
    ab.CalCFSfactors(cdx, gm.drv, 100.0, (Real)std::atof(argv[19]));
    FILE *op = std::fopen(argv[9], "wb");
    if (!op) return 4;
    Real *arr[9] = {ab.apr.APDx, ab.apr.Bx, ab.apr.DBx, ab.apr.APDy, ab.apr.By,
                    ab.apr.DBy,  ab.apr.APDz, ab.apr.Bz, ab.apr.DBz};
    const int len[3] = {cdx.nx, cdx.ny, cdx.nz};
    for (int q = 0; q < 9; ++q)
      for (int t = 0; t < len[q / 3]; ++t) {
        const double v = (double)arr[q][t];
        std::fwrite(&v, sizeof v, 1, op);
      }
    std::fclose(op);
  }
  return 0;
}
