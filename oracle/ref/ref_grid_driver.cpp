// ref_grid_driver.cpp -- runs the reference's own vmap grid generation
// (gridmesh::gridmesh + readdata -> read_vmapnew, src/gridmesh.cpp, built
// unmodified from its sources with the reference's TypeDouble option) on a
// vmap file, for the parity fixtures of cgfd_grid_vmap.
//
// TEST INFRASTRUCTURE ONLY (oracle/ref): never linked into the product.
//
// usage: ref_grid <dir> <ni> <nj> <nk> <hybrid> <conversion depth> <out>
//   <dir>/grid.dat must hold the vmap file (vmap_dims / vmap_gridpoints /
//   vmap_equalspacing / <vmap_anchor> block); the driver writes the par
//   files the reference reads next to it (keep <dir> short: the reference
//   keeps paths in 128-byte buffers).  <out>: int32 ConIndex, then x, y, z
//   as float64 full arrays (ni+6)(nj+6)(nk+6), z fastest.
#include "typenew.h"

#include <cstdio>
#include <cstdlib>

using namespace defstruct;

int main(int argc, char **argv) {
  if (argc != 8) {
    std::fprintf(stderr, "usage: ref_grid <dir> <ni> <nj> <nk> <hybrid> <depth> <out>\n");
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
  return 0;
}
