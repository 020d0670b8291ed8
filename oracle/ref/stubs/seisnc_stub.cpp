// seisnc_stub.cpp -- the members of the reference's class seisnc that its
// gridmesh.cpp refers to, for the grid parity driver (ref_grid).  TEST
// INFRASTRUCTURE: no NetCDF I/O is compiled in; the vmap path never calls
// these, and they stop the program if it ever does.
#include "typenew.h"

#include <cstdio>
#include <cstdlib>

static void no_netcdf(const char *what) {
  std::fprintf(stderr, "ref_grid: %s needs NetCDF, which this driver does not build\n", what);
  std::exit(5);
}

seisnc::seisnc() {}
void seisnc::varget(const char *, const char *, Real *, size_t *, size_t *, ptrdiff_t *) {
  no_netcdf("seisnc::varget");
}
void seisnc::grid_export(defstruct::coord, defstruct::deriv, defstruct::cindx, const char *,
                         const char *) {
  no_netcdf("seisnc::grid_export");
}
void seisnc::grid_import(defstruct::coord, defstruct::deriv, defstruct::cindx, const char *,
                         const char *) {
  no_netcdf("seisnc::grid_import");
}

// common::errorprint reports through the reference's MPI helper
// (src/datadis.cc); single process here: print and stop
void MpiErrorPrint(const char *file, int line, int code, const char *msg) {
  std::fprintf(stderr, "reference error %d at %s:%d: %s\n", code, file, line, msg);
  std::exit(code ? code : 1);
}
