// seisnc_stub.cpp -- the members of the reference's class seisnc that its
// gridmesh.cpp and source.cpp refer to, for the parity drivers (ref_grid,
// ref_source).  TEST
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

// members source.cpp refers to (focal NetCDF input, restart import/export);
// the parity drivers never reach them
size_t seisnc::dimsize(const char *, const char *) {
  no_netcdf("seisnc::dimsize");
  return 0;
}
void seisnc::attrget(const char *, const char *, Real *) { no_netcdf("seisnc::attrget"); }
void seisnc::varget(const char *, const char *, Real *) { no_netcdf("seisnc::varget"); }
void seisnc::force_export(defstruct::force, const char *, int, int) {
  no_netcdf("seisnc::force_export");
}
void seisnc::force_import(defstruct::force, const char *, int, int) {
  no_netcdf("seisnc::force_import");
}
void seisnc::moment_export(defstruct::moment, const char *, int, int) {
  no_netcdf("seisnc::moment_export");
}
void seisnc::moment_import(defstruct::moment, const char *, int, int) {
  no_netcdf("seisnc::moment_import");
}
void seisnc::focal_export(defstruct::Rmom, const char *) { no_netcdf("seisnc::focal_export"); }
void seisnc::focal_import(defstruct::Rmom, const char *) { no_netcdf("seisnc::focal_import"); }

// common::errorprint reports through the reference's MPI helper
// (src/datadis.cc); single process here: print and stop
void MpiErrorPrint(const char *file, int line, int code, const char *msg) {
  std::fprintf(stderr, "reference error %d at %s:%d: %s\n", code, file, line, msg);
  std::exit(code ? code : 1);
}
