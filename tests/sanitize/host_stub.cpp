// host_stub.cpp -- the few library-internal symbols the host-side sources
// (setup.cpp, ncread.cpp, ncinput.cpp, ncwrite.cpp) take from the solver's
// device code, so that they build alone into a sanitizer-instrumented
// library for tests/test_host_sanitizers.py.
#include "../../copara-cgfd3d_b200/csrc/abi_guard.h"
#include "../../include/cgfd.h"

#include <cstdio>
#include <string>

namespace cgfd {
thread_local std::string g_err;
void set_global_error(const char *msg) { g_err = msg; }
int abi_exception(const cgfd_solver *, const char *fn) noexcept {
  g_err = fn;
  return CGFD_ERR_NOMEM;
}
int abi_exception(const cgfd_batch *, const char *fn) noexcept {
  g_err = fn;
  return CGFD_ERR_NOMEM;
}
}  // namespace cgfd

extern "C" int cgfd_last_error(const cgfd_solver *, char *buf, size_t len) {
  if (!buf || len == 0) return CGFD_ERR_ARG;
  std::snprintf(buf, len, "%s", cgfd::g_err.c_str());
  return CGFD_OK;
}
