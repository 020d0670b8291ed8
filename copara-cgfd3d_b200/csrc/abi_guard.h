// abi_guard.h -- keeps C++ exceptions on this side of the C ABI.
//
// Every extern "C" entry point runs its body between CGFD_ABI_BEGIN and
// CGFD_ABI_END(handle).  A C++ exception raised inside -- in practice a host
// allocation that fails (std::bad_alloc, std::length_error) or a host thread
// that cannot be started (std::system_error) -- is caught there and becomes
// CGFD_ERR_NOMEM, with the entry point's name and the exception's text in the
// handle's last error (cgfd_last_error / cgfd_batch_last_error), or in the
// process-wide one when the call has no handle.  A C or Fortran caller, or one
// built without exception support, never sees an unwind through its frames.
#pragma once

#include <cstddef>

struct cgfd_solver;
struct cgfd_batch;

namespace cgfd {

// Called only from inside a catch handler: records the exception in flight
// and returns CGFD_ERR_NOMEM.
int abi_exception(const cgfd_solver *h, const char *fn) noexcept;
int abi_exception(const cgfd_batch *b, const char *fn) noexcept;
inline int abi_exception(std::nullptr_t, const char *fn) noexcept {
  return abi_exception(static_cast<const cgfd_solver *>(nullptr), fn);
}

}  // namespace cgfd

#define CGFD_ABI_BEGIN try {
#define CGFD_ABI_END(handle) \
  }                          \
  catch (...) { return ::cgfd::abi_exception((handle), __func__); }
