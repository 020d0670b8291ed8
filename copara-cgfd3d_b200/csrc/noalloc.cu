// noalloc.cu -- cgfd_count_nonfinite_noalloc: the NaN/Inf count of
// cgfd_check_finite on any float array already on the device, with no device
// memory allocation at all.
//
// Why: some callers cannot call cudaMalloc at the moment they want the check
// -- a host application whose memory pool owns the whole device, a
// real-time loop that must not take the allocator's implicit
// synchronisation, or code that only borrows device buffers from another
// framework.  They still pass the input (a device pointer and its length)
// and the output (a host integer).
//
// The two kernels are the ones cgfd_check_finite runs (nonfinite.cuh); only
// their scratch differs: instead of per-solver memory from cudaMalloc it is
// the file-scope array g_nonfinite_scratch below, NOALLOC_MAX_BLOCKS partial
// counts plus one total (131 KB; every GPU that loads the library holds it
// until exit).  One partial covers NF_CHUNK = 8192 values, so a call handles
// at most NOALLOC_MAX_VALUES = 134,217,728 values (512 MiB of floats) and
// rejects larger sizes with CGFD_ERR_ARG before touching the device.
//
// In host code the array's name is only a host-side stand-in, not a device
// address; every call looks the device address up with cudaGetSymbolAddress,
// with the array's device current (cheap once the module is loaded, and
// never stale: a cudaDeviceReset by the host program reloads the module and
// may move the array).  The first call on a device loads the module there,
// which is set-up work, so it should come before any stream capture.  Every
// call shares the one array and leaves its last
// contents there: each slot a call reads is written by the same call first,
// so nothing needs clearing, but calls that overlap on the GPU (on different
// streams, or from different host threads) race on it and must be serialised
// by the caller.
#include "../../include/cgfd.h"
#include "abi_guard.h"
#include "cgfd_internal.cuh"
#include "nonfinite.cuh"

#include <cuda_runtime.h>

#include <cstdio>

using namespace cgfd;
using namespace cgfd::nf;

namespace {

constexpr int NOALLOC_MAX_BLOCKS = 16384;
constexpr size_t NOALLOC_MAX_VALUES = (size_t)NOALLOC_MAX_BLOCKS * NF_CHUNK;
static_assert(NOALLOC_MAX_VALUES == (size_t)CGFD_NOALLOC_MAX_VALUES,
              "the header's limit is the scratch array's");

// partial counts [0, NOALLOC_MAX_BLOCKS) and the total at [nblocks]
static __device__ __align__(256) unsigned long long g_nonfinite_scratch[NOALLOC_MAX_BLOCKS + 1];

}  // namespace

extern "C" int cgfd_count_nonfinite_noalloc(const float *d_values, size_t n, long long *n_bad,
                                            void *stream) {
  CGFD_ABI_BEGIN
  if (!n_bad || (n > 0 && !d_values)) {
    set_global_error("cgfd_count_nonfinite_noalloc: null argument");
    return CGFD_ERR_ARG;
  }
  *n_bad = 0;
  if (n == 0) return CGFD_OK;
  if (n > NOALLOC_MAX_VALUES) {
    char buf[160];
    std::snprintf(buf, sizeof(buf),
                  "cgfd_count_nonfinite_noalloc: %zu values exceed the fixed scratch "
                  "(at most %zu values per call)", n, NOALLOC_MAX_VALUES);
    set_global_error(buf);
    return CGFD_ERR_ARG;
  }
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, d_values);
  if (e != cudaSuccess || (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) ||
      attr.device < 0) {
    cudaGetLastError();
    set_global_error("cgfd_count_nonfinite_noalloc: d_values is not device memory");
    return CGFD_ERR_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != attr.device) cudaSetDevice(attr.device);
  int status = CGFD_OK;
  unsigned long long *scratch = nullptr;
  {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_nonfinite_scratch);
    if (e == cudaSuccess) scratch = (unsigned long long *)p;
  }
  if (!scratch) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "cgfd_count_nonfinite_noalloc: cudaGetSymbolAddress: %s",
                  cudaGetErrorString(e));
    set_global_error(buf);
    status = CGFD_ERR_CUDA;
  } else {
    const int nblocks = (int)nonfinite_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    nonfinite_partial_kernel<<<nblocks, NF_THREADS, 0, s>>>(d_values, n, scratch);
    nonfinite_sum_kernel<<<1, NF_THREADS, 0, s>>>(scratch, nblocks);
    unsigned long long total = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&total, scratch + nblocks, sizeof(total), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      char buf[160];
      std::snprintf(buf, sizeof(buf), "cgfd_count_nonfinite_noalloc: %s", cudaGetErrorString(e));
      set_global_error(buf);
      status = CGFD_ERR_CUDA;
    } else {
      *n_bad = (long long)total;
      if (total) status = CGFD_ERR_NONFINITE;
    }
  }
  if (prev >= 0 && prev != attr.device) cudaSetDevice(prev);
  return status;
  CGFD_ABI_END(nullptr)
}
