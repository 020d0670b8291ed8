/* Replacement for the CUDA samples' helper_cuda.h (not in this image).
 * TEST INFRASTRUCTURE (oracle/ref). */
#ifndef CGFD_REF_STUB_HELPER_CUDA_H
#define CGFD_REF_STUB_HELPER_CUDA_H
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#define checkCudaErrors(call)                                                   \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),       \
              __FILE__, __LINE__);                                              \
      exit(92);                                                                 \
    }                                                                           \
  } while (0)
#endif
