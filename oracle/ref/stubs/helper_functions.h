/* Placeholder for the CUDA samples' helper_functions.h (nothing from it is
 * used by the reference's device runtime).  TEST INFRASTRUCTURE (oracle/ref). */
#ifndef CGFD_REF_STUB_HELPER_FUNCTIONS_H
#define CGFD_REF_STUB_HELPER_FUNCTIONS_H
#endif
