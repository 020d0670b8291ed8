/* A C99 caller of the C ABI (tests/test_abi.py builds and runs it): the
 * header compiles as strict C, the library links from C, a host-side entry
 * point computes, and an argument error comes back as a status with its
 * text -- no GPU is touched. */
#include "cgfd.h"

#include <stdio.h>

int main(void) {
  double m6[6];
  char err[256];
  cgfd_solver *h = NULL;
  cgfd_desc d = {0};
  if (cgfd_angle2moment(30.0, 60.0, 90.0, m6) != CGFD_OK) return 2;
  const int st = cgfd_create(&d, &h); /* ni = 0: refused before any device call */
  cgfd_last_error(NULL, err, sizeof err);
  printf("abi %d m6 %.6f %.6f %.6f create %d %s\n", CGFD_ABI_VERSION, m6[0], m6[1], m6[2], st,
         err);
  return h == NULL ? 0 : 3;
}
