/* Minimal MPI declarations so that the reference's sources compile into a
 * single-process program.  TEST INFRASTRUCTURE (oracle/ref): the parity driver
 * runs one rank with one device and never communicates; every call that would
 * communicate reports an error and stops the process. */
#ifndef CGFD_REF_STUB_MPI_H
#define CGFD_REF_STUB_MPI_H
#include <stdio.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_CHAR 4
#define MPI_LONG 5

static inline int cgfd_ref_no_mpi(const char *what) {
  fprintf(stderr, "reference driver: %s called in the single-process build\n", what);
  exit(90);
  return 1;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return cgfd_ref_no_mpi("MPI_Send"); }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return cgfd_ref_no_mpi("MPI_Recv"); }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code ? code : 91); return 0; }
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 1; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 2; return 0; }
#endif
