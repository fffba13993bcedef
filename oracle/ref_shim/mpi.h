/* Single-rank stand-in for the handful of MPI declarations that the
 * reference's hot-path headers name (NEWEST5/utils.h MaxTempGev,
 * NEWEST5/hydroKT.h CFL, NEWEST5/multiroot.h CheckRoot, NEWEST5/boundary.h
 * neighbour macros).  MPI is not installed in this image.  With one rank and
 * NPX = NPY = 1 every neighbour is BOUNDARY, so the halo exchange never
 * runs; reductions over one rank are copies.  This is test infrastructure
 * for the oracle only: nothing in the product links it.
 */
#ifndef VH_REF_SHIM_MPI_H
#define VH_REF_SHIM_MPI_H

#include <string.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef struct { int source, tag, error; } MPI_Status;
typedef int MPI_File;
typedef int MPI_Info;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_DOUBLE_INT 3
#define MPI_MAX 10
#define MPI_MIN 11
#define MPI_SUM 12
#define MPI_MAXLOC 13
#define MPI_MINLOC 14
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL 0
#define MPI_INFO_NULL 0
#define MPI_SEEK_SET 0
#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4

static inline int vh_shim_type_size(MPI_Datatype t) {
  return t == MPI_DOUBLE ? 8 : t == MPI_INT ? 4 : t == MPI_DOUBLE_INT ? 16 : 8;
}
/* one rank: every reduction is a copy of the send buffer */
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  memcpy(r, s, (size_t)n * vh_shim_type_size(t));
  return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  memcpy(r, s, (size_t)n * vh_shim_type_size(t));
  return 0;
}
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int c) { abort(); return c; }
static inline int MPI_Cart_rank(MPI_Comm, const int*, int* r) { *r = 0; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int, int* c) { c[0] = c[1] = c[2] = 0; return 0; }
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* c) { *c = 0; return 0; }
/* the halo exchange is unreachable with one rank; reaching it is a harness bug */
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { abort(); return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { abort(); return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }

#endif
