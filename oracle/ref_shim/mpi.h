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

/* MPI-IO on one rank: a file handle is an index into a table of stdio
 * streams (MPI_File_open with MPI_MODE_CREATE opens for update, creating the
 * file; seek, read and write move through the stream).  A harness that
 * defines VH_SHIM_NO_FILES brings its own. */
#ifndef VH_SHIM_NO_FILES
#include <stdio.h>
#define VH_SHIM_MAX_FILES 16
static FILE* vh_shim_files[VH_SHIM_MAX_FILES];
static inline int MPI_File_open(MPI_Comm, const char* name, int amode, MPI_Info, MPI_File* fh) {
  FILE* f = 0;
  if (amode & MPI_MODE_RDONLY) {
    f = fopen(name, "rb");
  } else {
    f = fopen(name, "r+b");
    if (!f && (amode & MPI_MODE_CREATE)) f = fopen(name, "w+b");
  }
  if (!f) return 1;
  for (int q = 1; q < VH_SHIM_MAX_FILES; q++)
    if (!vh_shim_files[q]) { vh_shim_files[q] = f; *fh = q; return 0; }
  fclose(f);
  return 1;
}
static inline int MPI_File_seek(MPI_File fh, MPI_Offset off, int) {
  return fseek(vh_shim_files[fh], (long)off, SEEK_SET) == 0 ? 0 : 1;
}
static inline int MPI_File_write(MPI_File fh, const void* buf, int n, MPI_Datatype t, MPI_Status*) {
  const size_t sz = (size_t)vh_shim_type_size(t);
  return fwrite(buf, sz, (size_t)n, vh_shim_files[fh]) == (size_t)n ? 0 : 1;
}
static inline int MPI_File_read(MPI_File fh, void* buf, int n, MPI_Datatype t, MPI_Status*) {
  const size_t sz = (size_t)vh_shim_type_size(t);
  return fread(buf, sz, (size_t)n, vh_shim_files[fh]) == (size_t)n ? 0 : 1;
}
static inline int MPI_File_close(MPI_File* fh) {
  if (*fh > 0 && *fh < VH_SHIM_MAX_FILES && vh_shim_files[*fh]) {
    fclose(vh_shim_files[*fh]);
    vh_shim_files[*fh] = 0;
  }
  *fh = 0;
  return 0;
}
static inline int MPI_Finalize(void) { return 0; }
#endif

#endif
