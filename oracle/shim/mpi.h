/* mpi.h -- single-process stand-in for the MPI calls the Grains3D sources
 * reference, so that the reference can be compiled unmodified as the
 * serial (Type="Standard") oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Semantics: one rank (rank 0 of size 1).  Collectives copy the send buffer
 * to the receive buffer; point-to-point calls abort, since a one-rank run
 * never reaches them.  MPI-IO writes go through stdio.  The signatures are
 * those of the MPI standard. */
#ifndef GRAINS_ORACLE_SHIM_MPI_H
#define GRAINS_ORACLE_SHIM_MPI_H

#include <limits.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Group;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef FILE* MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_COMM_SELF 2
#define MPI_GROUP_NULL 0
#define MPI_INFO_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)-1)
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_RDONLY 4
#define MPI_MODE_APPEND 8
#define MPI_UNDEFINED (-32766)

enum { MPI_CHAR = 1, MPI_INT, MPI_DOUBLE, MPI_UNSIGNED_LONG, MPI_UNSIGNED_SHORT, MPI_UNSIGNED,
       MPI_LONG, MPI_FLOAT, MPI_BYTE, MPI_SHORT, MPI_UNSIGNED_CHAR, MPI_LONG_LONG,
       MPI_UNSIGNED_LONG_LONG, MPI_C_BOOL, MPI_CXX_BOOL, MPI_DERIVED_BASE = 100 };
enum { MPI_SUM = 1, MPI_MIN, MPI_MAX, MPI_LAND, MPI_LOR, MPI_PROD };

#ifdef __cplusplus
extern "C" {
#endif
size_t grains_shim_type_size(MPI_Datatype t);
int grains_shim_type_register(size_t bytes);
#ifdef __cplusplus
}
#endif

static inline int grains_shim_abort(const char* what) {
  fprintf(stderr, "single-rank MPI shim: %s is not available\n", what);
  abort();
  return 1;
}

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Initialized(int* f) { *f = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int grains_shim_copy(const void* s, void* r, int n, MPI_Datatype t) {
  if (s != MPI_IN_PLACE && s != r && n > 0) memcpy(r, s, (size_t)n * grains_shim_type_size(t));
  return 0;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
  (void)o; (void)c; return grains_shim_copy(s, r, n, t);
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c) {
  (void)o; (void)root; (void)c; return grains_shim_copy(s, r, n, t);
}
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return 0;
}
static inline int MPI_Gather(const void* s, int ns, MPI_Datatype ts, void* r, int nr, MPI_Datatype tr,
                             int root, MPI_Comm c) {
  (void)nr; (void)tr; (void)root; (void)c; return grains_shim_copy(s, r, ns, ts);
}
static inline int MPI_Allgather(const void* s, int ns, MPI_Datatype ts, void* r, int nr, MPI_Datatype tr,
                                MPI_Comm c) {
  (void)nr; (void)tr; (void)c; return grains_shim_copy(s, r, ns, ts);
}
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return grains_shim_abort("MPI_Send");
}
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r; return grains_shim_abort("MPI_Isend");
}
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return grains_shim_abort("MPI_Recv");
}
static inline int MPI_Probe(int s, int tag, MPI_Comm c, MPI_Status* st) {
  (void)s; (void)tag; (void)c; (void)st; return grains_shim_abort("MPI_Probe");
}
static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* n) {
  (void)st; (void)t; *n = 0; return grains_shim_abort("MPI_Get_count");
}
static inline int MPI_Wait(MPI_Request* r, MPI_Status* st) { (void)r; (void)st; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Comm_group(MPI_Comm c, MPI_Group* g) { (void)c; *g = 1; return 0; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm* n) { (void)g; *n = c; return 0; }
static inline int MPI_Group_incl(MPI_Group g, int n, const int* r, MPI_Group* ng) {
  (void)n; (void)r; *ng = g; return 0;
}
static inline int MPI_Group_free(MPI_Group* g) { *g = MPI_GROUP_NULL; return 0; }
static inline int MPI_Cart_create(MPI_Comm c, int nd, const int* dims, const int* per, int reorder,
                                  MPI_Comm* n) {
  (void)nd; (void)dims; (void)per; (void)reorder; *n = c; return 0;
}
static inline int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int* coords) {
  (void)c; (void)rank; for (int i = 0; i < nd; ++i) coords[i] = 0; return 0;
}
static inline int MPI_Cart_rank(MPI_Comm c, const int* coords, int* rank) {
  (void)c; (void)coords; *rank = 0; return 0;
}
static inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype* nt) {
  *nt = grains_shim_type_register((size_t)n * grains_shim_type_size(old)); return 0;
}
static inline int MPI_Type_commit(MPI_Datatype* t) { (void)t; return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) { (void)t; return 0; }
static inline int MPI_File_open(MPI_Comm c, const char* name, int mode, MPI_Info info, MPI_File* f) {
  (void)c; (void)mode; (void)info;
  *f = fopen(name, "wb");
  return *f ? 0 : 1;
}
static inline int MPI_File_close(MPI_File* f) { if (*f) fclose(*f); *f = NULL; return 0; }
static inline int MPI_File_write(MPI_File f, const void* b, int n, MPI_Datatype t, MPI_Status* st) {
  (void)st; fwrite(b, grains_shim_type_size(t), (size_t)n, f); return 0;
}
static inline int MPI_File_write_at(MPI_File f, MPI_Offset off, const void* b, int n, MPI_Datatype t,
                                    MPI_Status* st) {
  (void)st; fseek(f, (long)off, SEEK_SET); fwrite(b, grains_shim_type_size(t), (size_t)n, f); return 0;
}
static inline int MPI_File_write_at_all(MPI_File f, MPI_Offset off, const void* b, int n,
                                        MPI_Datatype t, MPI_Status* st) {
  return MPI_File_write_at(f, off, b, n, t, st);
}

#endif
