/*
 * Single-process stand-in for <mpi.h>, used only to compile the reference's
 * own CPU sources (kernel templates, Euclidean primitives, structured mesh
 * generator) into the test-only library oracle/_ref/libcupcfd_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the shipped library includes this.
 * The reference translation units that are compiled only ever register MPI
 * datatypes (no communication happens on the face-loop path), so every
 * function here is a no-op that reports success on a one-rank world.
 */
#ifndef CUPCFD_ORACLE_MPI_STUB_H
#define CUPCFD_ORACLE_MPI_STUB_H

#include <stddef.h>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Win;
typedef int MPI_Group;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_DATATYPE_NULL 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_FLOAT 3
#define MPI_LONG 4
#define MPI_CXX_BOOL 5
#define MPI_CHAR 6
#define MPI_UNSIGNED 7
#define MPI_BYTE 8
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *, MPI_Datatype *t) { *t = 100; return MPI_SUCCESS; }
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype *t) { *t = 101; return MPI_SUCCESS; }
static inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint, MPI_Datatype *t) { *t = 102; return MPI_SUCCESS; }
static inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { *t = 0; return MPI_SUCCESS; }
static inline int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm *c) { *c = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *f) { *f = 1; return MPI_SUCCESS; }

#endif
