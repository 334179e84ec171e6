/*
 * Single-rank stand-in for <mpi.h>, written for this project.
 *
 * It lets the hpcscan sources (src/*.cpp of the reference, compiled
 * unchanged from where they lie) build and run as ONE process without an MPI
 * installation: in the B200 test-mode binary (hpcscan_b200/host), and in the
 * reference CPU build that the tests use as oracle and CPU baseline.
 *
 * Semantics for a world of size 1:
 *  - every neighbour is MPI_PROC_NULL (the reference computes that itself
 *    when -nsub1/2/3 are 1), so point-to-point calls are no-ops;
 *  - Reduce / Allreduce / Gather / Gatherv copy the send buffer to the
 *    receive buffer (identity reduction over one rank);
 *  - derived datatypes are opaque handles that are never dereferenced;
 *  - MPI-IO (used only by Grid::writeGlobal for snapshots) opens nothing and
 *    writes nothing.
 */
#ifndef HPCSCAN_B200_MPI_STUB_H_
#define HPCSCAN_B200_MPI_STUB_H_

#include <string.h>
#include <stdlib.h>
#include <sys/time.h>
#include <time.h>

#ifdef __cplusplus
extern "C++" {
#endif

typedef int MPI_Comm;
typedef long MPI_Aint;
typedef long MPI_Offset;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef int MPI_Errhandler;
/* A datatype handle encodes the element size in bytes for the basic types;
 * derived types get a distinct negative handle and are never used for
 * copies. */
typedef long MPI_Datatype;

typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_DATATYPE_NULL 0L
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_APPEND 128
#define MPI_INFO_NULL 0
#define MPI_ERRORS_ARE_FATAL 1
#define MPI_ERRORS_RETURN 2

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_CHAR        1L
#define MPI_BYTE        1L
#define MPI_REAL16      2L
#define MPI_INT         4L
#define MPI_FLOAT       1004L
#define MPI_LONG        8L
#define MPI_LONG_LONG   1008L
#define MPI_DOUBLE      2008L

static inline size_t hpcscan_stub_type_size(MPI_Datatype t)
{
	return (t > 0) ? (size_t)(t % 1000) : 0 ;
}

static inline double MPI_Wtime(void)
{
	struct timespec ts ;
	clock_gettime(CLOCK_MONOTONIC, &ts) ;
	return (double)ts.tv_sec + 1.0e-9 * (double)ts.tv_nsec ;
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS ; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS ; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code) ; return MPI_SUCCESS ; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1 ; return MPI_SUCCESS ; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0 ; return MPI_SUCCESS ; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS ; }

static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
	if (s != r && n > 0) memcpy(r, s, (size_t)n * hpcscan_stub_type_size(t)) ;
	return MPI_SUCCESS ;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
	if (s != r && n > 0) memcpy(r, s, (size_t)n * hpcscan_stub_type_size(t)) ;
	return MPI_SUCCESS ;
}
static inline int MPI_Gather(const void* s, int ns, MPI_Datatype ts, void* r, int, MPI_Datatype, int, MPI_Comm)
{
	if (s != r && ns > 0) memcpy(r, s, (size_t)ns * hpcscan_stub_type_size(ts)) ;
	return MPI_SUCCESS ;
}
static inline int MPI_Gatherv(const void* s, int ns, MPI_Datatype ts, void* r, const int*, const int* displs,
		MPI_Datatype tr, int, MPI_Comm)
{
	if (ns > 0) memcpy((char*)r + (size_t)displs[0] * hpcscan_stub_type_size(tr), s,
			(size_t)ns * hpcscan_stub_type_size(ts)) ;
	return MPI_SUCCESS ;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS ; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS ; }
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int,
		MPI_Comm, MPI_Status*) { return MPI_SUCCESS ; }

static inline MPI_Datatype hpcscan_stub_new_type(void)
{
	static long counter = -1 ;
	return counter-- ;
}
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype* t) { *t = hpcscan_stub_new_type() ; return MPI_SUCCESS ; }
static inline int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype* t) { *t = hpcscan_stub_new_type() ; return MPI_SUCCESS ; }
static inline int MPI_Type_create_hvector(int, int, MPI_Aint, MPI_Datatype, MPI_Datatype* t) { *t = hpcscan_stub_new_type() ; return MPI_SUCCESS ; }
static inline int MPI_Type_create_subarray(int, const int*, const int*, const int*, int, MPI_Datatype, MPI_Datatype* t)
{ *t = hpcscan_stub_new_type() ; return MPI_SUCCESS ; }
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS ; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS ; }

static inline int MPI_Info_create(MPI_Info* i) { *i = 0 ; return MPI_SUCCESS ; }
static inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File* f) { *f = 0 ; return MPI_SUCCESS ; }
static inline int MPI_File_set_errhandler(MPI_File, MPI_Errhandler) { return MPI_SUCCESS ; }
static inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) { return MPI_SUCCESS ; }
static inline int MPI_File_write_all(MPI_File, const void*, int, MPI_Datatype, MPI_Status*) { return MPI_SUCCESS ; }
static inline int MPI_File_close(MPI_File*) { return MPI_SUCCESS ; }

#ifdef __cplusplus
}
#endif

#endif
