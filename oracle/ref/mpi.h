/* Single-process stand-in for the subset of MPI that the reference solver's
 * sources use, so that its own translation units build and run as one rank on
 * one GPU without an MPI installation.  Test infrastructure: it exists only to
 * build the reference as a checker under oracle/_ref/.
 *
 * World size is 1 and rank 0.  Collectives copy the send buffer to the receive
 * buffer; point-to-point calls abort (a single-block, non-parallel run never
 * reaches them).  MPI-IO is plain POSIX file access with a byte view; a
 * datatype is a basic type, a contiguous run of a type, or a FORTRAN/C-order
 * subarray of a type, flattened to (offset, length) blocks when it is used. */
#ifndef ORACLE_REF_MPI_H
#define ORACLE_REF_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef long long MPI_Aint;
typedef struct mpi_shim_file *MPI_File;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_SELF ((MPI_Comm)1)
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_FILE_NULL ((MPI_File)0)

/* basic datatypes: the handle is an index into the shim's type table */
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_INT32_T ((MPI_Datatype)4)
#define MPI_INT64_T ((MPI_Datatype)5)
#define MPI_FLOAT ((MPI_Datatype)6)
#define MPI_REAL ((MPI_Datatype)7)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_OFFSET ((MPI_Datatype)9)
#define MPI_LONG_LONG ((MPI_Datatype)10)
#define MPI_UNSIGNED ((MPI_Datatype)11)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)

#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57

#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_EXCL 64
#define MPI_MODE_APPEND 128

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount, MPI_Datatype rtype,
               int root, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, const int *rcounts,
                const int *displs, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, const int *rcounts,
                   const int *displs, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Scatter(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount, MPI_Datatype rtype,
                int root, MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int *scounts, const int *displs, MPI_Datatype stype, void *recvbuf,
                 int rcount, MPI_Datatype rtype, int root, MPI_Comm comm);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[], int order,
                             MPI_Datatype old, MPI_Datatype *out);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype type, MPI_Status *status);
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Status *status);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type, MPI_Status *status);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void *buf, int count, MPI_Datatype type,
                      MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
