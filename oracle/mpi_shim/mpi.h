/*
 * Single-rank MPI shim — TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * The reference solver (DNS-solver-with-grid-embedding/src/*.c) is C99 + MPI.
 * This container has no MPI, so the oracle compiles the reference's own sources
 * unmodified against this header.  It implements exactly the MPI surface those
 * sources use (symbols found by grep over src/*.c), for ONE rank in a periodic
 * 1x1 Cartesian topology (XDIM = YDIM = 1):
 *
 *   - every neighbour is rank 0, so point-to-point traffic is a self-exchange:
 *     persistent requests are matched per tag in posting order (MPI's
 *     non-overtaking rule), MPI_Sendrecv packs with the send type and unpacks
 *     with the receive type;
 *   - derived datatypes (contiguous, 2-D/3-D C-order subarray) are flattened by
 *     recursive pack/unpack;
 *   - MPI-IO maps onto stdio with the file view's filetype tiling the file;
 *   - collectives are identities (one rank).
 *
 * Nothing under the product package links this shim.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Errhandler;
typedef long long MPI_Offset;

typedef struct shim_type {
  int kind;                 /* 0 basic, 1 contiguous, 2 subarray */
  size_t size;              /* bytes of data described */
  size_t extent;            /* bytes spanned (lower bound is always 0) */
  int count;                /* contiguous: repetitions of base */
  struct shim_type *base;   /* contiguous / subarray element type */
  int ndims;                /* subarray */
  int sizes[4], subsizes[4], starts[4];
  int committed;
} shim_type;
typedef shim_type *MPI_Datatype;

typedef struct {
  long long count_bytes;
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

typedef struct shim_req *MPI_Request;
typedef struct shim_file *MPI_File;

extern shim_type shim_type_double, shim_type_int, shim_type_char;
#define MPI_DOUBLE (&shim_type_double)
#define MPI_INT (&shim_type_int)
#define MPI_CHAR (&shim_type_char)

#define MPI_COMM_WORLD 0
#define MPI_SUM 1
#define MPI_ORDER_C 56
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_INFO_NULL 0
#define MPI_ERRORS_RETURN 0
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 256
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_REQUEST_NULL ((MPI_Request)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Barrier(MPI_Comm comm);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler h);
int MPI_Get_processor_name(char *name, int *len);
double MPI_Wtime(void);
int MPI_Error_class(int code, int *cls);
int MPI_Error_string(int code, char *str, int *len);

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_create_subarray(int ndims, const int *sizes, const int *subsizes,
                             const int *starts, int order, MPI_Datatype old,
                             MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);

int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag,
                  MPI_Comm comm, MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int source, int tag,
                  MPI_Comm comm, MPI_Request *req);
int MPI_Startall(int n, MPI_Request *reqs);
int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *st);
int MPI_Request_free(MPI_Request *req);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int source, int rtag,
                 MPI_Comm comm, MPI_Status *st);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op,
                  MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);

int MPI_Info_create(MPI_Info *info);
int MPI_Info_set(MPI_Info info, const char *key, const char *value);
int MPI_Info_free(MPI_Info *info);

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype,
                      MPI_Datatype filetype, const char *rep, MPI_Info info);
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_read_at_all(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t,
                       MPI_Status *st);
int MPI_File_close(MPI_File *fh);

#ifdef __cplusplus
}
#endif
#endif
