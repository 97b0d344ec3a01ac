/*
 * mpi.h -- single-rank MPI for builds of SHAFFT's single-GPU backend on a
 * machine without an MPI installation.
 *
 * The SHAFFT API carries an MPI_Comm in its signatures and calls a small set
 * of MPI routines at set-up time (configuration, communicator dup/split,
 * barriers).  With one process those calls have trivial answers; this header
 * declares exactly that set with single-rank semantics (rank 0 of size 1,
 * collectives are copies).  Put include/mpi_shim on the include path and link
 * libshafft_mpishim.so only when no real MPI is present; with a real MPI the
 * library is built against it and this directory is not used.
 */
#ifndef SHAFFT_MPI_SHIM_H
#define SHAFFT_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHAFFT_MPI_SHIM 1

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Fint;

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#define MPI_COMM_SELF ((MPI_Comm)0x44000001)

#define MPI_SUCCESS 0
#define MPI_ERR_COMM 5
#define MPI_ERR_ARG 12
#define MPI_ERR_OTHER 16
#define MPI_UNDEFINED (-32766)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 512
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL ((MPI_Info)0x1c000000)
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR ((MPI_Datatype)0x4c000101)
#define MPI_INT ((MPI_Datatype)0x4c000405)
#define MPI_LONG ((MPI_Datatype)0x4c000807)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)0x4c000808)
#define MPI_FLOAT ((MPI_Datatype)0x4c00040a)
#define MPI_DOUBLE ((MPI_Datatype)0x4c00080b)
#define MPI_C_BOOL ((MPI_Datatype)0x4c00013f)
#define MPI_C_COMPLEX ((MPI_Datatype)0x4c000840)
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)0x4c001041)

#define MPI_LAND ((MPI_Op)0x58000005)
#define MPI_LOR ((MPI_Op)0x58000007)
#define MPI_MAX ((MPI_Op)0x58000001)
#define MPI_MIN ((MPI_Op)0x58000002)
#define MPI_SUM ((MPI_Op)0x58000003)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
int MPI_Abort(MPI_Comm comm, int errorcode);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key, MPI_Info info, MPI_Comm* newcomm);
MPI_Fint MPI_Comm_c2f(MPI_Comm comm);
MPI_Comm MPI_Comm_f2c(MPI_Fint comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
                  MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Get_processor_name(char* name, int* resultlen);
int MPI_Error_string(int errorcode, char* string, int* resultlen);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Type_size(MPI_Datatype datatype, int* size);

#ifdef __cplusplus
}
#endif

#endif /* SHAFFT_MPI_SHIM_H */
