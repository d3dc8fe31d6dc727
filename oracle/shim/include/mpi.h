/*
 * In-process MPI test double used ONLY to compile and run the reference's own
 * layout and 2.5D Cannon sources on the CPU (the oracle's "reference" arm).
 * Every virtual rank is a host thread; point-to-point messages are packed
 * eagerly into a shared mailbox.  Only the subset of MPI the reference's hot-path
 * files call is provided:
 *   src/Decompositions/pblasDecomposition.cpp, src/Decompositions/2DBlockSequentialDecomposition.cpp,
 *   src/Transfers/mpiTransfers.cpp, src/25DCannon.cpp.
 * This is test infrastructure; nothing in the product links it.
 */
#ifndef ORACLE_FAKE_MPI_H
#define ORACLE_FAKE_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fake_comm_s* MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct fake_request_s* MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_UNDEFINED (-32766)

/* predefined datatypes: value = element size class */
#define MPI_BYTE   1
#define MPI_INT    2
#define MPI_FLOAT  3
#define MPI_DOUBLE 4
#define MPI_LONG_LONG 5

#define MPI_SUM 1

extern MPI_Comm fake_mpi_comm_world(void);
#define MPI_COMM_WORLD (fake_mpi_comm_world())

int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Isendrecv_replace(void* buf, int count, MPI_Datatype type, int dest, int sendtag, int source, int recvtag,
                          MPI_Comm comm, MPI_Request* req);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void* recvbuf,
                 int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status* status);
int MPI_Waitany(int count, MPI_Request* reqs, int* index, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);
int MPI_Ibcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request* req);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif

#endif
