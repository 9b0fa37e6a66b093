/*
 * In-process thread-rank stand-in for MPI.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference (an MPI program) is compiled against this header so that it runs here, where no
 * MPI library is installed: every rank is a thread of one process (launcher in mpi_shim.cpp).
 * It provides exactly the MPI entry points and constants the reference uses; messages are
 * buffered (sends never block), collectives reduce in rank order (deterministic).
 */
#ifndef S2L_MPI_SHIM_H
#define S2L_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct s2l_mpi_comm* MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct s2l_mpi_request* MPI_Request;
typedef int MPI_Fint;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

MPI_Comm s2l_mpi_comm_world(void);

#define MPI_COMM_WORLD (s2l_mpi_comm_world())
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

enum {
    MPI_CHAR = 1,
    MPI_INT,
    MPI_LONG,
    MPI_LONG_LONG,
    MPI_UNSIGNED,
    MPI_UNSIGNED_LONG,
    MPI_UNSIGNED_LONG_LONG,
    MPI_DOUBLE,
    MPI_FLOAT,
    MPI_INT64_T,
    MPI_INT32_T,
    MPI_UINT64_T,
    MPI_BYTE
};
#define MPI_LONG_LONG_INT MPI_LONG_LONG
enum { MPI_SUM = 1, MPI_MAX, MPI_MIN };

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
MPI_Fint MPI_Comm_c2f(MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Reduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt, int root,
               MPI_Comm comm);
int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, const int* rcounts, const int* displs,
                MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Scatterv(const void* sbuf, const int* scounts, const int* displs, MPI_Datatype st, void* rbuf, int rcount,
                 MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Allgather(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, const int* rcounts, const int* displs,
                   MPI_Datatype rt, MPI_Comm comm);
int MPI_Alltoall(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype st, void* rbuf,
                  const int* rcounts, const int* rdispls, MPI_Datatype rt, MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);

#ifdef __cplusplus
}
#endif

#endif
