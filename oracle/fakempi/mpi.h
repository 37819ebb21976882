/* The subset of MPI that the reference's CC sources call, for compiling them
 * unmodified on a host without an MPI installation.  TEST INFRASTRUCTURE
 * ONLY: it builds the checker in oracle/_ref, never the product.
 *
 * Ranks are processes that MPI_Init forks (FAKEMPI_NP of them, default 1);
 * see fakempi.c for the transport.  Handles are plain ints. */
#ifndef FAKEMPI_MPI_H
#define FAKEMPI_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;

typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    size_t count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_UNWEIGHTED ((int *)2)
#define MPI_WEIGHTS_EMPTY ((int *)3)

/* datatype = (kind << 8) | size in bytes; kind 1 signed, 2 unsigned,
 * 3 floating point, 4 bytes */
#define MPI_CHAR 0x101
#define MPI_SIGNED_CHAR 0x101
#define MPI_BYTE 0x401
#define MPI_UNSIGNED_CHAR 0x201
#define MPI_SHORT 0x102
#define MPI_UNSIGNED_SHORT 0x202
#define MPI_INT 0x104
#define MPI_UNSIGNED 0x204
#define MPI_LONG 0x108
#define MPI_UNSIGNED_LONG 0x208
#define MPI_LONG_LONG 0x108
#define MPI_LONG_LONG_INT 0x108
#define MPI_UNSIGNED_LONG_LONG 0x208
#define MPI_INT32_T 0x104
#define MPI_INT64_T 0x108
#define MPI_UINT8_T 0x201
#define MPI_UINT32_T 0x204
#define MPI_UINT64_T 0x208
#define MPI_FLOAT 0x304
#define MPI_DOUBLE 0x308

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5
#define MPI_BOR 6

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Abort(MPI_Comm comm, int errorcode);
double MPI_Wtime(void);

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status);

int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                  MPI_Datatype sendtype, void *recvbuf, const int *recvcounts,
                  const int *rdispls, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int *sendcounts, const int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int root, MPI_Comm comm);

int MPI_Dist_graph_create_adjacent(MPI_Comm comm_old, int indegree, const int sources[],
                                   const int sourceweights[], int outdegree,
                                   const int destinations[], const int destweights[],
                                   MPI_Info info, int reorder, MPI_Comm *comm_dist_graph);
int MPI_Neighbor_alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                          void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Neighbor_alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                           MPI_Datatype sendtype, void *recvbuf, const int recvcounts[],
                           const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Ineighbor_alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                            MPI_Datatype sendtype, void *recvbuf, const int recvcounts[],
                            const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm,
                            MPI_Request *request);
int MPI_Wait(MPI_Request *request, MPI_Status *status);
int MPI_Comm_free(MPI_Comm *comm);

#ifdef __cplusplus
}
#endif

#endif /* FAKEMPI_MPI_H */
