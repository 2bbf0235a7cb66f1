/*
 * Single-rank MPI stand-in used only to build the reference ParGeMSLR CPU
 * solver as the test oracle (test infrastructure, never shipped).
 *
 * The reference calls MPI even when it runs on one rank: dot products
 * all-reduce (SRC/vectors/vectorops.cpp:180-482) and the level permutations
 * travel as self-addressed Isend/Irecv pairs
 * (SRC/matrices/parallel_csr_matrix.cpp:571-983).  This header declares the
 * subset of the MPI-3 C interface the reference uses; mpi_single.cpp gives a
 * world of exactly one process in which collectives copy send buffers to
 * receive buffers and point-to-point messages are matched by (comm, tag) in
 * FIFO order.
 */
#ifndef PGX_ORACLE_MPI_SINGLE_H
#define PGX_ORACLE_MPI_SINGLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

typedef struct {
   int MPI_SOURCE;
   int MPI_TAG;
   int MPI_ERROR;
   int count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

/* datatypes: the value encodes (kind << 8) | size_in_bytes */
#define MPI_DATATYPE_NULL    ((MPI_Datatype)0)
#define MPI_CHAR             ((MPI_Datatype)((1 << 8) | 1))
#define MPI_INT              ((MPI_Datatype)((2 << 8) | 4))
#define MPI_LONG             ((MPI_Datatype)((3 << 8) | 8))
#define MPI_FLOAT            ((MPI_Datatype)((4 << 8) | 4))
#define MPI_DOUBLE           ((MPI_Datatype)((5 << 8) | 8))
#define MPI_C_FLOAT_COMPLEX  ((MPI_Datatype)((6 << 8) | 8))
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)((7 << 8) | 16))
#define MPI_LONG_LONG        ((MPI_Datatype)((8 << 8) | 8))
#define MPI_UNSIGNED         ((MPI_Datatype)((9 << 8) | 4))
#define MPI_BYTE             ((MPI_Datatype)((10 << 8) | 1))

#define MPI_SUM  ((MPI_Op)1)
#define MPI_MAX  ((MPI_Op)2)
#define MPI_MIN  ((MPI_Op)3)
#define MPI_PROD ((MPI_Op)4)

#define MPI_IN_PLACE ((void *)-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);
int MPI_Scan(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, const int *rcounts, const int *displs, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt, int root, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int rcount, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype sdt, void *recvbuf, const int *rcounts, const int *rdispls, MPI_Datatype rdt, MPI_Comm comm);

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype sdt, int dest, int stag, void *recvbuf, int rcount, MPI_Datatype rdt, int source, int rtag, MPI_Comm comm, MPI_Status *status);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Waitany(int count, MPI_Request *reqs, int *index, MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
