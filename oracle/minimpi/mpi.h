/* Checker infrastructure: the MPI calls the reference TeaLeaf host makes
 * (2d/comms.c, 3d/comms.c), implemented over Unix-domain sockets between
 * processes on one host, so the unmodified reference can run as N ranks here
 * and give multi-rank known answers. Not a general MPI: one communicator,
 * doubles only, Allreduce folding the ranks' values in rank order at rank 0.
 *
 * A launcher starts N processes with MINIMPI_RANK, MINIMPI_SIZE and
 * MINIMPI_DIR (a directory for the sockets) in their environment.
 */
#pragma once

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct MiniRequest* MPI_Request;
typedef struct {
    int unused;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Barrier(MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request* request);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
              MPI_Request* request);
int MPI_Waitall(int count, MPI_Request* requests, MPI_Status* statuses);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
