/*
 * mpi.h -- minimal MPI subset so that the reference's own src/src_c/decomp_2d.c
 * and src/src_c/mod_poisson_solver.c compile unmodified for the CPU oracle.
 * TEST INFRASTRUCTURE ONLY.
 *
 * Ranks are either the calling process alone (size 1) or processes forked by
 * oracle_mpi_run() that exchange messages through shared memory
 * (shim/mpi_shim.c).  Only the calls the two reference files make are
 * provided: Comm_rank/size, Cart_create/coords/sub/shift/rank, Comm_c2f,
 * Comm_free, Abort, Sendrecv, Alltoallv, Barrier.  Communicator handles are
 * small integers; MPI_PROC_NULL is a negative sentinel.
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Fint;
typedef int MPI_Datatype;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_DOUBLE 8
#define MPI_FLOAT 4
#define MPI_INT 5
#define MPI_BYTE 1

int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *comm_cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank);
int MPI_Cart_sub(MPI_Comm comm, const int remain_dims[], MPI_Comm *newcomm);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *rank_source, int *rank_dest);
MPI_Fint MPI_Comm_c2f(MPI_Comm comm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Abort(MPI_Comm comm, int errorcode);
int MPI_Barrier(MPI_Comm comm);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void *recvbuf, const int recvcounts[], const int rdispls[],
                  MPI_Datatype recvtype, MPI_Comm comm);

/* ---- oracle harness (not MPI) ---------------------------------------- */
/* Run fn(rank, arg) on nprocs ranks.  nprocs == 1 runs in the calling
 * process; otherwise nprocs children are forked (call this from a fresh
 * process, before any GPU or threading runtime is initialised) and the
 * call returns 0 when every child exited 0.  max_msg_bytes bounds one
 * point-to-point message or one Alltoallv block. */
int oracle_mpi_run(int nprocs, long max_msg_bytes, int (*fn)(int rank, void *arg), void *arg);

#ifdef __cplusplus
}
#endif

#endif
