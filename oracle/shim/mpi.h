/*
 * Single-rank stand-in for the MPI subset that GAMERA-OP's solver uses.
 *
 * Test infrastructure only: it lets the reference C sources compile and run
 * unmodified as the CPU oracle on a machine with no MPI installation.  It is
 * never linked into the product library.
 *
 * Semantics (one process, rank 0 of 1):
 *   - MPI_Cart_create records per-axis periodicity; MPI_Cart_shift returns
 *     rank 0 (self) on a periodic axis and MPI_PROC_NULL otherwise, which is
 *     what a 1x1x1 Cartesian communicator gives (src/setup_mpi.c:28-59).
 *   - Derived datatypes (vector / indexed over MPI_DOUBLE) are stored as
 *     block lists; MPI_Sendrecv to self packs the send layout and unpacks it
 *     into the receive layout, exactly the copy a real MPI performs
 *     (src/boundary_exchange.c:7-165).
 *   - MPI_Allreduce with one rank is the identity (src/solver_solve.c:97,105).
 *   - MPI_Send / MPI_Recv are only used by the pole ring average, which the
 *     oracle never enables; they report an error.
 *   - The wall-clock time of each MPI_Allreduce call is recorded so a driver
 *     can time the step loop without touching the solver sources.
 */
#ifndef GOP_SHIM_MPI_H
#define GOP_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef struct gop_mpi_type *MPI_Datatype;
typedef int MPI_Op;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

extern struct gop_mpi_type gop_mpi_double_type;
extern struct gop_mpi_type gop_mpi_int_type;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_DOUBLE (&gop_mpi_double_type)
#define MPI_INT (&gop_mpi_int_type)
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[],
                    const int periods[], int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source,
                   int *dest);
int MPI_Type_vector(int count, int blocklength, int stride,
                    MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_indexed(int count, const int blocklengths[],
                     const int displacements[], MPI_Datatype oldtype,
                     MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status);

/* Timing hook: wall-clock seconds (CLOCK_MONOTONIC) of the n-th
 * MPI_Allreduce call, and the number of calls so far. */
double gop_shim_allreduce_time(int n);
int gop_shim_allreduce_count(void);

#ifdef __cplusplus
}
#endif
#endif
