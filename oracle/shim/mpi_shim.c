/* Single-rank MPI stand-in used only to build the reference as the CPU
 * oracle.  See mpi.h for the semantics it provides. */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

struct gop_mpi_type {
  int nblocks;     /* number of (displacement, length) blocks */
  long *disp;      /* displacement of each block, in base elements */
  long *len;       /* length of each block, in base elements */
  size_t elem;     /* size of the base element in bytes */
  int builtin;     /* 1 for MPI_DOUBLE / MPI_INT */
};

static long gop_one_disp = 0, gop_one_len = 1;
struct gop_mpi_type gop_mpi_double_type = {1, &gop_one_disp, &gop_one_len,
                                           sizeof(double), 1};
struct gop_mpi_type gop_mpi_int_type = {1, &gop_one_disp, &gop_one_len,
                                        sizeof(int), 1};

static int g_periods[3] = {0, 0, 0};
static int g_ndims = 0;

#define GOP_MAX_TIMES 1000000
static double *g_times = NULL;
static int g_ntimes = 0;

static double now_seconds(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) {
  /* GOP_SHIM_TIMING=1: report the MPI_Allreduce timestamps.  Call 0 is the
   * initial dt (src/solver_solve.c:97), call n >= 1 opens step n
   * (src/solver_solve.c:105), so calls 1..last bracket last-1 whole steps. */
  const char *e = getenv("GOP_SHIM_TIMING");
  if (e && (e[0] == '1' || e[0] == '2') && g_ntimes >= 3) {
    fprintf(stderr, "GOP_SHIM_TIMING calls=%d t1=%.9f tlast=%.9f\n", g_ntimes,
            g_times[1], g_times[g_ntimes - 1]);
  }
  /* GOP_SHIM_TIMING=2 also lists every timestamp (per-step durations) */
  if (e && e[0] == '2') {
    fprintf(stderr, "GOP_SHIM_TIMES");
    for (int n = 0; n < g_ntimes; n++) fprintf(stderr, " %.9f", g_times[n]);
    fprintf(stderr, "\n");
  }
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  (void)comm;
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
  (void)comm;
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm *comm) {
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[],
                    const int periods[], int reorder, MPI_Comm *cart) {
  (void)old;
  (void)reorder;
  if (ndims > 3) return MPI_ERR_OTHER;
  for (int d = 0; d < ndims; d++) {
    if (dims[d] != 1) {
      fprintf(stderr, "mpi shim: only a 1x1x1 process grid is supported\n");
      return MPI_ERR_OTHER;
    }
    g_periods[d] = periods[d] ? 1 : 0;
  }
  g_ndims = ndims;
  *cart = 2;
  return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]) {
  (void)comm;
  (void)rank;
  for (int d = 0; d < maxdims; d++) coords[d] = 0;
  return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank) {
  (void)comm;
  for (int d = 0; d < g_ndims; d++) {
    if (coords[d] != 0 && !g_periods[d]) return MPI_ERR_OTHER;
  }
  *rank = 0;
  return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source,
                   int *dest) {
  (void)comm;
  (void)disp;
  int self = g_periods[direction] ? 0 : MPI_PROC_NULL;
  *source = self;
  *dest = self;
  return MPI_SUCCESS;
}

static MPI_Datatype new_type(int nblocks, size_t elem) {
  MPI_Datatype t = (MPI_Datatype)calloc(1, sizeof(struct gop_mpi_type));
  t->nblocks = nblocks;
  t->disp = (long *)malloc(sizeof(long) * (size_t)(nblocks > 0 ? nblocks : 1));
  t->len = (long *)malloc(sizeof(long) * (size_t)(nblocks > 0 ? nblocks : 1));
  t->elem = elem;
  t->builtin = 0;
  return t;
}

int MPI_Type_vector(int count, int blocklength, int stride,
                    MPI_Datatype oldtype, MPI_Datatype *newtype) {
  if (!oldtype->builtin) return MPI_ERR_OTHER;
  MPI_Datatype t = new_type(count, oldtype->elem);
  for (int b = 0; b < count; b++) {
    t->disp[b] = (long)b * stride;
    t->len[b] = blocklength;
  }
  *newtype = t;
  return MPI_SUCCESS;
}

int MPI_Type_indexed(int count, const int blocklengths[],
                     const int displacements[], MPI_Datatype oldtype,
                     MPI_Datatype *newtype) {
  if (!oldtype->builtin) return MPI_ERR_OTHER;
  MPI_Datatype t = new_type(count, oldtype->elem);
  for (int b = 0; b < count; b++) {
    t->disp[b] = displacements[b];
    t->len[b] = blocklengths[b];
  }
  *newtype = t;
  return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type) {
  (void)type;
  return MPI_SUCCESS;
}

int MPI_Type_free(MPI_Datatype *type) {
  if (type && *type && !(*type)->builtin) {
    free((*type)->disp);
    free((*type)->len);
    free(*type);
  }
  if (type) *type = NULL;
  return MPI_SUCCESS;
}

static long type_size(MPI_Datatype t) {
  long n = 0;
  for (int b = 0; b < t->nblocks; b++) n += t->len[b];
  return n;
}

/* Message passing to self: pack the send layout into a contiguous buffer,
 * then unpack it into the receive layout.  Packing first makes overlapping
 * send/receive regions behave like a real (buffered) exchange. */
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
  (void)sendtag;
  (void)recvtag;
  (void)comm;
  (void)status;
  if (dest == MPI_PROC_NULL && source == MPI_PROC_NULL) return MPI_SUCCESS;
  if (dest != 0 || source != 0) return MPI_ERR_OTHER;
  long nsend = type_size(sendtype) * sendcount;
  long nrecv = type_size(recvtype) * recvcount;
  if (nsend != nrecv || sendtype->elem != recvtype->elem) return MPI_ERR_OTHER;
  size_t es = sendtype->elem;
  char *tmp = (char *)malloc((size_t)nsend * es + 1);
  if (!tmp) return MPI_ERR_OTHER;
  /* the extent of a derived type is not needed: every call uses count 1 */
  long pos = 0;
  for (int c = 0; c < sendcount; c++) {
    for (int b = 0; b < sendtype->nblocks; b++) {
      memcpy(tmp + (size_t)pos * es,
             (const char *)sendbuf + (size_t)sendtype->disp[b] * es,
             (size_t)sendtype->len[b] * es);
      pos += sendtype->len[b];
    }
  }
  pos = 0;
  for (int c = 0; c < recvcount; c++) {
    for (int b = 0; b < recvtype->nblocks; b++) {
      memcpy((char *)recvbuf + (size_t)recvtype->disp[b] * es,
             tmp + (size_t)pos * es, (size_t)recvtype->len[b] * es);
      pos += recvtype->len[b];
    }
  }
  free(tmp);
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm) {
  (void)op;
  (void)comm;
  if (!g_times) g_times = (double *)malloc(sizeof(double) * GOP_MAX_TIMES);
  if (g_times && g_ntimes < GOP_MAX_TIMES) g_times[g_ntimes++] = now_seconds();
  if (sendbuf != recvbuf)
    memcpy(recvbuf, sendbuf, (size_t)count * datatype->elem);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm) {
  (void)buf;
  (void)count;
  (void)datatype;
  (void)dest;
  (void)tag;
  (void)comm;
  fprintf(stderr, "mpi shim: MPI_Send is not supported (ring average)\n");
  return MPI_ERR_OTHER;
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
  (void)buf;
  (void)count;
  (void)datatype;
  (void)source;
  (void)tag;
  (void)comm;
  (void)status;
  fprintf(stderr, "mpi shim: MPI_Recv is not supported (ring average)\n");
  return MPI_ERR_OTHER;
}

double gop_shim_allreduce_time(int n) {
  if (n < 0 || n >= g_ntimes) return -1.0;
  return g_times[n];
}
int gop_shim_allreduce_count(void) { return g_ntimes; }
