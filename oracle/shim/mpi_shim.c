/* MPI stand-in used only to build the reference as the CPU oracle and the
 * timed CPU baseline.  See mpi.h for the semantics it provides.
 *
 * One rank by default.  With GOP_SHIM_RANKS=N (N > 1) MPI_Init forks N-1
 * children, so the reference runs as N processes of one thread each, the
 * mode its README uses (mpirun -n N, OMP_NUM_THREADS=1); the ranks talk
 * through one shared anonymous memory mapping made before the fork:
 *   - a mailbox per ordered rank pair: a data slot of GOP_SHIM_SLOT_MB
 *     megabytes (default 16) with "sent" and "taken" chunk counters.  A
 *     message is packed by its datatype, cut into slot-sized chunks, and
 *     the sender and the receiver of MPI_Sendrecv move chunks both ways in
 *     one loop, so exchanges of any size between any pair cannot deadlock;
 *     messages between two ranks arrive in the order sent (tags unchecked);
 *   - a sense-reversing barrier on one shared counter;
 *   - MPI_Allreduce: every rank posts its values, the barrier, then every
 *     rank folds the posts in rank order 0..N-1 (the same bits everywhere),
 *     and a second barrier frees the posts.
 * Every wait spins on the shared counters and gives up after
 * GOP_SHIM_TIMEOUT seconds (default 3600), or at once when another rank has
 * failed: the process then exits with status 5.  Children die with their
 * parent (PR_SET_PDEATHSIG); rank 0's MPI_Finalize waits for every child
 * and exits with status 6 if one of them failed. */
#define _GNU_SOURCE
#include "mpi.h"

#include <sched.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

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

#define MAX_RANKS 64
#define MAX_RED 16

struct mbox {
  long sent;   /* chunks written by the sender */
  long taken;  /* chunks read by the receiver */
  long bytes;  /* bytes in the current chunk */
  char pad[40];
};

struct ctl {
  int count;   /* barrier arrivals */
  int gen;     /* barrier generation */
  int failed;  /* nonzero once a rank gave up */
  int pad;
  double red[MAX_RANKS][MAX_RED];
  struct mbox box[MAX_RANKS][MAX_RANKS];
};

static int g_rank = 0, g_size = 1;
static struct ctl *g_ctl = NULL;
static char *g_slots = NULL;
static size_t g_slot = 0;
static pid_t g_child[MAX_RANKS];
static double g_timeout = 3600.0;

static int g_dims[3] = {1, 1, 1};
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

static void give_up(const char *what) {
  if (g_ctl) __atomic_store_n(&g_ctl->failed, 1, __ATOMIC_RELEASE);
  fprintf(stderr, "mpi shim: rank %d gave up waiting in %s\n", g_rank, what);
  _exit(5);
}

/* spins until *p (read with acquire) satisfies cmp(*p, v) */
#define WAIT_UNTIL(cond, what)                                             \
  do {                                                                     \
    double t0_ = -1.0;                                                     \
    for (long it_ = 0; !(cond); it_++) {                                   \
      if (__atomic_load_n(&g_ctl->failed, __ATOMIC_ACQUIRE)) give_up(what); \
      if (it_ < 256) continue;                                             \
      sched_yield();                                                       \
      if ((it_ & 1023) == 0) {                                             \
        double t_ = now_seconds();                                         \
        if (t0_ < 0.0) t0_ = t_;                                           \
        else if (t_ - t0_ > g_timeout) give_up(what);                      \
      }                                                                    \
    }                                                                      \
  } while (0)

static char *slot_of(int src, int dst) {
  return g_slots + ((size_t)src * (size_t)g_size + (size_t)dst) * g_slot;
}

int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  const char *e = getenv("GOP_SHIM_RANKS");
  int n = e ? atoi(e) : 1;
  if (n <= 1) return MPI_SUCCESS;
  if (n > MAX_RANKS) {
    fprintf(stderr, "mpi shim: at most %d ranks\n", MAX_RANKS);
    return MPI_ERR_OTHER;
  }
  const char *mb = getenv("GOP_SHIM_SLOT_MB");
  g_slot = (size_t)(mb ? atol(mb) : 16) << 20;
  const char *to = getenv("GOP_SHIM_TIMEOUT");
  if (to) g_timeout = atof(to);
  size_t ctl_bytes = (sizeof(struct ctl) + 4095) & ~(size_t)4095;
  size_t bytes = ctl_bytes + (size_t)n * (size_t)n * g_slot;
  void *m = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE,
                 -1, 0);
  if (m == MAP_FAILED) {
    perror("mpi shim: mmap");
    return MPI_ERR_OTHER;
  }
  g_ctl = (struct ctl *)m;
  memset(g_ctl, 0, sizeof(struct ctl));
  g_slots = (char *)m + ctl_bytes;
  g_size = n;
  fflush(NULL);
  const pid_t parent = getpid();
  for (int r = 1; r < n; r++) {
    pid_t p = fork();
    if (p < 0) {
      perror("mpi shim: fork");
      __atomic_store_n(&g_ctl->failed, 1, __ATOMIC_RELEASE);
      return MPI_ERR_OTHER;
    }
    if (p == 0) {
      prctl(PR_SET_PDEATHSIG, SIGKILL);
      if (getppid() != parent) _exit(5);
      g_rank = r;
      return MPI_SUCCESS;
    }
    g_child[r] = p;
  }
  g_rank = 0;
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  if (g_size == 1) return MPI_SUCCESS;
  const int gen = __atomic_load_n(&g_ctl->gen, __ATOMIC_ACQUIRE);
  if (__atomic_add_fetch(&g_ctl->count, 1, __ATOMIC_ACQ_REL) == g_size) {
    __atomic_store_n(&g_ctl->count, 0, __ATOMIC_RELAXED);
    __atomic_store_n(&g_ctl->gen, gen + 1, __ATOMIC_RELEASE);
  } else {
    WAIT_UNTIL(__atomic_load_n(&g_ctl->gen, __ATOMIC_ACQUIRE) != gen, "MPI_Barrier");
  }
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  MPI_Barrier(MPI_COMM_WORLD);
  /* GOP_SHIM_TIMING=1: report the MPI_Allreduce timestamps.  Call 0 is the
   * initial dt (src/solver_solve.c:97), call n >= 1 opens step n
   * (src/solver_solve.c:105), so calls 1..last bracket last-1 whole steps. */
  const char *e = getenv("GOP_SHIM_TIMING");
  if (g_rank == 0 && e && (e[0] == '1' || e[0] == '2') && g_ntimes >= 3) {
    fprintf(stderr, "GOP_SHIM_TIMING calls=%d t1=%.9f tlast=%.9f ranks=%d\n", g_ntimes,
            g_times[1], g_times[g_ntimes - 1], g_size);
  }
  /* GOP_SHIM_TIMING=2 also lists every timestamp (per-step durations) */
  if (g_rank == 0 && e && e[0] == '2') {
    fprintf(stderr, "GOP_SHIM_TIMES");
    for (int n = 0; n < g_ntimes; n++) fprintf(stderr, " %.9f", g_times[n]);
    fprintf(stderr, "\n");
  }
  if (g_size > 1 && g_rank == 0) {
    int bad = 0;
    for (int r = 1; r < g_size; r++) {
      int st = 0;
      if (waitpid(g_child[r], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
    }
    if (bad) {
      fprintf(stderr, "mpi shim: a rank failed\n");
      fflush(NULL);
      _exit(6);
    }
  }
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  (void)comm;
  *rank = g_rank;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
  (void)comm;
  *size = g_size;
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm *comm) {
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}

/* row-major Cartesian ranks (the last axis fastest), as MPI numbers them */
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[],
                    const int periods[], int reorder, MPI_Comm *cart) {
  (void)old;
  (void)reorder;
  if (ndims > 3) return MPI_ERR_OTHER;
  int prod = 1;
  for (int d = 0; d < ndims; d++) {
    g_dims[d] = dims[d];
    g_periods[d] = periods[d] ? 1 : 0;
    prod *= dims[d];
  }
  if (prod != g_size) {
    fprintf(stderr, "mpi shim: process grid of %d ranks, %d running\n", prod, g_size);
    return MPI_ERR_OTHER;
  }
  g_ndims = ndims;
  *cart = 2;
  return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]) {
  (void)comm;
  for (int d = g_ndims - 1; d >= 0; d--) {
    if (d < maxdims) coords[d] = rank % g_dims[d];
    rank /= g_dims[d];
  }
  for (int d = g_ndims; d < maxdims; d++) coords[d] = 0;
  return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank) {
  (void)comm;
  int r = 0;
  for (int d = 0; d < g_ndims; d++) {
    int c = coords[d];
    if (c < 0 || c >= g_dims[d]) {
      if (!g_periods[d]) return MPI_ERR_OTHER;
      c = ((c % g_dims[d]) + g_dims[d]) % g_dims[d];
    }
    r = r * g_dims[d] + c;
  }
  *rank = r;
  return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source,
                   int *dest) {
  int c[3];
  MPI_Cart_coords(comm, g_rank, 3, c);
  for (int s = 0; s < 2; s++) {
    int cc[3] = {c[0], c[1], c[2]};
    cc[direction] += s == 0 ? -disp : disp;
    int r = MPI_PROC_NULL;
    if (MPI_Cart_rank(comm, cc, &r) != MPI_SUCCESS) r = MPI_PROC_NULL;
    if (s == 0) *source = r;
    else *dest = r;
  }
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

/* every call site passes count 1 of a derived type or count n of a builtin;
 * a builtin of count n is one block of n elements */
static size_t pack(const void *buf, int count, MPI_Datatype t, char *out) {
  const size_t es = t->elem;
  if (t->builtin) {
    memcpy(out, buf, (size_t)count * es);
    return (size_t)count * es;
  }
  size_t pos = 0;
  for (int c = 0; c < count; c++)
    for (int b = 0; b < t->nblocks; b++) {
      memcpy(out + pos, (const char *)buf + (size_t)t->disp[b] * es, (size_t)t->len[b] * es);
      pos += (size_t)t->len[b] * es;
    }
  return pos;
}

static void unpack(void *buf, int count, MPI_Datatype t, const char *in) {
  const size_t es = t->elem;
  if (t->builtin) {
    memcpy(buf, in, (size_t)count * es);
    return;
  }
  size_t pos = 0;
  for (int c = 0; c < count; c++)
    for (int b = 0; b < t->nblocks; b++) {
      memcpy((char *)buf + (size_t)t->disp[b] * es, in + pos, (size_t)t->len[b] * es);
      pos += (size_t)t->len[b] * es;
    }
}

static size_t msg_bytes(int count, MPI_Datatype t) {
  return (size_t)(t->builtin ? count : type_size(t) * count) * t->elem;
}

/* moves one packed message to dest and one from source, chunk by chunk in
 * a single loop; either side may be absent (MPI_PROC_NULL) */
static int exchange(const char *out, size_t nout, int dest, char *in, size_t nin, int source) {
  size_t sent = 0, got = 0;
  int send_on = dest != MPI_PROC_NULL, recv_on = source != MPI_PROC_NULL;
  struct mbox *ob = send_on ? &g_ctl->box[g_rank][dest] : NULL;
  struct mbox *ib = recv_on ? &g_ctl->box[source][g_rank] : NULL;
  /* a zero-byte message still moves one (empty) chunk */
  int send_done = !send_on, recv_done = !recv_on;
  double t0 = -1.0;
  for (long it = 0; !(send_done && recv_done); it++) {
    int moved = 0;
    if (!send_done && __atomic_load_n(&ob->taken, __ATOMIC_ACQUIRE) ==
                          __atomic_load_n(&ob->sent, __ATOMIC_RELAXED)) {
      size_t n = nout - sent < g_slot ? nout - sent : g_slot;
      memcpy(slot_of(g_rank, dest), out + sent, n);
      ob->bytes = (long)n;
      __atomic_add_fetch(&ob->sent, 1, __ATOMIC_RELEASE);
      sent += n;
      if (sent >= nout) send_done = 1;
      moved = 1;
    }
    if (!recv_done && __atomic_load_n(&ib->sent, __ATOMIC_ACQUIRE) >
                          __atomic_load_n(&ib->taken, __ATOMIC_RELAXED)) {
      size_t n = (size_t)ib->bytes;
      if (got + n > nin) {
        fprintf(stderr, "mpi shim: rank %d received %zu bytes, expected %zu\n", g_rank,
                got + n, nin);
        give_up("MPI_Sendrecv (size mismatch)");
      }
      memcpy(in + got, slot_of(source, g_rank), n);
      __atomic_add_fetch(&ib->taken, 1, __ATOMIC_RELEASE);
      got += n;
      if (got >= nin) recv_done = 1;
      moved = 1;
    }
    if (moved) {
      t0 = -1.0;
      continue;
    }
    if (__atomic_load_n(&g_ctl->failed, __ATOMIC_ACQUIRE)) give_up("MPI_Sendrecv");
    if (it < 256) continue;
    sched_yield();
    if ((it & 1023) == 0) {
      double t = now_seconds();
      if (t0 < 0.0) t0 = t;
      else if (t - t0 > g_timeout) give_up("MPI_Sendrecv");
    }
  }
  return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                 int dest, int sendtag, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
  (void)sendtag;
  (void)recvtag;
  (void)comm;
  (void)status;
  if (dest == MPI_PROC_NULL && source == MPI_PROC_NULL) return MPI_SUCCESS;
  if (dest != MPI_PROC_NULL && (dest < 0 || dest >= g_size)) return MPI_ERR_OTHER;
  if (source != MPI_PROC_NULL && (source < 0 || source >= g_size)) return MPI_ERR_OTHER;
  size_t nsend = dest != MPI_PROC_NULL ? msg_bytes(sendcount, sendtype) : 0;
  size_t nrecv = source != MPI_PROC_NULL ? msg_bytes(recvcount, recvtype) : 0;
  /* pack first: overlapping send and receive regions behave like a real
   * (buffered) exchange */
  char *out = (char *)malloc(nsend + 1);
  char *in = (char *)malloc(nrecv + 1);
  if (!out || !in) {
    free(out);
    free(in);
    return MPI_ERR_OTHER;
  }
  if (dest != MPI_PROC_NULL) pack(sendbuf, sendcount, sendtype, out);
  if (dest == g_rank && source == g_rank) {
    if (nsend != nrecv) {
      free(out);
      free(in);
      return MPI_ERR_OTHER;
    }
    memcpy(in, out, nsend);
  } else {
    int rc = exchange(out, nsend, dest, in, nrecv, source);
    if (rc != MPI_SUCCESS) {
      free(out);
      free(in);
      return rc;
    }
  }
  if (source != MPI_PROC_NULL) unpack(recvbuf, recvcount, recvtype, in);
  free(out);
  free(in);
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype datatype, MPI_Op op, MPI_Comm comm) {
  (void)comm;
  if (g_size > 1) MPI_Barrier(MPI_COMM_WORLD);  /* the timestamp marks all ranks' arrival */
  if (!g_times) g_times = (double *)malloc(sizeof(double) * GOP_MAX_TIMES);
  if (g_times && g_ntimes < GOP_MAX_TIMES) g_times[g_ntimes++] = now_seconds();
  if (g_size == 1) {
    if (sendbuf != recvbuf) memcpy(recvbuf, sendbuf, (size_t)count * datatype->elem);
    return MPI_SUCCESS;
  }
  if (count > MAX_RED || !datatype->builtin) return MPI_ERR_OTHER;
  const int isint = datatype->elem == sizeof(int);
  for (int c = 0; c < count; c++)
    g_ctl->red[g_rank][c] = isint ? (double)((const int *)sendbuf)[c] : ((const double *)sendbuf)[c];
  MPI_Barrier(MPI_COMM_WORLD);
  for (int c = 0; c < count; c++) {
    double v = g_ctl->red[0][c];
    for (int r = 1; r < g_size; r++) {
      double x = g_ctl->red[r][c];
      if (op == MPI_MIN) v = x < v ? x : v;
      else if (op == MPI_MAX) v = x > v ? x : v;
      else v = v + x;
    }
    if (isint) ((int *)recvbuf)[c] = (int)v;
    else ((double *)recvbuf)[c] = v;
  }
  MPI_Barrier(MPI_COMM_WORLD);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm) {
  (void)tag;
  (void)comm;
  if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
  if (g_size == 1 || dest < 0 || dest >= g_size || dest == g_rank) {
    fprintf(stderr, "mpi shim: MPI_Send to rank %d is not supported\n", dest);
    return MPI_ERR_OTHER;
  }
  size_t n = msg_bytes(count, datatype);
  char *out = (char *)malloc(n + 1);
  if (!out) return MPI_ERR_OTHER;
  pack(buf, count, datatype, out);
  int rc = exchange(out, n, dest, NULL, 0, MPI_PROC_NULL);
  free(out);
  return rc;
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
  (void)tag;
  (void)comm;
  (void)status;
  if (source == MPI_PROC_NULL) return MPI_SUCCESS;
  if (g_size == 1 || source < 0 || source >= g_size || source == g_rank) {
    fprintf(stderr, "mpi shim: MPI_Recv from rank %d is not supported\n", source);
    return MPI_ERR_OTHER;
  }
  size_t n = msg_bytes(count, datatype);
  char *in = (char *)malloc(n + 1);
  if (!in) return MPI_ERR_OTHER;
  int rc = exchange(NULL, 0, MPI_PROC_NULL, in, n, source);
  if (rc == MPI_SUCCESS) unpack(buf, count, datatype, in);
  free(in);
  return rc;
}

double gop_shim_allreduce_time(int n) {
  if (n < 0 || n >= g_ntimes) return -1.0;
  return g_times[n];
}
int gop_shim_allreduce_count(void) { return g_ntimes; }
