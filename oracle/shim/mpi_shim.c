/*
 * mpi_shim.c -- the MPI subset of shim/mpi.h.  TEST INFRASTRUCTURE ONLY.
 *
 * Single process: every call is a local copy or a no-op.  Several ranks:
 * oracle_mpi_run() forks them after mapping one shared region that holds,
 * for every ordered pair (src, dst), a one-message mailbox guarded by two
 * process-shared semaphores (empty/full).  MPI_Sendrecv posts into
 * mailbox(me, dest) and then takes from mailbox(source, me); MPI_Alltoallv
 * posts one block to every peer, then takes one from every peer.  A rank
 * waits only for messages its peers post in the same collective step, so
 * the reference's call sequence cannot deadlock on one-slot mailboxes.
 * Cartesian communicators use row-major rank order (last dimension fastest),
 * as MPI specifies for MPI_Cart_create with reorder = 0.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <pthread.h>
#include <semaphore.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>

#define SHIM_MAXP 64
#define SHIM_MAXCOMM 64

typedef struct {
    sem_t full, empty;
    long bytes;
} shim_slot;

typedef struct {
    int nprocs;
    long cap;
    pthread_barrier_t barrier;
    shim_slot slot[SHIM_MAXP * SHIM_MAXP];
    /* followed by nprocs*nprocs*cap bytes of payload */
} shim_shared;

typedef struct {
    int used;
    int n;
    int world[SHIM_MAXP];
    int me;
    int ndims;
    int dims[4];
    int periods[4];
} shim_comm;

static int g_rank = 0, g_size = 1;
static shim_shared *g_sh = NULL;
static shim_comm g_comm[SHIM_MAXCOMM];
static int g_comm_init = 0;

static void comm_table_reset(void)
{
    memset(g_comm, 0, sizeof(g_comm));
    g_comm[0].used = 1;
    g_comm[0].n = g_size;
    for (int i = 0; i < g_size; i++) g_comm[0].world[i] = i;
    g_comm[0].me = g_rank;
    g_comm[0].ndims = 1;
    g_comm[0].dims[0] = g_size;
    g_comm[0].periods[0] = 0;
    g_comm_init = 1;
}

static shim_comm *get_comm(MPI_Comm c)
{
    if (!g_comm_init) comm_table_reset();
    if (c < 0 || c >= SHIM_MAXCOMM || !g_comm[c].used) {
        fprintf(stderr, "oracle mpi shim: invalid communicator %d\n", c);
        abort();
    }
    return &g_comm[c];
}

static int new_comm(void)
{
    if (!g_comm_init) comm_table_reset();
    for (int i = 1; i < SHIM_MAXCOMM; i++)
        if (!g_comm[i].used) {
            memset(&g_comm[i], 0, sizeof(g_comm[i]));
            g_comm[i].used = 1;
            return i;
        }
    fprintf(stderr, "oracle mpi shim: out of communicators\n");
    abort();
}

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_DOUBLE: return 8;
    case MPI_FLOAT: return 4;
    case MPI_INT: return 4;
    case MPI_BYTE: return 1;
    default: fprintf(stderr, "oracle mpi shim: unknown datatype %d\n", t); abort();
    }
}

static char *payload(int src, int dst)
{
    char *base = (char *)(g_sh + 1);
    return base + ((size_t)src * g_sh->nprocs + dst) * (size_t)g_sh->cap;
}

static void sem_wait_retry(sem_t *s)
{
    while (sem_wait(s) != 0)
        if (errno != EINTR) {
            perror("oracle mpi shim: sem_wait");
            abort();
        }
}

static void post(int src, int dst, const void *buf, long bytes)
{
    if (bytes > g_sh->cap) {
        fprintf(stderr, "oracle mpi shim: message of %ld bytes exceeds mailbox %ld\n", bytes, g_sh->cap);
        abort();
    }
    shim_slot *s = &g_sh->slot[src * g_sh->nprocs + dst];
    sem_wait_retry(&s->empty);
    memcpy(payload(src, dst), buf, (size_t)bytes);
    s->bytes = bytes;
    sem_post(&s->full);
}

static void take(int src, int dst, void *buf, long bytes)
{
    shim_slot *s = &g_sh->slot[src * g_sh->nprocs + dst];
    sem_wait_retry(&s->full);
    if (s->bytes != bytes) {
        fprintf(stderr, "oracle mpi shim: expected %ld bytes from %d, got %ld\n", bytes, src, s->bytes);
        abort();
    }
    memcpy(buf, payload(src, dst), (size_t)bytes);
    sem_post(&s->empty);
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
    *rank = get_comm(comm)->me;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    *size = get_comm(comm)->n;
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm comm, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *comm_cart)
{
    (void)reorder;
    shim_comm *c = get_comm(comm);
    int prod = 1;
    for (int d = 0; d < ndims; d++) prod *= dims[d];
    if (prod != c->n || ndims > 4) {
        fprintf(stderr, "oracle mpi shim: cart dims do not match communicator size\n");
        abort();
    }
    int h = new_comm();
    shim_comm *n = &g_comm[h];
    c = get_comm(comm);
    n->n = c->n;
    memcpy(n->world, c->world, sizeof(int) * (size_t)c->n);
    n->me = c->me;
    n->ndims = ndims;
    for (int d = 0; d < ndims; d++) {
        n->dims[d] = dims[d];
        n->periods[d] = periods[d] ? 1 : 0;
    }
    *comm_cart = h;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[])
{
    shim_comm *c = get_comm(comm);
    int r = rank;
    for (int d = c->ndims - 1; d >= 0; d--) {
        if (d < maxdims) coords[d] = r % c->dims[d];
        r /= c->dims[d];
    }
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank)
{
    shim_comm *c = get_comm(comm);
    int r = 0;
    for (int d = 0; d < c->ndims; d++) {
        int x = coords[d];
        if (c->periods[d]) {
            x %= c->dims[d];
            if (x < 0) x += c->dims[d];
        } else if (x < 0 || x >= c->dims[d]) {
            *rank = MPI_PROC_NULL;
            return MPI_SUCCESS;
        }
        r = r * c->dims[d] + x;
    }
    *rank = r;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *rank_source, int *rank_dest)
{
    shim_comm *c = get_comm(comm);
    int co[4];
    MPI_Cart_coords(comm, c->me, 4, co);
    int t[4];
    memcpy(t, co, sizeof(t));
    t[direction] = co[direction] + disp;
    MPI_Cart_rank(comm, t, rank_dest);
    t[direction] = co[direction] - disp;
    MPI_Cart_rank(comm, t, rank_source);
    return MPI_SUCCESS;
}

int MPI_Cart_sub(MPI_Comm comm, const int remain_dims[], MPI_Comm *newcomm)
{
    shim_comm *c = get_comm(comm);
    int mine[4];
    MPI_Cart_coords(comm, c->me, 4, mine);
    int h = new_comm();
    shim_comm *n = &g_comm[h];
    c = get_comm(comm);
    n->n = 0;
    n->me = -1;
    for (int r = 0; r < c->n; r++) {
        int co[4];
        MPI_Cart_coords(comm, r, 4, co);
        int same = 1;
        for (int d = 0; d < c->ndims; d++)
            if (!remain_dims[d] && co[d] != mine[d]) same = 0;
        if (same) {
            if (r == c->me) n->me = n->n;
            n->world[n->n++] = c->world[r];
        }
    }
    n->ndims = 0;
    for (int d = 0; d < c->ndims; d++)
        if (remain_dims[d]) {
            n->dims[n->ndims] = c->dims[d];
            n->periods[n->ndims] = c->periods[d];
            n->ndims++;
        }
    if (n->ndims == 0) {
        n->ndims = 1;
        n->dims[0] = 1;
    }
    *newcomm = h;
    return MPI_SUCCESS;
}

MPI_Fint MPI_Comm_c2f(MPI_Comm comm) { return (MPI_Fint)comm; }

int MPI_Comm_free(MPI_Comm *comm)
{
    if (*comm > 0 && *comm < SHIM_MAXCOMM) g_comm[*comm].used = 0;
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void)comm;
    fprintf(stderr, "oracle mpi shim: MPI_Abort(%d) on rank %d\n", errorcode, g_rank);
    fflush(stderr);
    if (g_sh) _exit(errorcode ? errorcode : 1);
    exit(errorcode ? errorcode : 1);
}

int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    if (g_sh && g_sh->nprocs > 1) pthread_barrier_wait(&g_sh->barrier);
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status)
{
    (void)sendtag;
    (void)recvtag;
    (void)status;
    shim_comm *c = get_comm(comm);
    long sb = (long)sendcount * (long)type_size(sendtype);
    long rb = (long)recvcount * (long)type_size(recvtype);
    int dw = (dest == MPI_PROC_NULL) ? -1 : c->world[dest];
    int sw = (source == MPI_PROC_NULL) ? -1 : c->world[source];
    int me = c->world[c->me];
    if (!g_sh) {
        /* single process: only self-messages are possible */
        if (dw == me && sw == me) memmove(recvbuf, sendbuf, (size_t)sb);
        return MPI_SUCCESS;
    }
    if (dw >= 0) post(me, dw, sendbuf, sb);
    if (sw >= 0) take(sw, me, recvbuf, rb);
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void *recvbuf, const int recvcounts[], const int rdispls[],
                  MPI_Datatype recvtype, MPI_Comm comm)
{
    shim_comm *c = get_comm(comm);
    size_t se = type_size(sendtype), re = type_size(recvtype);
    int me = c->world[c->me];
    /* local block first */
    memmove((char *)recvbuf + (size_t)rdispls[c->me] * re, (const char *)sendbuf + (size_t)sdispls[c->me] * se,
            (size_t)sendcounts[c->me] * se);
    if (c->n == 1) return MPI_SUCCESS;
    if (!g_sh) {
        fprintf(stderr, "oracle mpi shim: multi-rank Alltoallv outside oracle_mpi_run\n");
        abort();
    }
    for (int p = 0; p < c->n; p++)
        if (p != c->me)
            post(me, c->world[p], (const char *)sendbuf + (size_t)sdispls[p] * se, (long)sendcounts[p] * (long)se);
    for (int p = 0; p < c->n; p++)
        if (p != c->me)
            take(c->world[p], me, (char *)recvbuf + (size_t)rdispls[p] * re, (long)recvcounts[p] * (long)re);
    return MPI_SUCCESS;
}

int oracle_mpi_run(int nprocs, long max_msg_bytes, int (*fn)(int rank, void *arg), void *arg)
{
    if (nprocs < 1 || nprocs > SHIM_MAXP) return -1;
    if (nprocs == 1) {
        g_rank = 0;
        g_size = 1;
        g_sh = NULL;
        comm_table_reset();
        return fn(0, arg);
    }
    if (max_msg_bytes < 64) max_msg_bytes = 64;
    max_msg_bytes = (max_msg_bytes + 63) / 64 * 64;
    size_t total = sizeof(shim_shared) + (size_t)nprocs * nprocs * (size_t)max_msg_bytes;
    shim_shared *sh = (shim_shared *)mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (sh == MAP_FAILED) return -2;
    sh->nprocs = nprocs;
    sh->cap = max_msg_bytes;
    pthread_barrierattr_t ba;
    pthread_barrierattr_init(&ba);
    pthread_barrierattr_setpshared(&ba, PTHREAD_PROCESS_SHARED);
    pthread_barrier_init(&sh->barrier, &ba, (unsigned)nprocs);
    for (int i = 0; i < nprocs * nprocs; i++) {
        sem_init(&sh->slot[i].full, 1, 0);
        sem_init(&sh->slot[i].empty, 1, 1);
    }
    fflush(stdout);
    fflush(stderr);
    pid_t pids[SHIM_MAXP];
    for (int r = 0; r < nprocs; r++) {
        pid_t pid = fork();
        if (pid < 0) return -3;
        if (pid == 0) {
            g_rank = r;
            g_size = nprocs;
            g_sh = sh;
            comm_table_reset();
            int rc = fn(r, arg);
            fflush(stdout);
            fflush(stderr);
            _exit(rc == 0 ? 0 : 1);
        }
        pids[r] = pid;
    }
    int fail = 0;
    for (int r = 0; r < nprocs; r++) {
        int st = 0;
        waitpid(pids[r], &st, 0);
        if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) fail = 1;
    }
    munmap(sh, total);
    return fail ? 1 : 0;
}
