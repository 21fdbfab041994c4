/*
 * Test-oracle MPI stand-in (see mpi.h).  NOT product code.
 *
 * A "world" is created by shim_mpi_run(n, fn, arg): with n == 1 fn runs in the
 * calling process as rank 0 of 1; with n > 1 the caller forks n children that
 * share one anonymous MAP_SHARED arena.  Collectives copy each rank's
 * contribution into its own arena slot, then every rank reduces the slots in
 * rank order, so results are deterministic and identical on every rank.
 * Point-to-point messages go through one mailbox per (source, destination)
 * pair; a send blocks only while the previous message on that pair is unread.
 * That covers the reference's use: halo exchanges with MPI_PROC_NULL peers
 * (blocks never straddle ranks in MLmap) and the final Send/Recv gather of the
 * map pieces to rank 0 (mappraiser/src/mappraiser.c:244-292).
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <execinfo.h>
#include <pthread.h>
#include <sched.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define SHIM_MAXR 64

typedef struct {
    volatile int full;
    int          tag;
    size_t       bytes;
} shim_mbox;

typedef struct {
    pthread_barrier_t bar;
    int               size;
    size_t            slot_bytes; /* per-rank collective slot */
    size_t            mbox_bytes; /* per-pair mailbox payload */
    shim_mbox         mb[SHIM_MAXR][SHIM_MAXR];
} shim_hdr;

static int       g_rank = 0;
static int       g_size = 1;
static shim_hdr *g_hdr  = NULL; /* NULL: single process world */
static char     *g_slots = NULL;
static char     *g_mbox  = NULL;

static size_t dt_size(MPI_Datatype dt) { return (size_t) (dt >> 8) & 0xff; }

static void die(const char *msg) {
    fprintf(stderr, "[shim_mpi rank %d] %s\n", g_rank, msg);
    fflush(stderr);
    _exit(3);
}

int MPI_Init(int *argc, char ***argv) {
    (void) argc;
    (void) argv;
    return MPI_SUCCESS;
}
int MPI_Initialized(int *flag) {
    *flag = 1;
    return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) {
    (void) comm;
    fprintf(stderr, "[shim_mpi rank %d] MPI_Abort(%d)\n", g_rank, code);
    _exit(code ? code : 1);
}

double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
    *rank = (comm == MPI_COMM_SELF) ? 0 : g_rank;
    return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
    *size = (comm == MPI_COMM_SELF) ? 1 : g_size;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    (void) comm;
    if (g_hdr) pthread_barrier_wait(&g_hdr->bar);
    return MPI_SUCCESS;
}

static void reduce_into(void *out, const void *in, int count, MPI_Datatype dt, MPI_Op op) {
    int i;
#define RED(T)                                                                                     \
    {                                                                                              \
        T *o = (T *) out;                                                                          \
        const T *a = (const T *) in;                                                               \
        for (i = 0; i < count; i++) {                                                              \
            if (op == MPI_SUM) o[i] += a[i];                                                       \
            else if (op == MPI_MAX) o[i] = a[i] > o[i] ? a[i] : o[i];                              \
            else if (op == MPI_MIN) o[i] = a[i] < o[i] ? a[i] : o[i];                              \
        }                                                                                          \
    }
    if (dt == MPI_DOUBLE) RED(double)
    else if (dt == MPI_INT) RED(int)
    else if (dt == MPI_FLOAT) RED(float)
    else if (dt == MPI_LONG || dt == MPI_INT64_T) RED(int64_t)
    else die("unsupported datatype in reduction");
#undef RED
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op,
                  MPI_Comm comm) {
    size_t bytes = (size_t) count * dt_size(dt);
    const void *src = (sendbuf == MPI_IN_PLACE) ? recvbuf : sendbuf;
    if (comm == MPI_COMM_SELF || !g_hdr) {
        if (src != recvbuf) memmove(recvbuf, src, bytes);
        return MPI_SUCCESS;
    }
    if (bytes > g_hdr->slot_bytes) die("Allreduce payload exceeds the shared arena slot");
    memcpy(g_slots + (size_t) g_rank * g_hdr->slot_bytes, src, bytes);
    pthread_barrier_wait(&g_hdr->bar);
    memcpy(recvbuf, g_slots, bytes);
    for (int r = 1; r < g_size; r++)
        reduce_into(recvbuf, g_slots + (size_t) r * g_hdr->slot_bytes, count, dt, op);
    pthread_barrier_wait(&g_hdr->bar);
    return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root,
               MPI_Comm comm) {
    if (!g_hdr || comm == MPI_COMM_SELF) {
        const void *src = (sendbuf == MPI_IN_PLACE) ? recvbuf : sendbuf;
        if (src != recvbuf) memmove(recvbuf, src, (size_t) count * dt_size(dt));
        return MPI_SUCCESS;
    }
    /* the reduction is computed everywhere; only root's buffer is written */
    size_t bytes = (size_t) count * dt_size(dt);
    void  *tmp   = malloc(bytes ? bytes : 1);
    const void *src = (sendbuf == MPI_IN_PLACE) ? recvbuf : sendbuf;
    MPI_Allreduce(src, tmp, count, dt, op, comm);
    if (g_rank == root) memcpy(recvbuf, tmp, bytes);
    free(tmp);
    return MPI_SUCCESS;
}

int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm) {
    size_t sb = (size_t) sendcount * dt_size(sendtype);
    size_t rb = (size_t) recvcount * dt_size(recvtype);
    if (!g_hdr || comm == MPI_COMM_SELF) {
        if (sendbuf != MPI_IN_PLACE) memmove(recvbuf, sendbuf, sb);
        return MPI_SUCCESS;
    }
    if (sb > g_hdr->slot_bytes) die("Gather payload exceeds the shared arena slot");
    memcpy(g_slots + (size_t) g_rank * g_hdr->slot_bytes, sendbuf, sb);
    pthread_barrier_wait(&g_hdr->bar);
    if (g_rank == root)
        for (int r = 0; r < g_size; r++)
            memcpy((char *) recvbuf + (size_t) r * rb, g_slots + (size_t) r * g_hdr->slot_bytes, rb);
    pthread_barrier_wait(&g_hdr->bar);
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                  MPI_Datatype sendtype, void *recvbuf, const int *recvcounts, const int *rdispls,
                  MPI_Datatype recvtype, MPI_Comm comm) {
    size_t ss = dt_size(sendtype), rs = dt_size(recvtype);
    if (!g_hdr || comm == MPI_COMM_SELF) {
        memmove((char *) recvbuf + (size_t) rdispls[0] * rs, (const char *) sendbuf + (size_t) sdispls[0] * ss,
                (size_t) sendcounts[0] * ss);
        return MPI_SUCCESS;
    }
    /* slot layout: [dest][bytes...] written by each sender as a packed run */
    size_t total = 0;
    for (int d = 0; d < g_size; d++) total += (size_t) sendcounts[d] * ss;
    if (total + (size_t) g_size * sizeof(size_t) > g_hdr->slot_bytes) die("Alltoallv payload too large");
    char   *slot = g_slots + (size_t) g_rank * g_hdr->slot_bytes;
    size_t *offs = (size_t *) slot;
    size_t  pos  = (size_t) g_size * sizeof(size_t);
    for (int d = 0; d < g_size; d++) {
        offs[d] = pos;
        memcpy(slot + pos, (const char *) sendbuf + (size_t) sdispls[d] * ss, (size_t) sendcounts[d] * ss);
        pos += (size_t) sendcounts[d] * ss;
    }
    pthread_barrier_wait(&g_hdr->bar);
    for (int s = 0; s < g_size; s++) {
        char   *sl = g_slots + (size_t) s * g_hdr->slot_bytes;
        size_t *of = (size_t *) sl;
        memcpy((char *) recvbuf + (size_t) rdispls[s] * rs, sl + of[g_rank], (size_t) recvcounts[s] * rs);
    }
    pthread_barrier_wait(&g_hdr->bar);
    return MPI_SUCCESS;
}

static void p2p_send(const void *buf, size_t bytes, int dest, int tag) {
    if (dest == MPI_PROC_NULL) return;
    if (!g_hdr) {
        if (dest == 0) die("send to self in a one-rank world");
        die("send to a rank that does not exist");
    }
    if (dest < 0 || dest >= g_size) die("send to an invalid rank");
    shim_mbox *mb = &g_hdr->mb[g_rank][dest];
    if (bytes > g_hdr->mbox_bytes) die("point-to-point message exceeds the mailbox");
    while (mb->full) sched_yield();
    __sync_synchronize();
    memcpy(g_mbox + ((size_t) g_rank * g_size + dest) * g_hdr->mbox_bytes, buf, bytes);
    mb->tag   = tag;
    mb->bytes = bytes;
    __sync_synchronize();
    mb->full = 1;
}

static void p2p_recv(void *buf, size_t maxbytes, int source, int tag, MPI_Status *st) {
    if (source == MPI_PROC_NULL) {
        if (st && st != MPI_STATUS_IGNORE) {
            st->MPI_SOURCE = MPI_PROC_NULL;
            st->count_bytes = 0;
        }
        return;
    }
    if (!g_hdr || source < 0 || source >= g_size) die("receive from an invalid rank");
    shim_mbox *mb = &g_hdr->mb[source][g_rank];
    while (!mb->full) sched_yield();
    __sync_synchronize();
    if (tag != MPI_ANY_TAG && mb->tag != tag) die("message tag order mismatch");
    if (mb->bytes > maxbytes) die("message truncated");
    memcpy(buf, g_mbox + ((size_t) source * g_size + g_rank) * g_hdr->mbox_bytes, mb->bytes);
    if (st && st != MPI_STATUS_IGNORE) {
        st->MPI_SOURCE  = source;
        st->MPI_TAG     = mb->tag;
        st->count_bytes = (int) mb->bytes;
    }
    __sync_synchronize();
    mb->full = 0;
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm) {
    (void) comm;
    p2p_send(buf, (size_t) count * dt_size(dt), dest, tag);
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
             MPI_Status *status) {
    (void) comm;
    p2p_recv(buf, (size_t) count * dt_size(dt), source, tag, status);
    return MPI_SUCCESS;
}

/* deferred receives: the request remembers the arguments, MPI_Wait performs it */
typedef struct {
    int    used, is_recv, source, tag;
    void  *buf;
    size_t bytes;
} shim_req;
static shim_req g_reqs[256];

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm,
              MPI_Request *req) {
    MPI_Send(buf, count, dt, dest, tag, comm);
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
              MPI_Request *req) {
    (void) comm;
    for (int i = 0; i < 256; i++)
        if (!g_reqs[i].used) {
            g_reqs[i] = (shim_req){1, 1, source, tag, buf, (size_t) count * dt_size(dt)};
            *req      = i + 1;
            return MPI_SUCCESS;
        }
    die("too many pending receives");
    return 1;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status) {
    if (*req == MPI_REQUEST_NULL || *req <= 0 || *req > 256) {
        *req = MPI_REQUEST_NULL;
        return MPI_SUCCESS;
    }
    shim_req *r = &g_reqs[*req - 1];
    if (r->used && r->is_recv) p2p_recv(r->buf, r->bytes, r->source, r->tag, status);
    r->used = 0;
    *req    = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]) {
    for (int i = 0; i < count; i++)
        MPI_Wait(&reqs[i], statuses == MPI_STATUSES_IGNORE ? MPI_STATUS_IGNORE : &statuses[i]);
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
    MPI_Send(sendbuf, sendcount, sendtype, dest, sendtag, comm);
    MPI_Recv(recvbuf, recvcount, recvtype, source, recvtag, comm, status);
    return MPI_SUCCESS;
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype dt, int dest, int sendtag, int source,
                         int recvtag, MPI_Comm comm, MPI_Status *status) {
    size_t bytes = (size_t) count * dt_size(dt);
    void  *tmp   = malloc(bytes ? bytes : 1);
    memcpy(tmp, buf, bytes);
    MPI_Send(tmp, count, dt, dest, sendtag, comm);
    MPI_Recv(buf, count, dt, source, recvtag, comm, status);
    free(tmp);
    return MPI_SUCCESS;
}

/* a crashing rank prints where it crashed before it dies */
static void crash_handler(int sig) {
    void *frames[64];
    int   n = backtrace(frames, 64);
    char  msg[96];
    int   len = snprintf(msg, sizeof(msg), "[shim_mpi rank %d] fatal signal %d, backtrace:\n", g_rank, sig);
    if (write(2, msg, (size_t) len) < 0) _exit(128 + sig);
    backtrace_symbols_fd(frames, n, 2);
    _exit(128 + sig);
}

int shim_mpi_run(int nranks, void (*fn)(int rank, void *arg), void *arg) {
    if (nranks <= 1) {
        g_rank = 0;
        g_size = 1;
        g_hdr  = NULL;
        fn(0, arg);
        return 0;
    }
    if (nranks > SHIM_MAXR) return -1;
    const char *env     = getenv("SHIM_MPI_SLOT_MB");
    size_t      slot_mb = env ? (size_t) atol(env) : 256;
    env                 = getenv("SHIM_MPI_MBOX_MB");
    size_t mbox_mb      = env ? (size_t) atol(env) : 64;
    size_t hdr_bytes    = (sizeof(shim_hdr) + 4095) & ~(size_t) 4095;
    size_t total        = hdr_bytes + (size_t) nranks * slot_mb * (1u << 20)
                 + (size_t) nranks * nranks * mbox_mb * (1u << 20);
    char *base = mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE,
                      -1, 0);
    if (base == MAP_FAILED) return -2;
    shim_hdr *h = (shim_hdr *) base;
    memset(h, 0, sizeof(*h));
    pthread_barrierattr_t ba;
    pthread_barrierattr_init(&ba);
    pthread_barrierattr_setpshared(&ba, PTHREAD_PROCESS_SHARED);
    pthread_barrier_init(&h->bar, &ba, (unsigned) nranks);
    h->size       = nranks;
    h->slot_bytes = slot_mb << 20;
    h->mbox_bytes = mbox_mb << 20;

    fflush(stdout);
    fflush(stderr);
    pid_t pids[SHIM_MAXR];
    for (int r = 0; r < nranks; r++) {
        pid_t p = fork();
        if (p == 0) {
            signal(SIGSEGV, crash_handler);
            signal(SIGBUS, crash_handler);
            signal(SIGFPE, crash_handler);
            g_rank  = r;
            g_size  = nranks;
            g_hdr   = h;
            g_slots = base + hdr_bytes;
            g_mbox  = g_slots + (size_t) nranks * h->slot_bytes;
            fn(r, arg);
            fflush(stdout);
            fflush(stderr);
            _exit(0);
        }
        if (p < 0) return -3;
        pids[r] = p;
    }
    int failed = 0, alive = nranks;
    while (alive > 0) {
        int   st;
        pid_t p = waitpid(-1, &st, 0);
        if (p < 0) break;
        for (int r = 0; r < nranks; r++)
            if (pids[r] == p) {
                pids[r] = 0;
                alive--;
                if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) {
                    if (!failed) {
                        if (WIFSIGNALED(st))
                            fprintf(stderr, "[shim_mpi] rank %d killed by signal %d\n", r, WTERMSIG(st));
                        else
                            fprintf(stderr, "[shim_mpi] rank %d exited with status %d\n", r, WEXITSTATUS(st));
                    }
                    failed = 1;
                }
            }
        if (failed)
            for (int r = 0; r < nranks; r++)
                if (pids[r] > 0) kill(pids[r], SIGKILL);
    }
    pthread_barrier_destroy(&h->bar);
    munmap(base, total);
    return failed ? 1 : 0;
}
