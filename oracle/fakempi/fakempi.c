/* fakempi: the MPI subset the reference's CC path calls, so that its sources
 * (cc_mpi.c, exchange_plan.c, graph_dist.c, mpi_cc_benchmark.c) compile and
 * run unmodified on one host.  TEST INFRASTRUCTURE ONLY: it is linked into the
 * reference-built checker under oracle/_ref, never into the product.
 *
 * Process model: MPI_Init maps one shared anonymous region and forks
 * FAKEMPI_NP - 1 children (rank 0 is the original process), so every rank
 * returns from MPI_Init with the same argc/argv.  Children die with rank 0
 * (PR_SET_PDEATHSIG); rank 0 watches its children (SIGCHLD) and a child that
 * exits non-zero or by a signal, or any MPI_Abort, raises a shared abort flag
 * that every waiting rank checks, so a failure ends the whole job with that
 * rank's code, like mpirun.  MPI_Finalize ends with a barrier; rank 0 then
 * reaps the children and exits non-zero if one of them failed.
 *
 * Transport: one byte ring per ordered rank pair (src -> dst, single writer,
 * single reader, acquire/release counters).  A message is a 16-byte header
 * {bytes, tag, context} followed by its payload, streamed through the ring in
 * pieces, so a message may be far larger than the ring.  Receives are
 * FIFO per pair: the next message on the ring must carry the expected tag and
 * context, and anything else aborts with a diagnostic (the reference never
 * relies on tag reordering).  Every call, collectives included, is a list
 * of sends and receives handed to one progress loop that moves whatever can
 * move on any ring, so a call never blocks on a full ring while another of
 * its transfers could proceed.  A wait with no progress for FAKEMPI_TIMEOUT_S
 * seconds (default 1800) aborts the job.
 *
 * Collectives: barrier (gather to rank 0, release), bcast and scatterv from
 * the root, reduce to the root, allreduce as all-to-all plus a local
 * reduction in rank order (identical result on every rank), alltoall(v), and
 * the neighbourhood collectives over the lists given to
 * MPI_Dist_graph_create_adjacent (which needs no communication).
 * MPI_Ineighbor_alltoallv completes before it returns; MPI_Wait is a no-op. */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <sched.h>
#include <signal.h>
#include <stdarg.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define FMPI_MAX_RANKS 64
#define FMPI_RING_BYTES ((uint64_t)4 << 20)
#define FMPI_MAX_COMMS 256

enum {
    TAG_BARRIER = -1, TAG_BCAST = -2, TAG_REDUCE = -3, TAG_ALLREDUCE = -4, TAG_ALLTOALL = -5,
    TAG_ALLTOALLV = -6, TAG_SCATTERV = -7, TAG_NB_ALLTOALL = -8, TAG_NB_ALLTOALLV = -9,
    TAG_NB_IALLTOALLV = -10
};

typedef struct {
    _Atomic uint64_t head; /* bytes written, by the sender */
    char pad0[56];
    _Atomic uint64_t tail; /* bytes read, by the receiver */
    char pad1[56];
} ring_ctl;

typedef struct {
    _Atomic int aborted;
    _Atomic int abort_code;
    int np;
    int pad;
} shm_hdr;

typedef struct {
    int used;
    int indeg, outdeg;
    int *src, *dst;
} graph_comm;

static shm_hdr *g_hdr;
static ring_ctl *g_ctl;
static char *g_ring;
static int g_rank, g_np = 1, g_init;
static pid_t g_child[FMPI_MAX_RANKS];
static double g_timeout_s = 1800.0;
static graph_comm g_comms[FMPI_MAX_COMMS]; /* id 0 is MPI_COMM_WORLD */

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void die(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3), noreturn));
static void die(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "fakempi[rank %d]: ", g_rank);
    vfprintf(stderr, fmt, ap);
    fputc('\n', stderr);
    va_end(ap);
    if (code == 0)
        code = 1;
    if (g_hdr) {
        int zero = 0;
        if (atomic_compare_exchange_strong(&g_hdr->aborted, &zero, 1))
            atomic_store(&g_hdr->abort_code, code);
    }
    fflush(stdout);
    fflush(stderr);
    _exit(code);
}

static void check_abort(void)
{
    if (g_hdr && atomic_load_explicit(&g_hdr->aborted, memory_order_acquire)) {
        int code = atomic_load(&g_hdr->abort_code);
        fflush(stdout);
        fflush(stderr);
        _exit(code ? code : 1);
    }
}

static void on_sigchld(int sig)
{
    (void)sig;
    siginfo_t si;
    for (int r = 1; r < g_np; ++r) {
        memset(&si, 0, sizeof(si));
        if (waitid(P_PID, (id_t)g_child[r], &si, WEXITED | WNOHANG | WNOWAIT) != 0)
            continue;
        if (si.si_pid == 0)
            continue;
        int bad = (si.si_code == CLD_EXITED) ? si.si_status : 128 + si.si_status;
        if (bad) {
            int zero = 0;
            if (atomic_compare_exchange_strong(&g_hdr->aborted, &zero, 1))
                atomic_store(&g_hdr->abort_code, bad);
        }
    }
}

static size_t type_size(MPI_Datatype t)
{
    size_t s = (size_t)(t & 0xff);
    if (s == 0 || ((t >> 8) & 0xff) == 0)
        die(1, "unknown datatype 0x%x", t);
    return s;
}

/* ------------------------------------------------------------- rings */

static ring_ctl *ctl_of(int src, int dst) { return &g_ctl[src * g_np + dst]; }
static char *buf_of(int src, int dst)
{
    return g_ring + (uint64_t)(src * g_np + dst) * FMPI_RING_BYTES;
}

/* Write up to len bytes into the (g_rank -> dst) ring; returns bytes written. */
static uint64_t ring_put(int dst, const char *p, uint64_t len)
{
    ring_ctl *c = ctl_of(g_rank, dst);
    char *b = buf_of(g_rank, dst);
    uint64_t head = atomic_load_explicit(&c->head, memory_order_relaxed);
    uint64_t tail = atomic_load_explicit(&c->tail, memory_order_acquire);
    uint64_t space = FMPI_RING_BYTES - (head - tail);
    uint64_t k = len < space ? len : space;
    if (!k)
        return 0;
    uint64_t off = head % FMPI_RING_BYTES, first = FMPI_RING_BYTES - off;
    if (first > k)
        first = k;
    memcpy(b + off, p, first);
    if (k > first)
        memcpy(b, p + first, k - first);
    atomic_store_explicit(&c->head, head + k, memory_order_release);
    return k;
}

/* Read up to len bytes from the (src -> g_rank) ring; returns bytes read. */
static uint64_t ring_get(int src, char *p, uint64_t len)
{
    ring_ctl *c = ctl_of(src, g_rank);
    char *b = buf_of(src, g_rank);
    uint64_t tail = atomic_load_explicit(&c->tail, memory_order_relaxed);
    uint64_t head = atomic_load_explicit(&c->head, memory_order_acquire);
    uint64_t avail = head - tail;
    uint64_t k = len < avail ? len : avail;
    if (!k)
        return 0;
    uint64_t off = tail % FMPI_RING_BYTES, first = FMPI_RING_BYTES - off;
    if (first > k)
        first = k;
    memcpy(p, b + off, first);
    if (k > first)
        memcpy(p + first, b, k - first);
    atomic_store_explicit(&c->tail, tail + k, memory_order_release);
    return k;
}

/* ---------------------------------------------------- transfers */

typedef struct {
    uint64_t bytes;
    int32_t tag;
    int32_t ctx;
} msg_hdr;

typedef struct {
    int is_send;
    int peer;
    int tag, ctx;
    char *p;          /* payload (send: source, receive: destination) */
    uint64_t n;       /* send: payload bytes; receive: capacity */
    uint64_t got;     /* receive: payload bytes announced */
    msg_hdr h;
    uint64_t hdr_done, done;
    int complete;
} xfer;

static void xfer_send(xfer *x, int peer, const void *p, uint64_t n, int tag, int ctx)
{
    memset(x, 0, sizeof(*x));
    x->is_send = 1;
    x->peer = peer;
    x->p = (char *)p;
    x->n = n;
    x->tag = tag;
    x->ctx = ctx;
    x->h.bytes = n;
    x->h.tag = tag;
    x->h.ctx = ctx;
}

static void xfer_recv(xfer *x, int peer, void *p, uint64_t cap, int tag, int ctx)
{
    memset(x, 0, sizeof(*x));
    x->peer = peer;
    x->p = (char *)p;
    x->n = cap;
    x->tag = tag;
    x->ctx = ctx;
}

/* Moves bytes of one transfer; returns the bytes moved (0 = none possible). */
static uint64_t xfer_step(xfer *x)
{
    uint64_t moved = 0;
    if (x->is_send) {
        if (x->hdr_done < sizeof(msg_hdr)) {
            uint64_t k = ring_put(x->peer, (const char *)&x->h + x->hdr_done,
                                  sizeof(msg_hdr) - x->hdr_done);
            x->hdr_done += k;
            moved += k;
            if (x->hdr_done < sizeof(msg_hdr))
                return moved;
        }
        if (x->done < x->n) {
            uint64_t k = ring_put(x->peer, x->p + x->done, x->n - x->done);
            x->done += k;
            moved += k;
        }
        if (x->done == x->n)
            x->complete = 1;
        return moved ? moved : (uint64_t)x->complete;
    }
    if (x->hdr_done < sizeof(msg_hdr)) {
        uint64_t k = ring_get(x->peer, (char *)&x->h + x->hdr_done, sizeof(msg_hdr) - x->hdr_done);
        x->hdr_done += k;
        moved += k;
        if (x->hdr_done < sizeof(msg_hdr))
            return moved;
        if (x->h.tag != x->tag || x->h.ctx != x->ctx)
            die(1, "message from rank %d has tag %d context %d, the receive expects tag %d "
                   "context %d (messages between two ranks must be received in send order)",
                x->peer, x->h.tag, x->h.ctx, x->tag, x->ctx);
        if (x->h.bytes > x->n)
            die(1, "message of %llu bytes from rank %d truncated to a %llu-byte receive",
                (unsigned long long)x->h.bytes, x->peer, (unsigned long long)x->n);
        x->got = x->h.bytes;
    }
    if (x->done < x->got) {
        uint64_t k = ring_get(x->peer, x->p + x->done, x->got - x->done);
        x->done += k;
        moved += k;
    }
    if (x->done == x->got)
        x->complete = 1;
    return moved ? moved : (uint64_t)x->complete;
}

/* Drives every transfer to completion.  Transfers on the same ring and in
 * the same direction go strictly in list order. */
static void run_xfers(xfer *xs, int k)
{
    double last = now_s();
    unsigned idle = 0;
    for (;;) {
        int pending = 0;
        uint64_t moved = 0;
        for (int i = 0; i < k; ++i) {
            if (xs[i].complete)
                continue;
            int blocked = 0;
            for (int j = 0; j < i && !blocked; ++j)
                blocked = !xs[j].complete && xs[j].is_send == xs[i].is_send &&
                          xs[j].peer == xs[i].peer;
            pending++;
            if (!blocked)
                moved += xfer_step(&xs[i]);
        }
        int left = 0;
        for (int i = 0; i < k; ++i)
            left += !xs[i].complete;
        if (!left)
            return;
        (void)pending;
        if (moved) {
            idle = 0;
            last = now_s();
            continue;
        }
        check_abort();
        if (++idle < 256) {
            sched_yield();
            continue;
        }
        struct timespec ts = {0, idle < 4096 ? 2000 : 50000};
        nanosleep(&ts, NULL);
        if ((idle & 255) == 0 && now_s() - last > g_timeout_s)
            die(1, "no progress for %.0f s in a transfer (a rank is missing from a collective "
                   "or a send/receive pair)", g_timeout_s);
    }
}

/* ------------------------------------------------------ init / exit */

int MPI_Init(int *argc, char ***argv)
{
    (void)argc;
    (void)argv;
    if (g_init)
        die(1, "MPI_Init called twice");
    const char *e = getenv("FAKEMPI_NP");
    g_np = e ? atoi(e) : 1;
    if (g_np < 1 || g_np > FMPI_MAX_RANKS)
        die(1, "FAKEMPI_NP=%s out of range 1..%d", e ? e : "", FMPI_MAX_RANKS);
    const char *t = getenv("FAKEMPI_TIMEOUT_S");
    if (t && atof(t) > 0)
        g_timeout_s = atof(t);

    size_t ctl_bytes = sizeof(ring_ctl) * (size_t)g_np * (size_t)g_np;
    size_t hdr_bytes = 4096;
    size_t total = hdr_bytes + ctl_bytes + (size_t)g_np * (size_t)g_np * FMPI_RING_BYTES;
    void *base = mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (base == MAP_FAILED)
        die(1, "mmap of %zu shared bytes failed: %s", total, strerror(errno));
    g_hdr = (shm_hdr *)base;
    g_hdr->np = g_np;
    g_ctl = (ring_ctl *)((char *)base + hdr_bytes);
    g_ring = (char *)base + hdr_bytes + ctl_bytes;
    memset(g_comms, 0, sizeof(g_comms));
    g_comms[0].used = 1;

    fflush(stdout);
    fflush(stderr);
    pid_t parent = getpid();
    g_rank = 0;
    for (int r = 1; r < g_np; ++r) {
        pid_t pid = fork();
        if (pid < 0)
            die(1, "fork failed: %s", strerror(errno));
        if (pid == 0) {
            g_rank = r;
            prctl(PR_SET_PDEATHSIG, SIGKILL);
            if (getppid() != parent)
                _exit(1);
            break;
        }
        g_child[r] = pid;
    }
    if (g_rank == 0 && g_np > 1) {
        struct sigaction sa;
        memset(&sa, 0, sizeof(sa));
        sa.sa_handler = on_sigchld;
        sa.sa_flags = SA_RESTART | SA_NOCLDSTOP;
        sigaction(SIGCHLD, &sa, NULL);
    }
    /* whole lines per write, so the ranks' lines do not interleave */
    setvbuf(stdout, NULL, _IOLBF, 0);
    g_init = 1;
    return MPI_SUCCESS;
}

int MPI_Initialized(int *flag)
{
    *flag = g_init;
    return MPI_SUCCESS;
}

int MPI_Finalize(void)
{
    MPI_Barrier(MPI_COMM_WORLD);
    fflush(stdout);
    fflush(stderr);
    if (g_rank != 0)
        return MPI_SUCCESS;
    int failed = 0;
    signal(SIGCHLD, SIG_DFL);
    for (int r = 1; r < g_np; ++r) {
        int st = 0;
        while (waitpid(g_child[r], &st, 0) < 0 && errno == EINTR)
            ;
        if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) {
            fprintf(stderr, "fakempi: rank %d ended with status 0x%x\n", r, st);
            failed = 1;
        }
    }
    if (failed)
        exit(1);
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
    (void)comm;
    *rank = g_rank;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    (void)comm;
    *size = g_np;
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void)comm;
    die(errorcode, "MPI_Abort(%d)", errorcode);
}

double MPI_Wtime(void) { return now_s(); }

/* ------------------------------------------------------ point to point */

static int ctx_of(MPI_Comm comm)
{
    if (comm < 0 || comm >= FMPI_MAX_COMMS || !g_comms[comm].used)
        die(1, "invalid communicator %d", comm);
    return comm == MPI_COMM_WORLD ? 0 : 1;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    if (dest < 0 || dest >= g_np || tag < 0 || count < 0)
        die(1, "MPI_Send: bad dest %d / tag %d / count %d", dest, tag, count);
    xfer x;
    xfer_send(&x, dest, buf, (uint64_t)count * type_size(type), tag, ctx_of(comm));
    run_xfers(&x, 1);
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status)
{
    if (source < 0 || source >= g_np || tag < 0 || count < 0)
        die(1, "MPI_Recv: bad source %d / tag %d / count %d (wildcards are not supported)",
            source, tag, count);
    xfer x;
    xfer_recv(&x, source, buf, (uint64_t)count * type_size(type), tag, ctx_of(comm));
    run_xfers(&x, 1);
    if (status) {
        status->MPI_SOURCE = source;
        status->MPI_TAG = tag;
        status->MPI_ERROR = MPI_SUCCESS;
        status->count_bytes = x.got;
    }
    return MPI_SUCCESS;
}

/* ------------------------------------------------------ collectives */

int MPI_Barrier(MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    xfer xs[FMPI_MAX_RANKS];
    char dummy = 0;
    int k = 0;
    if (g_rank == 0) {
        for (int r = 1; r < g_np; ++r)
            xfer_recv(&xs[k++], r, &dummy, 0, TAG_BARRIER, ctx);
        run_xfers(xs, k);
        k = 0;
        for (int r = 1; r < g_np; ++r)
            xfer_send(&xs[k++], r, &dummy, 0, TAG_BARRIER, ctx);
        run_xfers(xs, k);
    } else {
        xfer_send(&xs[0], 0, &dummy, 0, TAG_BARRIER, ctx);
        xfer_recv(&xs[1], 0, &dummy, 0, TAG_BARRIER, ctx);
        run_xfers(xs, 2);
    }
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    uint64_t bytes = (uint64_t)count * type_size(type);
    xfer xs[FMPI_MAX_RANKS];
    int k = 0;
    if (g_rank == root) {
        for (int r = 0; r < g_np; ++r)
            if (r != root)
                xfer_send(&xs[k++], r, buf, bytes, TAG_BCAST, ctx);
    } else {
        xfer_recv(&xs[k++], root, buf, bytes, TAG_BCAST, ctx);
    }
    run_xfers(xs, k);
    return MPI_SUCCESS;
}

static void reduce_into(void *acc, const void *in, int count, MPI_Datatype type, MPI_Op op)
{
    int kind = (type >> 8) & 0xff;
    size_t sz = type_size(type);
    for (int i = 0; i < count; ++i) {
        if (kind == 3) {
            double a = sz == 8 ? ((double *)acc)[i] : ((float *)acc)[i];
            double b = sz == 8 ? ((const double *)in)[i] : ((const float *)in)[i];
            double r = op == MPI_SUM ? a + b : op == MPI_MAX ? (a > b ? a : b)
                     : op == MPI_MIN ? (a < b ? a : b) : (die(1, "op %d on floats", op), 0.0);
            if (sz == 8)
                ((double *)acc)[i] = r;
            else
                ((float *)acc)[i] = (float)r;
            continue;
        }
        /* integers: widen to 64 bits, signed or unsigned */
        int64_t sa = 0, sb = 0;
        uint64_t ua = 0, ub = 0;
        switch (sz) {
        case 1: sa = ((int8_t *)acc)[i]; sb = ((const int8_t *)in)[i];
                ua = ((uint8_t *)acc)[i]; ub = ((const uint8_t *)in)[i]; break;
        case 2: sa = ((int16_t *)acc)[i]; sb = ((const int16_t *)in)[i];
                ua = ((uint16_t *)acc)[i]; ub = ((const uint16_t *)in)[i]; break;
        case 4: sa = ((int32_t *)acc)[i]; sb = ((const int32_t *)in)[i];
                ua = ((uint32_t *)acc)[i]; ub = ((const uint32_t *)in)[i]; break;
        case 8: sa = ((int64_t *)acc)[i]; sb = ((const int64_t *)in)[i];
                ua = ((uint64_t *)acc)[i]; ub = ((const uint64_t *)in)[i]; break;
        default: die(1, "datatype size %zu", sz);
        }
        uint64_t r;
        int is_signed = kind == 1;
        switch (op) {
        case MPI_SUM: r = ua + ub; break;
        case MPI_MAX: r = is_signed ? (uint64_t)(sa > sb ? sa : sb) : (ua > ub ? ua : ub); break;
        case MPI_MIN: r = is_signed ? (uint64_t)(sa < sb ? sa : sb) : (ua < ub ? ua : ub); break;
        case MPI_LOR: r = (ua != 0) || (ub != 0); break;
        case MPI_LAND: r = (ua != 0) && (ub != 0); break;
        case MPI_BOR: r = ua | ub; break;
        default: die(1, "unsupported reduction op %d", op);
        }
        switch (sz) {
        case 1: ((uint8_t *)acc)[i] = (uint8_t)r; break;
        case 2: ((uint16_t *)acc)[i] = (uint16_t)r; break;
        case 4: ((uint32_t *)acc)[i] = (uint32_t)r; break;
        default: ((uint64_t *)acc)[i] = r; break;
        }
    }
}

/* Every rank's contribution, in rank order, into all[r * bytes]. */
static char *gather_all(const void *sendbuf, uint64_t bytes, int to_all, int root, int tag,
                        int ctx)
{
    char *all = NULL;
    int receiver = to_all || g_rank == root;
    if (receiver) {
        all = (char *)malloc(bytes * (uint64_t)g_np + 1);
        if (!all)
            die(1, "out of memory in a reduction");
        memcpy(all + bytes * (uint64_t)g_rank, sendbuf, bytes);
    }
    xfer xs[2 * FMPI_MAX_RANKS];
    int k = 0;
    for (int r = 0; r < g_np; ++r) {
        if (r == g_rank)
            continue;
        if (to_all || r == root)
            xfer_send(&xs[k++], r, sendbuf, bytes, tag, ctx);
        if (receiver)
            xfer_recv(&xs[k++], r, all + bytes * (uint64_t)r, bytes, tag, ctx);
    }
    run_xfers(xs, k);
    return all;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    uint64_t bytes = (uint64_t)count * type_size(type);
    char *all = gather_all(sendbuf, bytes, 0, root, TAG_REDUCE, ctx);
    if (g_rank == root) {
        memcpy(recvbuf, all, bytes);
        for (int r = 1; r < g_np; ++r)
            reduce_into(recvbuf, all + bytes * (uint64_t)r, count, type, op);
    }
    free(all);
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    uint64_t bytes = (uint64_t)count * type_size(type);
    char *all = gather_all(sendbuf, bytes, 1, 0, TAG_ALLREDUCE, ctx);
    memcpy(recvbuf, all, bytes);
    for (int r = 1; r < g_np; ++r)
        reduce_into(recvbuf, all + bytes * (uint64_t)r, count, type, op);
    free(all);
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    uint64_t sb = (uint64_t)sendcount * type_size(sendtype);
    uint64_t rb = (uint64_t)recvcount * type_size(recvtype);
    xfer xs[2 * FMPI_MAX_RANKS];
    int k = 0;
    for (int r = 0; r < g_np; ++r) {
        xfer_send(&xs[k++], r, (const char *)sendbuf + sb * (uint64_t)r, sb, TAG_ALLTOALL, ctx);
        xfer_recv(&xs[k++], r, (char *)recvbuf + rb * (uint64_t)r, rb, TAG_ALLTOALL, ctx);
    }
    run_xfers(xs, k);
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                  MPI_Datatype sendtype, void *recvbuf, const int *recvcounts,
                  const int *rdispls, MPI_Datatype recvtype, MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    size_t ss = type_size(sendtype), rs = type_size(recvtype);
    xfer xs[2 * FMPI_MAX_RANKS];
    int k = 0;
    for (int r = 0; r < g_np; ++r) {
        xfer_send(&xs[k++], r, (const char *)sendbuf + ss * (uint64_t)sdispls[r],
                  ss * (uint64_t)sendcounts[r], TAG_ALLTOALLV, ctx);
        xfer_recv(&xs[k++], r, (char *)recvbuf + rs * (uint64_t)rdispls[r],
                  rs * (uint64_t)recvcounts[r], TAG_ALLTOALLV, ctx);
    }
    run_xfers(xs, k);
    return MPI_SUCCESS;
}

int MPI_Scatterv(const void *sendbuf, const int *sendcounts, const int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int root, MPI_Comm comm)
{
    int ctx = ctx_of(comm);
    size_t ss = type_size(sendtype), rs = type_size(recvtype);
    xfer xs[2 * FMPI_MAX_RANKS];
    int k = 0;
    if (g_rank == root)
        for (int r = 0; r < g_np; ++r)
            xfer_send(&xs[k++], r, (const char *)sendbuf + ss * (uint64_t)displs[r],
                      ss * (uint64_t)sendcounts[r], TAG_SCATTERV, ctx);
    xfer_recv(&xs[k++], root, recvbuf, rs * (uint64_t)recvcount, TAG_SCATTERV, ctx);
    run_xfers(xs, k);
    return MPI_SUCCESS;
}

/* ------------------------------------------------ neighbourhood collectives */

int MPI_Dist_graph_create_adjacent(MPI_Comm comm_old, int indegree, const int sources[],
                                   const int sourceweights[], int outdegree,
                                   const int destinations[], const int destweights[],
                                   MPI_Info info, int reorder, MPI_Comm *comm_dist_graph)
{
    (void)sourceweights;
    (void)destweights;
    (void)info;
    (void)reorder;
    ctx_of(comm_old);
    int id = 1;
    while (id < FMPI_MAX_COMMS && g_comms[id].used)
        id++;
    if (id == FMPI_MAX_COMMS)
        die(1, "too many graph communicators");
    graph_comm *g = &g_comms[id];
    g->indeg = indegree;
    g->outdeg = outdegree;
    g->src = (int *)malloc(sizeof(int) * (size_t)(indegree + 1));
    g->dst = (int *)malloc(sizeof(int) * (size_t)(outdegree + 1));
    if (!g->src || !g->dst)
        die(1, "out of memory in MPI_Dist_graph_create_adjacent");
    for (int i = 0; i < indegree; ++i) {
        if (sources[i] < 0 || sources[i] >= g_np)
            die(1, "graph source %d out of range", sources[i]);
        g->src[i] = sources[i];
    }
    for (int i = 0; i < outdegree; ++i) {
        if (destinations[i] < 0 || destinations[i] >= g_np)
            die(1, "graph destination %d out of range", destinations[i]);
        g->dst[i] = destinations[i];
    }
    g->used = 1;
    *comm_dist_graph = id;
    return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm)
{
    if (comm && *comm > 0 && *comm < FMPI_MAX_COMMS && g_comms[*comm].used) {
        free(g_comms[*comm].src);
        free(g_comms[*comm].dst);
        memset(&g_comms[*comm], 0, sizeof(graph_comm));
    }
    if (comm)
        *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}

static graph_comm *graph_of(MPI_Comm comm)
{
    if (comm <= 0 || comm >= FMPI_MAX_COMMS || !g_comms[comm].used)
        die(1, "neighbourhood collective on communicator %d, which is not a graph", comm);
    return &g_comms[comm];
}

static void neighbor_v(const void *sendbuf, const int *sendcounts, const int *sdispls,
                       MPI_Datatype sendtype, void *recvbuf, const int *recvcounts,
                       const int *rdispls, MPI_Datatype recvtype, MPI_Comm comm, int tag)
{
    graph_comm *g = graph_of(comm);
    size_t ss = type_size(sendtype), rs = type_size(recvtype);
    int k = 0, cap = g->indeg + g->outdeg;
    xfer *xs = (xfer *)malloc(sizeof(xfer) * (size_t)(cap + 1));
    if (!xs)
        die(1, "out of memory in a neighbourhood collective");
    for (int i = 0; i < g->outdeg; ++i)
        xfer_send(&xs[k++], g->dst[i], (const char *)sendbuf + ss * (uint64_t)sdispls[i],
                  ss * (uint64_t)sendcounts[i], tag, 1);
    for (int i = 0; i < g->indeg; ++i)
        xfer_recv(&xs[k++], g->src[i], (char *)recvbuf + rs * (uint64_t)rdispls[i],
                  rs * (uint64_t)recvcounts[i], tag, 1);
    run_xfers(xs, k);
    free(xs);
}

int MPI_Neighbor_alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                          void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm)
{
    graph_comm *g = graph_of(comm);
    int n = (g->indeg > g->outdeg ? g->indeg : g->outdeg) + 1;
    int *sc = (int *)malloc(sizeof(int) * (size_t)n), *sd = (int *)malloc(sizeof(int) * (size_t)n);
    int *rc = (int *)malloc(sizeof(int) * (size_t)n), *rd = (int *)malloc(sizeof(int) * (size_t)n);
    if (!sc || !sd || !rc || !rd)
        die(1, "out of memory in MPI_Neighbor_alltoall");
    for (int i = 0; i < n; ++i) {
        sc[i] = sendcount;
        sd[i] = i * sendcount;
        rc[i] = recvcount;
        rd[i] = i * recvcount;
    }
    neighbor_v(sendbuf, sc, sd, sendtype, recvbuf, rc, rd, recvtype, comm, TAG_NB_ALLTOALL);
    free(sc);
    free(sd);
    free(rc);
    free(rd);
    return MPI_SUCCESS;
}

int MPI_Neighbor_alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                           MPI_Datatype sendtype, void *recvbuf, const int recvcounts[],
                           const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm)
{
    neighbor_v(sendbuf, sendcounts, sdispls, sendtype, recvbuf, recvcounts, rdispls, recvtype,
               comm, TAG_NB_ALLTOALLV);
    return MPI_SUCCESS;
}

int MPI_Ineighbor_alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                            MPI_Datatype sendtype, void *recvbuf, const int recvcounts[],
                            const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm,
                            MPI_Request *request)
{
    neighbor_v(sendbuf, sendcounts, sdispls, sendtype, recvbuf, recvcounts, rdispls, recvtype,
               comm, TAG_NB_IALLTOALLV);
    if (request)
        *request = 0;
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status)
{
    (void)status;
    if (request)
        *request = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
