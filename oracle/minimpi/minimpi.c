/* Checker infrastructure: the MPI calls of the reference TeaLeaf host over
 * Unix-domain sockets between processes (see mpi.h).
 *
 * Rank r listens on MINIMPI_DIR/r.sock, connects to every lower rank and
 * accepts every higher one, so each pair of ranks shares one stream. A
 * message is a frame {tag, count, count doubles}. MPI_Isend copies its data
 * into the destination's outgoing queue (the send buffer is free at once);
 * MPI_Irecv is matched, in arrival order, against the frames received from
 * its source with its tag (MPI's non-overtaking rule). Every wait drives one
 * progress loop that writes queued frames and reads arrived ones with
 * poll(), so two ranks sending to each other never block on a full socket.
 * Every wait is bounded (MINIMPI_TIMEOUT seconds, default 120): a rank that
 * waits longer, or on a peer that has closed, exits with status 3.
 */
#include "mpi.h"

#include <errno.h>
#include <fcntl.h>
#include <poll.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/socket.h>
#include <sys/un.h>
#include <time.h>
#include <unistd.h>

typedef struct Frame {
    int src, tag, count;
    double* data;
    struct Frame* next;
} Frame;

typedef struct Out {
    char* bytes;
    size_t len, off;
    struct Out* next;
} Out;

typedef struct {
    int fd;       /* -1: this rank, or closed */
    Out* out;     /* frames still to write, oldest first */
    char* in;     /* bytes read and not yet parsed into frames */
    size_t in_len, in_cap;
} Peer;

struct MiniRequest {
    int is_recv, done;
    void* buf;
    int count, src, tag;
};

enum { kTagReduce = -101, kTagResult = -102 };

static int g_rank = 0, g_size = 1;
static Peer* g_peers = NULL;
static Frame* g_inbox = NULL;   /* arrived frames not yet received, oldest first */
static double g_timeout = 120.0;

static void fail(const char* what)
{
    fprintf(stderr, "minimpi rank %d: %s (%s)\n", g_rank, what, errno ? strerror(errno) : "");
    exit(3);
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void sock_path(struct sockaddr_un* a, const char* dir, int rank)
{
    memset(a, 0, sizeof(*a));
    a->sun_family = AF_UNIX;
    if ((size_t)snprintf(a->sun_path, sizeof(a->sun_path), "%s/%d.sock", dir, rank) >= sizeof(a->sun_path))
        fail("socket path too long");
}

static void blocking_io(int fd, void* p, size_t n, int writing)
{
    char* c = (char*)p;
    while (n > 0) {
        ssize_t k = writing ? write(fd, c, n) : read(fd, c, n);
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0) fail(writing ? "hello write" : "hello read");
        c += k;
        n -= (size_t)k;
    }
}

int MPI_Init(int* argc, char*** argv)
{
    (void)argc;
    (void)argv;
    const char* r = getenv("MINIMPI_RANK");
    const char* s = getenv("MINIMPI_SIZE");
    const char* dir = getenv("MINIMPI_DIR");
    const char* t = getenv("MINIMPI_TIMEOUT");
    if (t) g_timeout = atof(t);
    if (r && s && dir) {
        g_rank = atoi(r);
        g_size = atoi(s);
    }
    if (g_size < 1 || g_rank < 0 || g_rank >= g_size) fail("bad MINIMPI_RANK / MINIMPI_SIZE");
    g_peers = (Peer*)calloc((size_t)g_size, sizeof(Peer));
    for (int p = 0; p < g_size; ++p) g_peers[p].fd = -1;
    if (g_size == 1) return 0;

    struct sockaddr_un a;
    sock_path(&a, dir, g_rank);
    unlink(a.sun_path);
    int ls = socket(AF_UNIX, SOCK_STREAM, 0);
    if (ls < 0 || bind(ls, (struct sockaddr*)&a, sizeof(a)) < 0 || listen(ls, g_size) < 0) fail("listen");
    for (int p = 0; p < g_rank; ++p) {   /* connect to every lower rank */
        struct sockaddr_un pa;
        sock_path(&pa, dir, p);
        const double t0 = now_s();
        int fd = -1;
        for (;;) {
            fd = socket(AF_UNIX, SOCK_STREAM, 0);
            if (fd < 0) fail("socket");
            if (connect(fd, (struct sockaddr*)&pa, sizeof(pa)) == 0) break;
            close(fd);
            if (now_s() - t0 > g_timeout) fail("connect timed out");
            struct timespec d = {0, 10 * 1000 * 1000};
            nanosleep(&d, NULL);
        }
        blocking_io(fd, &g_rank, sizeof(int), 1);
        g_peers[p].fd = fd;
    }
    for (int k = g_rank + 1; k < g_size; ++k) {   /* accept every higher rank */
        struct pollfd pf = {ls, POLLIN, 0};
        if (poll(&pf, 1, (int)(g_timeout * 1000.0)) <= 0) fail("accept timed out");
        int fd = accept(ls, NULL, NULL);
        if (fd < 0) fail("accept");
        int who = -1;
        blocking_io(fd, &who, sizeof(int), 0);
        if (who <= g_rank || who >= g_size || g_peers[who].fd >= 0) fail("unexpected peer");
        g_peers[who].fd = fd;
    }
    close(ls);
    unlink(a.sun_path);
    for (int p = 0; p < g_size; ++p)
        if (g_peers[p].fd >= 0) fcntl(g_peers[p].fd, F_SETFL, fcntl(g_peers[p].fd, F_GETFL) | O_NONBLOCK);
    return 0;
}

int MPI_Comm_rank(MPI_Comm comm, int* rank)
{
    (void)comm;
    *rank = g_rank;
    return 0;
}

int MPI_Comm_size(MPI_Comm comm, int* size)
{
    (void)comm;
    *size = g_size;
    return 0;
}

/* -- frames and the progress loop ------------------------------------------------ */

static void enqueue(int dest, int tag, int count, const double* data)
{
    if (dest < 0 || dest >= g_size || dest == g_rank || g_peers[dest].fd < 0) fail("send to a bad rank");
    Out* o = (Out*)malloc(sizeof(Out));
    o->len = 2 * sizeof(int) + (size_t)count * sizeof(double);
    o->bytes = (char*)malloc(o->len);
    memcpy(o->bytes, &tag, sizeof(int));
    memcpy(o->bytes + sizeof(int), &count, sizeof(int));
    if (count > 0) memcpy(o->bytes + 2 * sizeof(int), data, (size_t)count * sizeof(double));
    o->off = 0;
    o->next = NULL;
    Out** tail = &g_peers[dest].out;
    while (*tail) tail = &(*tail)->next;
    *tail = o;
}

static void take_frames(int src)
{
    Peer* p = &g_peers[src];
    size_t pos = 0;
    while (p->in_len - pos >= 2 * sizeof(int)) {
        int tag, count;
        memcpy(&tag, p->in + pos, sizeof(int));
        memcpy(&count, p->in + pos + sizeof(int), sizeof(int));
        const size_t need = 2 * sizeof(int) + (size_t)count * sizeof(double);
        if (p->in_len - pos < need) break;
        Frame* f = (Frame*)malloc(sizeof(Frame));
        f->src = src;
        f->tag = tag;
        f->count = count;
        f->data = (double*)malloc((size_t)(count > 0 ? count : 1) * sizeof(double));
        if (count > 0) memcpy(f->data, p->in + pos + 2 * sizeof(int), (size_t)count * sizeof(double));
        f->next = NULL;
        Frame** tail = &g_inbox;
        while (*tail) tail = &(*tail)->next;
        *tail = f;
        pos += need;
    }
    memmove(p->in, p->in + pos, p->in_len - pos);
    p->in_len -= pos;
}

/* One pass: write what the sockets take, read what has arrived (waiting up
 * to timeout_ms for either). */
static void progress(int timeout_ms)
{
    struct pollfd fds[g_size > 1 ? g_size : 1];
    int who[g_size > 1 ? g_size : 1];
    int n = 0;
    for (int p = 0; p < g_size; ++p) {
        if (g_peers[p].fd < 0) continue;
        fds[n].fd = g_peers[p].fd;
        fds[n].events = (short)(POLLIN | (g_peers[p].out ? POLLOUT : 0));
        fds[n].revents = 0;
        who[n++] = p;
    }
    if (n == 0) return;
    if (poll(fds, (nfds_t)n, timeout_ms) < 0) {
        if (errno == EINTR) return;
        fail("poll");
    }
    for (int k = 0; k < n; ++k) {
        Peer* p = &g_peers[who[k]];
        if (fds[k].revents & POLLOUT) {
            while (p->out) {
                Out* o = p->out;
                ssize_t w = write(p->fd, o->bytes + o->off, o->len - o->off);
                if (w < 0) {
                    if (errno == EAGAIN || errno == EWOULDBLOCK || errno == EINTR) break;
                    fail("write");
                }
                o->off += (size_t)w;
                if (o->off < o->len) break;
                p->out = o->next;
                free(o->bytes);
                free(o);
            }
        }
        if (fds[k].revents & (POLLIN | POLLHUP | POLLERR)) {
            for (;;) {
                if (p->in_cap - p->in_len < 65536) {
                    p->in_cap = p->in_cap * 2 + 65536;
                    p->in = (char*)realloc(p->in, p->in_cap);
                }
                ssize_t r = read(p->fd, p->in + p->in_len, p->in_cap - p->in_len);
                if (r > 0) {
                    p->in_len += (size_t)r;
                    continue;
                }
                if (r == 0) {   /* the peer has finished and closed */
                    close(p->fd);
                    p->fd = -1;
                    break;
                }
                if (errno == EAGAIN || errno == EWOULDBLOCK) break;
                if (errno == EINTR) continue;
                fail("read");
            }
            take_frames(who[k]);
        }
    }
}

static int match(struct MiniRequest* q)
{
    for (Frame** pp = &g_inbox; *pp; pp = &(*pp)->next) {
        Frame* f = *pp;
        if (f->src != q->src || f->tag != q->tag) continue;
        if (f->count > q->count) fail("message longer than its receive");
        memcpy(q->buf, f->data, (size_t)f->count * sizeof(double));
        *pp = f->next;
        free(f->data);
        free(f);
        q->done = 1;
        return 1;
    }
    return 0;
}

static void wait_requests(int count, struct MiniRequest** reqs)
{
    const double t0 = now_s();
    for (;;) {
        int pending = 0;
        for (int i = 0; i < count; ++i) {
            struct MiniRequest* q = reqs[i];
            if (!q || q->done) continue;
            if (q->is_recv && match(q)) continue;
            if (q->is_recv && g_peers[q->src].fd < 0) fail("receive from a rank that has closed");
            ++pending;
        }
        if (!pending) return;
        if (now_s() - t0 > g_timeout) fail("wait timed out");
        progress(50);
    }
}

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request* request)
{
    (void)comm;
    if (type != MPI_DOUBLE) fail("only MPI_DOUBLE");
    enqueue(dest, tag, count, (const double*)buf);
    struct MiniRequest* q = (struct MiniRequest*)calloc(1, sizeof(struct MiniRequest));
    q->done = 1;   /* the data is copied: the send buffer may be reused */
    *request = q;
    progress(0);
    return 0;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* request)
{
    (void)comm;
    if (type != MPI_DOUBLE) fail("only MPI_DOUBLE");
    if (source < 0 || source >= g_size || source == g_rank) fail("receive from a bad rank");
    struct MiniRequest* q = (struct MiniRequest*)calloc(1, sizeof(struct MiniRequest));
    q->is_recv = 1;
    q->buf = buf;
    q->count = count;
    q->src = source;
    q->tag = tag;
    *request = q;
    return 0;
}

int MPI_Waitall(int count, MPI_Request* requests, MPI_Status* statuses)
{
    (void)statuses;
    wait_requests(count, requests);
    for (int i = 0; i < count; ++i) {
        free(requests[i]);
        requests[i] = NULL;
    }
    return 0;
}

static void recv_now(int src, int tag, double* buf, int count)
{
    struct MiniRequest q = {1, 0, buf, count, src, tag};
    struct MiniRequest* p = &q;
    wait_requests(1, &p);
}

/* Rank 0 folds the ranks' values in rank order (SUM: ((v0 + v1) + v2) + ...;
 * MIN: the least) and sends the result back to every rank. */
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)comm;
    if (type != MPI_DOUBLE || (op != MPI_SUM && op != MPI_MIN)) fail("only MPI_DOUBLE with MPI_SUM or MPI_MIN");
    double* acc = (double*)malloc((size_t)(count > 0 ? count : 1) * sizeof(double));
    memcpy(acc, sendbuf, (size_t)count * sizeof(double));
    if (g_rank == 0) {
        double* v = (double*)malloc((size_t)(count > 0 ? count : 1) * sizeof(double));
        for (int r = 1; r < g_size; ++r) {
            recv_now(r, kTagReduce, v, count);
            for (int k = 0; k < count; ++k) acc[k] = (op == MPI_SUM) ? acc[k] + v[k] : (v[k] < acc[k] ? v[k] : acc[k]);
        }
        free(v);
        for (int r = 1; r < g_size; ++r) enqueue(r, kTagResult, count, acc);
        progress(0);
    } else {
        enqueue(0, kTagReduce, count, acc);
        recv_now(0, kTagResult, acc, count);
    }
    memcpy(recvbuf, acc, (size_t)count * sizeof(double));
    free(acc);
    return 0;
}

int MPI_Barrier(MPI_Comm comm)
{
    double zero = 0.0, out = 0.0;
    return MPI_Allreduce(&zero, &out, 1, MPI_DOUBLE, MPI_SUM, comm);
}

/* Writes every queued frame, then closes the streams. */
int MPI_Finalize(void)
{
    const double t0 = now_s();
    for (;;) {
        int queued = 0;
        for (int p = 0; p < g_size; ++p) queued |= g_peers[p].fd >= 0 && g_peers[p].out != NULL;
        if (!queued) break;
        if (now_s() - t0 > g_timeout) fail("finalize timed out");
        progress(50);
    }
    for (int p = 0; p < g_size; ++p)
        if (g_peers[p].fd >= 0) close(g_peers[p].fd);
    return 0;
}

int MPI_Abort(MPI_Comm comm, int code)
{
    (void)comm;
    exit(code ? code : 1);
}
