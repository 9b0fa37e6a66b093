// Thread-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY.
//
// The program's main() is compiled as s2l_rank_main() (-Dmain=s2l_rank_main on the file that
// defines it); the real main() below starts S2L_NP threads (default 1), each one an MPI rank of
// MPI_COMM_WORLD, and returns the largest exit code.
#include "mpi.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <pthread.h>
#include <vector>

int s2l_rank_main(int argc, char** argv);

namespace {

thread_local int tl_world = 0;

struct Msg {
    int src, tag;
    std::vector<char> data;
};

struct Box {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Msg> q;
};

}  // namespace

struct s2l_mpi_comm {
    int size = 0;
    std::vector<int> world;            // world rank of every member
    std::vector<std::unique_ptr<Box>> box;
    // collective slots
    std::mutex bm;
    std::condition_variable bcv;
    int arrived = 0;
    long gen = 0;
    std::vector<const void*> p0, p1, p2, p3;
    std::vector<long> v0, v1;
    std::vector<s2l_mpi_comm*> made;

    explicit s2l_mpi_comm(std::vector<int> members) : size((int)members.size()), world(std::move(members))
    {
        for (int i = 0; i < size; ++i) box.emplace_back(new Box);
        p0.assign(size, nullptr);
        p1.assign(size, nullptr);
        p2.assign(size, nullptr);
        p3.assign(size, nullptr);
        v0.assign(size, 0);
        v1.assign(size, 0);
        made.assign(size, nullptr);
    }
    int rank() const
    {
        for (int i = 0; i < size; ++i)
            if (world[i] == tl_world) return i;
        return -1;
    }
    void barrier()
    {
        std::unique_lock<std::mutex> g(bm);
        const long my = gen;
        if (++arrived == size) {
            arrived = 0;
            ++gen;
            bcv.notify_all();
        } else {
            bcv.wait(g, [&] { return gen != my; });
        }
    }
};

struct s2l_mpi_request {
    void* buf;
    size_t bytes;
    int src, tag;
    MPI_Comm comm;
};

namespace {

s2l_mpi_comm* g_world = nullptr;

size_t tsize(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR:
    case MPI_BYTE: return 1;
    case MPI_INT:
    case MPI_UNSIGNED:
    case MPI_FLOAT:
    case MPI_INT32_T: return 4;
    default: return 8;
    }
}

template <typename T>
void red(T* acc, const T* x, int n, MPI_Op op)
{
    for (int i = 0; i < n; ++i) {
        if (op == MPI_SUM) acc[i] += x[i];
        else if (op == MPI_MAX) acc[i] = std::max(acc[i], x[i]);
        else acc[i] = std::min(acc[i], x[i]);
    }
}

void reduce_into(void* acc, const void* x, int n, MPI_Datatype t, MPI_Op op)
{
    switch (t) {
    case MPI_INT:
    case MPI_INT32_T: red((int32_t*)acc, (const int32_t*)x, n, op); break;
    case MPI_UNSIGNED: red((uint32_t*)acc, (const uint32_t*)x, n, op); break;
    case MPI_LONG:
    case MPI_LONG_LONG:
    case MPI_INT64_T: red((int64_t*)acc, (const int64_t*)x, n, op); break;
    case MPI_UNSIGNED_LONG:
    case MPI_UNSIGNED_LONG_LONG:
    case MPI_UINT64_T: red((uint64_t*)acc, (const uint64_t*)x, n, op); break;
    case MPI_DOUBLE: red((double*)acc, (const double*)x, n, op); break;
    case MPI_FLOAT: red((float*)acc, (const float*)x, n, op); break;
    case MPI_CHAR:
    case MPI_BYTE: red((char*)acc, (const char*)x, n, op); break;
    default: std::fprintf(stderr, "mpi shim: unsupported datatype in reduction\n"); std::abort();
    }
}

void post(MPI_Comm c, int dst_rank, int tag, const void* buf, size_t bytes)
{
    Box& b = *c->box[dst_rank];
    Msg m;
    m.src = c->rank();
    m.tag = tag;
    m.data.assign((const char*)buf, (const char*)buf + bytes);
    {
        std::lock_guard<std::mutex> g(b.mu);
        b.q.push_back(std::move(m));
    }
    b.cv.notify_all();
}

void take(MPI_Comm c, int src, int tag, void* buf, size_t maxbytes, MPI_Status* st)
{
    Box& b = *c->box[c->rank()];
    std::unique_lock<std::mutex> g(b.mu);
    for (;;) {
        for (auto it = b.q.begin(); it != b.q.end(); ++it) {
            if ((src == MPI_ANY_SOURCE || it->src == src) && (tag == MPI_ANY_TAG || it->tag == tag)) {
                if (it->data.size() > maxbytes) {
                    std::fprintf(stderr, "mpi shim: message truncated (%zu > %zu bytes)\n", it->data.size(), maxbytes);
                    std::abort();
                }
                std::memcpy(buf, it->data.data(), it->data.size());
                if (st) {
                    st->MPI_SOURCE = it->src;
                    st->MPI_TAG = it->tag;
                    st->MPI_ERROR = 0;
                    st->count_bytes = (int)it->data.size();
                }
                b.q.erase(it);
                return;
            }
        }
        b.cv.wait(g);
    }
}

struct Launch {
    int rank, argc;
    char** argv;
    int code;
};

void* rank_thread(void* p)
{
    Launch* l = (Launch*)p;
    tl_world = l->rank;
    l->code = s2l_rank_main(l->argc, l->argv);
    return nullptr;
}

}  // namespace

extern "C" {

MPI_Comm s2l_mpi_comm_world(void) { return g_world; }
int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code)
{
    std::fflush(stdout);
    std::fflush(stderr);
    std::_Exit(code ? code : 1);
}
double MPI_Wtime(void)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
int MPI_Comm_rank(MPI_Comm c, int* r)
{
    *r = c->rank();
    return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm c, int* s)
{
    *s = c->size;
    return MPI_SUCCESS;
}
MPI_Fint MPI_Comm_c2f(MPI_Comm) { return 0; }

int MPI_Barrier(MPI_Comm c)
{
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm* out)
{
    const int r = c->rank();
    c->v0[r] = color;
    c->v1[r] = key;
    c->barrier();
    // the smallest rank of every color builds the new communicator
    bool leader = color != MPI_UNDEFINED;
    for (int q = 0; q < r && leader; ++q) leader = c->v0[q] != color;
    if (leader) {
        std::vector<std::pair<std::pair<long, int>, int>> mem;
        for (int q = 0; q < c->size; ++q)
            if (c->v0[q] == color) mem.push_back({{c->v1[q], q}, c->world[q]});
        std::sort(mem.begin(), mem.end());
        std::vector<int> w;
        for (auto& m : mem) w.push_back(m.second);
        c->made[r] = new s2l_mpi_comm(w);
    }
    c->barrier();
    if (color == MPI_UNDEFINED) {
        *out = MPI_COMM_NULL;
    } else {
        int lead = 0;
        while (c->v0[lead] != color) ++lead;
        *out = c->made[lead];
    }
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm* c)
{
    *c = MPI_COMM_NULL;  // communicators live until exit
    return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm c)
{
    const int r = c->rank();
    if (r == root) c->p0[root] = buf;
    c->barrier();
    if (r != root) std::memcpy(buf, c->p0[root], count * tsize(t));
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    const int r = c->rank();
    const size_t b = count * tsize(t);
    c->p0[r] = (sbuf == MPI_IN_PLACE) ? rbuf : sbuf;
    c->barrier();
    std::vector<char> acc((const char*)c->p0[0], (const char*)c->p0[0] + b);
    for (int q = 1; q < c->size; ++q) reduce_into(acc.data(), c->p0[q], count, t, op);
    c->barrier();
    std::memcpy(rbuf, acc.data(), b);
    return MPI_SUCCESS;
}

int MPI_Reduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    const int r = c->rank();
    const size_t b = count * tsize(t);
    c->p0[r] = (sbuf == MPI_IN_PLACE) ? rbuf : sbuf;
    c->barrier();
    std::vector<char> acc;
    if (r == root) {
        acc.assign((const char*)c->p0[0], (const char*)c->p0[0] + b);
        for (int q = 1; q < c->size; ++q) reduce_into(acc.data(), c->p0[q], count, t, op);
    }
    c->barrier();
    if (r == root) std::memcpy(rbuf, acc.data(), b);
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, const int* rcounts, const int* displs,
                MPI_Datatype rt, int root, MPI_Comm c)
{
    const int r = c->rank();
    c->p0[r] = sbuf;
    c->v0[r] = (long)(scount * tsize(st));
    c->barrier();
    if (r == root)
        for (int q = 0; q < c->size; ++q)
            if (!(q == root && sbuf == MPI_IN_PLACE))
                std::memcpy((char*)rbuf + displs[q] * tsize(rt), c->p0[q], (size_t)rcounts[q] * tsize(rt));
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Gather(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt, int root,
               MPI_Comm c)
{
    std::vector<int> cnt(c->size, rcount), dsp(c->size);
    for (int q = 0; q < c->size; ++q) dsp[q] = q * rcount;
    return MPI_Gatherv(sbuf, scount, st, rbuf, cnt.data(), dsp.data(), rt, root, c);
}

int MPI_Scatterv(const void* sbuf, const int* scounts, const int* displs, MPI_Datatype st, void* rbuf, int rcount,
                 MPI_Datatype rt, int root, MPI_Comm c)
{
    const int r = c->rank();
    if (r == root) {
        c->p0[root] = sbuf;
        c->p1[root] = scounts;
        c->p2[root] = displs;
    }
    c->barrier();
    if (!(r == root && rbuf == MPI_IN_PLACE)) {
        const int* sc = (const int*)c->p1[root];
        const int* dp = (const int*)c->p2[root];
        const size_t b = std::min((size_t)sc[r] * tsize(st), (size_t)rcount * tsize(rt));
        std::memcpy(rbuf, (const char*)c->p0[root] + dp[r] * tsize(st), b);
    }
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Allgatherv(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, const int* rcounts, const int* displs,
                   MPI_Datatype rt, MPI_Comm c)
{
    const int r = c->rank();
    std::vector<char> mine;
    if (sbuf == MPI_IN_PLACE) {
        mine.assign((const char*)rbuf + displs[r] * tsize(rt), (const char*)rbuf + (displs[r] + rcounts[r]) * tsize(rt));
        c->p0[r] = mine.data();
    } else {
        c->p0[r] = sbuf;
    }
    (void)scount;
    (void)st;
    c->barrier();
    std::vector<char> out((size_t)(displs[c->size - 1] + rcounts[c->size - 1]) * tsize(rt));
    for (int q = 0; q < c->size; ++q)
        std::memcpy(out.data() + displs[q] * tsize(rt), c->p0[q], (size_t)rcounts[q] * tsize(rt));
    c->barrier();
    for (int q = 0; q < c->size; ++q)
        std::memcpy((char*)rbuf + displs[q] * tsize(rt), out.data() + displs[q] * tsize(rt), (size_t)rcounts[q] * tsize(rt));
    return MPI_SUCCESS;
}

int MPI_Allgather(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt,
                  MPI_Comm c)
{
    std::vector<int> cnt(c->size, rcount), dsp(c->size);
    for (int q = 0; q < c->size; ++q) dsp[q] = q * rcount;
    return MPI_Allgatherv(sbuf, scount, st, rbuf, cnt.data(), dsp.data(), rt, c);
}

int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype st, void* rbuf,
                  const int* rcounts, const int* rdispls, MPI_Datatype rt, MPI_Comm c)
{
    const int r = c->rank();
    c->p0[r] = sbuf;
    c->p1[r] = scounts;
    c->p2[r] = sdispls;
    c->barrier();
    for (int q = 0; q < c->size; ++q) {
        const int* sc = (const int*)c->p1[q];
        const int* sd = (const int*)c->p2[q];
        const size_t b = (size_t)sc[r] * tsize(st);
        if (b > (size_t)rcounts[q] * tsize(rt)) {
            std::fprintf(stderr, "mpi shim: alltoallv truncation\n");
            std::abort();
        }
        std::memcpy((char*)rbuf + rdispls[q] * tsize(rt), (const char*)c->p0[q] + sd[r] * tsize(st), b);
    }
    c->barrier();
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void* sbuf, int scount, MPI_Datatype st, void* rbuf, int rcount, MPI_Datatype rt, MPI_Comm c)
{
    std::vector<int> sc(c->size, scount), sd(c->size), rc(c->size, rcount), rd(c->size);
    for (int q = 0; q < c->size; ++q) {
        sd[q] = q * scount;
        rd[q] = q * rcount;
    }
    return MPI_Alltoallv(sbuf, sc.data(), sd.data(), st, rbuf, rc.data(), rd.data(), rt, c);
}

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    post(c, dest, tag, buf, (size_t)count * tsize(t));
    return MPI_SUCCESS;
}

int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status* st)
{
    take(c, src, tag, buf, (size_t)count * tsize(t), st);
    return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request* req)
{
    post(c, dest, tag, buf, (size_t)count * tsize(t));
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request* req)
{
    *req = new s2l_mpi_request{buf, (size_t)count * tsize(t), src, tag, c};
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* sts)
{
    for (int i = 0; i < count; ++i) {
        if (reqs[i] == MPI_REQUEST_NULL) continue;
        s2l_mpi_request* q = reqs[i];
        take(q->comm, q->src, q->tag, q->buf, q->bytes, sts ? &sts[i] : nullptr);
        delete q;
        reqs[i] = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}

}  // extern "C"

int main(int argc, char** argv)
{
    const char* e = std::getenv("S2L_NP");
    const int np = e ? std::max(1, std::atoi(e)) : 1;
    std::vector<int> w(np);
    for (int i = 0; i < np; ++i) w[i] = i;
    g_world = new s2l_mpi_comm(w);
    std::vector<Launch> ls(np);
    std::vector<pthread_t> th(np);
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, (size_t)64 << 20);
    for (int i = 0; i < np; ++i) {
        ls[i] = {i, argc, argv, 0};
        if (pthread_create(&th[i], &attr, rank_thread, &ls[i]) != 0) {
            std::fprintf(stderr, "mpi shim: cannot start rank thread %d\n", i);
            return 1;
        }
    }
    int code = 0;
    for (int i = 0; i < np; ++i) {
        pthread_join(th[i], nullptr);
        code = std::max(code, ls[i].code);
    }
    return code;
}
