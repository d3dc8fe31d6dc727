// In-process MPI test double (see include/mpi.h).  Each virtual rank is a host
// thread started by fake_mpi_run(); sends are eager (packed at post time), so a
// send request is complete as soon as it is posted and only receives wait.
//
// ANY_SOURCE matching of MPI_Isendrecv_replace: the reference's Cannon step loop
// (src/25DCannon.cpp:305,310,341,344) receives each round's tile with
// MPI_ANY_SOURCE and the same tag in every round, so under real MPI a fast
// neighbour's round-r+1 tile can match a slow rank's round-r receive.  The
// double removes that race by numbering each rank's Isendrecv_replace calls per
// tag ("epoch") and matching a receive only with a send of the same epoch, which
// is the schedule the reference intends.
#include "mpi.h"

#include "host_pool.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

struct fake_comm_s {
    int context;
    std::vector<int> members;  // comm rank -> world rank
};

struct fake_request_s {
    bool done = false;
    bool is_recv = false;
    void* buf = nullptr;
    int count = 0;
    MPI_Datatype type = MPI_BYTE;
    int context = 0;
    int src = 0;  // comm rank or MPI_ANY_SOURCE
    int dst = 0;  // my comm rank
    int tag = 0;
    int epoch = -1;
};

namespace {

struct Message {
    int context, src, dst, tag, epoch;
    PoolBytes bytes;  // packed payload (pool memory: no zero fill, no fresh pages per message)
};

struct TypeInfo {
    int count, blocklen, stride;
    size_t elem;
};

struct FakeAbort : std::runtime_error {
    explicit FakeAbort(const std::string& s) : std::runtime_error(s) {}
};

// internal tags (negative, never used by the reference)
constexpr int TAG_SPLIT = -100, TAG_SPLIT_REPLY = -101, TAG_BCAST = -102, TAG_REDUCE = -103, TAG_BARRIER = -104,
              TAG_BARRIER_REL = -105;

struct Job {
    int size = 0;
    fake_comm_s* world = nullptr;
    std::mutex m;
    std::condition_variable cv;
    std::deque<Message> mailbox;
    std::vector<fake_comm_s*> comms;  // owned
    std::atomic<int> next_context{1};
    bool aborted = false;
    std::string abort_reason;
    double wait_limit_s = 60.0;
};

Job* g_job = nullptr;
thread_local int tl_world_rank = -1;
thread_local std::map<std::pair<int, int>, int> tl_epochs;  // (context, tag) -> next epoch

std::mutex g_type_mutex;
std::vector<TypeInfo> g_types;  // derived types, handle = 100 + index

size_t predefined_size(MPI_Datatype t) {
    switch (t) {
        case MPI_BYTE: return 1;
        case MPI_INT: return 4;
        case MPI_FLOAT: return 4;
        case MPI_DOUBLE: return 8;
        case MPI_LONG_LONG: return 8;
        default: return 0;
    }
}

TypeInfo type_info(MPI_Datatype t) {
    if (t < 100) return TypeInfo{1, 1, 1, predefined_size(t)};
    std::lock_guard<std::mutex> g(g_type_mutex);
    return g_types.at(t - 100);
}

// extent in elements of one instance of the type
long long type_extent(const TypeInfo& ti) { return (long long)(ti.count - 1) * ti.stride + ti.blocklen; }

PoolBytes pack(const void* buf, int count, MPI_Datatype type) {
    TypeInfo ti = type_info(type);
    PoolBytes out((size_t)count * ti.count * ti.blocklen * ti.elem);
    if (!out.data()) throw FakeAbort("out of host memory for a message");
    const unsigned char* b = static_cast<const unsigned char*>(buf);
    if (ti.count == 1 || ti.stride == ti.blocklen) {  // contiguous: one copy
        host_copy(out.data(), b, out.size());
        return out;
    }
    size_t o = 0;
    for (int c = 0; c < count; ++c) {
        const unsigned char* base = b + (size_t)c * type_extent(ti) * ti.elem;
        for (int v = 0; v < ti.count; ++v) {
            size_t n = (size_t)ti.blocklen * ti.elem;
            std::memcpy(out.data() + o, base + (size_t)v * ti.stride * ti.elem, n);
            o += n;
        }
    }
    return out;
}

void unpack(const PoolBytes& in, void* buf, int count, MPI_Datatype type) {
    TypeInfo ti = type_info(type);
    size_t need = (size_t)count * ti.count * ti.blocklen * ti.elem;
    if (in.size() != need) throw FakeAbort("message size mismatch");
    unsigned char* b = static_cast<unsigned char*>(buf);
    if (ti.count == 1 || ti.stride == ti.blocklen) {  // contiguous: one copy
        host_copy(b, in.data(), need);
        return;
    }
    size_t o = 0;
    for (int c = 0; c < count; ++c) {
        unsigned char* base = b + (size_t)c * type_extent(ti) * ti.elem;
        for (int v = 0; v < ti.count; ++v) {
            size_t n = (size_t)ti.blocklen * ti.elem;
            std::memcpy(base + (size_t)v * ti.stride * ti.elem, in.data() + o, n);
            o += n;
        }
    }
}

int comm_rank_of(MPI_Comm comm, int world_rank) {
    for (size_t i = 0; i < comm->members.size(); ++i)
        if (comm->members[i] == world_rank) return (int)i;
    return -1;
}

void check_abort_locked() {
    if (g_job->aborted) throw FakeAbort("aborted: " + g_job->abort_reason);
}

void post_message(Message&& msg) {
    std::lock_guard<std::mutex> g(g_job->m);
    check_abort_locked();
    g_job->mailbox.push_back(std::move(msg));
    g_job->cv.notify_all();
}

// Try to complete a receive request; caller holds the lock.
bool try_match_locked(fake_request_s* r, MPI_Status* st) {
    for (auto it = g_job->mailbox.begin(); it != g_job->mailbox.end(); ++it) {
        if (it->context != r->context || it->dst != r->dst || it->tag != r->tag || it->epoch != r->epoch) continue;
        if (r->src != MPI_ANY_SOURCE && it->src != r->src) continue;
        unpack(it->bytes, r->buf, r->count, r->type);
        if (st) {
            st->MPI_SOURCE = it->src;
            st->MPI_TAG = it->tag;
            st->MPI_ERROR = 0;
        }
        g_job->mailbox.erase(it);
        r->done = true;
        return true;
    }
    return false;
}

fake_request_s* make_recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, int epoch) {
    auto* r = new fake_request_s;
    r->is_recv = true;
    r->buf = buf;
    r->count = count;
    r->type = type;
    r->context = comm->context;
    r->src = source;
    r->dst = comm_rank_of(comm, tl_world_rank);
    r->tag = tag;
    r->epoch = epoch;
    return r;
}

void send_msg(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, int epoch) {
    Message m;
    m.context = comm->context;
    m.src = comm_rank_of(comm, tl_world_rank);
    m.dst = dest;
    m.tag = tag;
    m.epoch = epoch;
    m.bytes = pack(buf, count, type);
    post_message(std::move(m));
}

void wait_one(fake_request_s* r, MPI_Status* st) {
    if (r->done) return;
    std::unique_lock<std::mutex> lk(g_job->m);
    auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(g_job->wait_limit_s);
    while (true) {
        check_abort_locked();
        if (try_match_locked(r, st)) return;
        if (g_job->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
            g_job->aborted = true;
            g_job->abort_reason = "receive wait exceeded its limit (deadlock in the rank program)";
            g_job->cv.notify_all();
            throw FakeAbort(g_job->abort_reason);
        }
    }
}

void recv_blocking(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm) {
    fake_request_s* r = make_recv(buf, count, type, source, tag, comm, -1);
    wait_one(r, nullptr);
    delete r;
}

}  // namespace

extern "C" {

MPI_Comm fake_mpi_comm_world(void) { return g_job ? g_job->world : nullptr; }

}  // extern "C"

int fake_mpi_world_rank(void) { return tl_world_rank; }

extern "C" {

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
    *rank = comm_rank_of(comm, tl_world_rank);
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int* size) {
    *size = (int)comm->members.size();
    return MPI_SUCCESS;
}

// Collective: members send (color, key) to comm rank 0, which builds the groups
// (ordered by key, then by old rank, as MPI specifies) and replies with the new comm.
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm) {
    int me = comm_rank_of(comm, tl_world_rank);
    int n = (int)comm->members.size();
    int ck[2] = {color, key};
    send_msg(ck, 2, MPI_INT, 0, TAG_SPLIT, comm, -1);
    if (me == 0) {
        std::vector<std::array<int, 3>> all(n);
        for (int r = 0; r < n; ++r) {
            int got[2];
            recv_blocking(got, 2, MPI_INT, r, TAG_SPLIT, comm);
            all[r] = {got[0], got[1], r};
        }
        std::map<int, std::vector<std::array<int, 3>>> groups;
        for (auto& a : all) groups[a[0]].push_back(a);
        std::vector<fake_comm_s*> result(n, nullptr);
        for (auto& kv : groups) {
            auto v = kv.second;
            std::stable_sort(v.begin(), v.end(), [](const std::array<int, 3>& x, const std::array<int, 3>& y) {
                return x[1] != y[1] ? x[1] < y[1] : x[2] < y[2];
            });
            auto* c = new fake_comm_s;
            c->context = g_job->next_context.fetch_add(1);
            for (auto& a : v) c->members.push_back(comm->members[a[2]]);
            {
                std::lock_guard<std::mutex> g(g_job->m);
                g_job->comms.push_back(c);
            }
            for (auto& a : v) result[a[2]] = (kv.first == MPI_UNDEFINED) ? nullptr : c;
        }
        for (int r = 0; r < n; ++r) {
            unsigned long long p = (unsigned long long)(uintptr_t)result[r];
            send_msg(&p, 1, MPI_LONG_LONG, r, TAG_SPLIT_REPLY, comm, -1);
        }
    }
    unsigned long long p = 0;
    recv_blocking(&p, 1, MPI_LONG_LONG, 0, TAG_SPLIT_REPLY, comm);
    *newcomm = (MPI_Comm)(uintptr_t)p;
    return MPI_SUCCESS;
}

int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype* newtype) {
    if (oldtype >= 100) return MPI_ERR_OTHER;
    std::lock_guard<std::mutex> g(g_type_mutex);
    g_types.push_back(TypeInfo{count, blocklength, stride, predefined_size(oldtype)});
    *newtype = 100 + (int)g_types.size() - 1;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req) {
    send_msg(buf, count, type, dest, tag, comm, -1);
    auto* r = new fake_request_s;
    r->done = true;
    *req = r;
    return MPI_SUCCESS;
}

int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req) {
    *req = make_recv(buf, count, type, source, tag, comm, -1);
    return MPI_SUCCESS;
}

int MPI_Isendrecv_replace(void* buf, int count, MPI_Datatype type, int dest, int sendtag, int source, int recvtag,
                          MPI_Comm comm, MPI_Request* req) {
    int epoch_s = tl_epochs[{comm->context, sendtag}]++;
    send_msg(buf, count, type, dest, sendtag, comm, epoch_s);
    int epoch_r = (recvtag == sendtag) ? epoch_s : tl_epochs[{comm->context, recvtag}]++;
    *req = make_recv(buf, count, type, source, recvtag, comm, epoch_r);
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void* recvbuf,
                 int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status* status) {
    send_msg(sendbuf, sendcount, sendtype, dest, sendtag, comm, -1);
    fake_request_s* r = make_recv(recvbuf, recvcount, recvtype, source, recvtag, comm, -1);
    wait_one(r, status);
    delete r;
    return MPI_SUCCESS;
}

int MPI_Waitany(int count, MPI_Request* reqs, int* index, MPI_Status* status) {
    // complete the first request (in posting order) that can complete, else wait
    std::unique_lock<std::mutex> lk(g_job->m);
    auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(g_job->wait_limit_s);
    while (true) {
        check_abort_locked();
        bool any_active = false;
        for (int i = 0; i < count; ++i) {
            fake_request_s* r = reqs[i];
            if (!r) continue;
            any_active = true;
            if (r->done || try_match_locked(r, status)) {
                delete r;
                reqs[i] = nullptr;
                *index = i;
                return MPI_SUCCESS;
            }
        }
        if (!any_active) {
            *index = MPI_UNDEFINED;
            return MPI_SUCCESS;
        }
        if (g_job->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
            g_job->aborted = true;
            g_job->abort_reason = "MPI_Waitany exceeded its limit";
            g_job->cv.notify_all();
            throw FakeAbort(g_job->abort_reason);
        }
    }
}

int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status*) {
    for (int i = 0; i < count; ++i) {
        if (!reqs[i]) continue;
        wait_one(reqs[i], nullptr);
        delete reqs[i];
        reqs[i] = nullptr;
    }
    return MPI_SUCCESS;
}

int MPI_Ibcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request* req) {
    int me = comm_rank_of(comm, tl_world_rank);
    if (me == root) {
        for (int r = 0; r < (int)comm->members.size(); ++r)
            if (r != root) send_msg(buf, count, type, r, TAG_BCAST, comm, -1);
        auto* q = new fake_request_s;
        q->done = true;
        *req = q;
    } else {
        *req = make_recv(buf, count, type, root, TAG_BCAST, comm, -1);
    }
    return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm) {
    MPI_Request r;
    MPI_Ibcast(buf, count, type, root, comm, &r);
    return MPI_Waitall(1, &r, MPI_STATUSES_IGNORE);
}

// Root adds the other ranks' contributions in comm-rank order (deterministic).
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm) {
    if (op != MPI_SUM || (type != MPI_DOUBLE && type != MPI_FLOAT)) return MPI_ERR_OTHER;
    int me = comm_rank_of(comm, tl_world_rank);
    if (me != root) {
        send_msg(sendbuf, count, type, root, TAG_REDUCE, comm, -1);
        return MPI_SUCCESS;
    }
    size_t es = predefined_size(type);
    if (sendbuf != MPI_IN_PLACE) host_copy(recvbuf, sendbuf, (size_t)count * es);
    PoolBytes tmp((size_t)count * es);
    if (!tmp.data()) return MPI_ERR_OTHER;
    for (int r = 0; r < (int)comm->members.size(); ++r) {
        if (r == root) continue;
        recv_blocking(tmp.data(), count, type, r, TAG_REDUCE, comm);
        if (type == MPI_DOUBLE) {
            double* d = static_cast<double*>(recvbuf);
            const double* s = reinterpret_cast<const double*>(tmp.data());
            for (int i = 0; i < count; ++i) d[i] += s[i];
        } else {
            float* d = static_cast<float*>(recvbuf);
            const float* s = reinterpret_cast<const float*>(tmp.data());
            for (int i = 0; i < count; ++i) d[i] += s[i];
        }
    }
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    int me = comm_rank_of(comm, tl_world_rank);
    int n = (int)comm->members.size();
    int token = 0;
    send_msg(&token, 1, MPI_INT, 0, TAG_BARRIER, comm, -1);
    if (me == 0) {
        for (int r = 0; r < n; ++r) recv_blocking(&token, 1, MPI_INT, r, TAG_BARRIER, comm);
        for (int r = 0; r < n; ++r) send_msg(&token, 1, MPI_INT, r, TAG_BARRIER_REL, comm, -1);
    }
    recv_blocking(&token, 1, MPI_INT, 0, TAG_BARRIER_REL, comm);
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int code) {
    {
        std::lock_guard<std::mutex> g(g_job->m);
        g_job->aborted = true;
        g_job->abort_reason = "MPI_Abort(" + std::to_string(code) + ")";
        g_job->cv.notify_all();
    }
    throw FakeAbort("MPI_Abort");
}

double MPI_Wtime(void) {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"

// Runs fn(rank) on `size` threads as one MPI job.  Returns 0 on success, -1 if any
// rank aborted (the reason is copied into err).
int fake_mpi_run(int size, const std::function<void(int)>& fn, std::string* err) {
    Job job;
    job.size = size;
    auto* world = new fake_comm_s;
    world->context = 0;
    for (int r = 0; r < size; ++r) world->members.push_back(r);
    job.world = world;
    job.comms.push_back(world);
    g_job = &job;
    std::vector<std::thread> threads;
    std::vector<std::string> errors(size);
    for (int r = 0; r < size; ++r) {
        threads.emplace_back([&, r]() {
            tl_world_rank = r;
            tl_epochs.clear();
            try {
                fn(r);
            } catch (const std::exception& e) {
                errors[r] = e.what();
                std::lock_guard<std::mutex> g(job.m);
                if (!job.aborted) {
                    job.aborted = true;
                    job.abort_reason = e.what();
                }
                job.cv.notify_all();
            }
            tl_world_rank = -1;
        });
    }
    for (auto& t : threads) t.join();
    g_job = nullptr;
    for (auto* c : job.comms) delete c;
    {
        std::lock_guard<std::mutex> g(g_type_mutex);
        g_types.clear();
    }
    if (job.aborted) {
        if (err) *err = job.abort_reason;
        return -1;
    }
    return 0;
}
