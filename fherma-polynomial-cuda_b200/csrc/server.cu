// Serving form: a request loop with continuous batching.
//
// New in this library (the reference has one synchronous product per call,
// src/main.cpp:164-204). A session fixes (W, L, q); its plans (one per ring
// size N, parameter tables resident on the device) are built when the session
// opens or on the first request of a new N. Requests are submitted from any
// thread and return at once. One dispatcher thread admits queued requests, in
// arrival order, whenever a stream slot is free and the request's device memory
// (work space + operand/result buffers, from a stream-ordered pool) fits the
// HBM budget; each admitted request runs copy-in, product and copy-out on its
// slot's stream, so requests that arrive while others run overlap with them on
// the device. Completion is signalled by a host callback on the slot's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "plan_internal.h"

using namespace negacyclic;
using namespace negacyclic::detail;

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Session {
    uint32_t w = 0, limbs = 0;
    std::vector<uint32_t> q;
    std::map<uint32_t, std::unique_ptr<negacyclic_plan>> plans;  // by N
};

struct Request;

struct Slot {
    cudaStream_t stream = nullptr;
    Request* busy = nullptr;
};

struct Request {
    uint64_t id = 0;
    uint32_t session = 0, n = 0;
    const uint32_t* a = nullptr;
    const uint32_t* b = nullptr;
    uint32_t* c = nullptr;
    double submitted = 0, admitted = 0, finished = 0;
    int status = NEGACYCLIC_OK;
    std::string error;
    bool done = false;
    size_t bytes = 0;  // device memory held while in flight
    uint32_t slot = 0;
    struct negacyclic_server* server = nullptr;
};

}  // namespace

struct negacyclic_server {
    int device = 0;
    uint64_t budget = 0, resident = 0, in_flight = 0;
    std::vector<Session> sessions;
    std::vector<Slot> slots;
    std::deque<Request*> pending;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    std::mutex mu;
    std::condition_variable wake, finished;
    std::thread dispatcher;
    bool stopping = false;
    std::vector<double> latencies;  // completed requests, ms
    uint64_t completed = 0, failed = 0;
    double first_submit = 0, last_finish = 0;

    void run();
    bool admit_one(std::unique_lock<std::mutex>& lock);
    static void CUDART_CB on_done(void* data);
};

namespace {

size_t request_bytes(const negacyclic_plan& plan) {
    const size_t io = (size_t(plan.host.n) * plan.host.limbs * 4 + 255) / 256 * 256;
    return plan.work_bytes + 3 * io;
}

// Builds a session plan for ring size n. Must be called WITHOUT the server lock:
// plan creation can synchronise the device, and the completion callbacks of
// requests in flight need the lock to finish.
int build_session_plan(int device, uint32_t slots, uint32_t w, uint32_t limbs, const uint32_t* q, uint32_t n,
                       negacyclic_plan** out) {
    negacyclic_options o{};
    o.device = device;
    o.external_work = 1;
    const int status = negacyclic_init(n, w, limbs, q, &o, out);
    if (status != NEGACYCLIC_OK) return status;
    // requests on several slots run concurrently: they use the single-CTA tensor-core
    // kernel, because concurrent launches of the CTA-pair kernel from several streams stalled
    if (slots > 1) (*out)->gemm_pairs_allowed = false;
    return NEGACYCLIC_OK;
}

// Adds a built plan to a session under the budget. Caller holds the lock.
int install_plan(negacyclic_server& s, Session& session, uint32_t n, negacyclic_plan* plan, negacyclic_plan** out) {
    auto it = session.plans.find(n);
    if (it != session.plans.end()) {  // built twice: keep the first
        negacyclic_free(plan);
        *out = it->second.get();
        return NEGACYCLIC_OK;
    }
    if (s.resident + plan->table_bytes > s.budget) {
        negacyclic_free(plan);
        return fail(NEGACYCLIC_ENOMEM, "plan tables exceed the HBM budget");
    }
    s.resident += plan->table_bytes;
    session.plans.emplace(n, plan);
    *out = plan;
    return NEGACYCLIC_OK;
}

}  // namespace

void CUDART_CB negacyclic_server::on_done(void* data) {
    Request* r = static_cast<Request*>(data);
    negacyclic_server* s = r->server;
    std::lock_guard<std::mutex> lock(s->mu);
    r->finished = now_ms();
    r->done = true;
    s->in_flight -= r->bytes;
    s->slots[r->slot].busy = nullptr;
    ++s->completed;
    s->latencies.push_back(r->finished - r->submitted);
    s->last_finish = std::max(s->last_finish, r->finished);
    s->finished.notify_all();
    s->wake.notify_one();
}

// Admits the head of the queue if a slot is free and its memory fits the budget.
bool negacyclic_server::admit_one(std::unique_lock<std::mutex>& lock) {
    if (pending.empty()) return false;
    auto free_slot = std::find_if(slots.begin(), slots.end(), [](const Slot& x) { return x.busy == nullptr; });
    if (free_slot == slots.end()) return false;
    Request* r = pending.front();
    negacyclic_plan* plan = nullptr;
    int status = NEGACYCLIC_OK;
    {
        Session& session = sessions[r->session];
        auto it = session.plans.find(r->n);
        if (it != session.plans.end()) {
            plan = it->second.get();
        } else {  // first request of this ring size: build its plan without the lock
            const uint32_t w = session.w, limbs = session.limbs;
            const std::vector<uint32_t> q = session.q;
            const uint32_t n = r->n, session_id = r->session;
            lock.unlock();
            negacyclic_plan* built = nullptr;
            status = build_session_plan(device, uint32_t(slots.size()), w, limbs, q.data(), n, &built);
            std::string error = status == NEGACYCLIC_OK ? "" : negacyclic_last_error();
            lock.lock();
            if (status == NEGACYCLIC_OK) status = install_plan(*this, sessions[session_id], n, built, &plan);
            if (status != NEGACYCLIC_OK && error.empty()) error = negacyclic_last_error();
            if (status != NEGACYCLIC_OK) {
                r = pending.front();  // the queue head is unchanged: only this thread pops it
                pending.pop_front();
                r->status = status;
                r->error = error;
                r->done = true;
                r->finished = now_ms();
                ++failed;
                finished.notify_all();
                return true;
            }
            return true;  // re-evaluate slots and budget with the plan in place
        }
    }
    auto reject = [&](int code, const std::string& why) {
        pending.pop_front();
        r->status = code;
        r->error = why;
        r->done = true;
        r->finished = now_ms();
        ++failed;
        finished.notify_all();
        return true;
    };
    const size_t need = request_bytes(*plan);
    if (resident + in_flight + need > budget) {
        const bool idle = std::all_of(slots.begin(), slots.end(), [](const Slot& x) { return x.busy == nullptr; });
        if (idle) return reject(NEGACYCLIC_ENOMEM, "request exceeds the HBM budget");
        return false;  // wait for memory to free up (arrival order is kept)
    }
    pending.pop_front();
    const uint32_t index = uint32_t(free_slot - slots.begin());
    free_slot->busy = r;
    r->slot = index;
    r->bytes = need;
    r->admitted = now_ms();
    in_flight += need;
    cudaStream_t st = free_slot->stream;
    // enqueue without holding the lock (copies from pageable memory block the host)
    lock.unlock();
    std::string error;
    try {
        void* mem = nullptr;
        check(cudaMallocAsync(&mem, need, st), "cudaMallocAsync");
        const std::string why = bind_work(*plan, mem);
        if (!why.empty()) throw CudaError{cudaErrorInvalidValue, "bind_work"};
        const size_t words = size_t(r->n) * plan->host.limbs;
        const size_t io = (words * 4 + 255) / 256 * 256;
        uint8_t* base = static_cast<uint8_t*>(mem) + plan->work_bytes;
        uint32_t* d_a = reinterpret_cast<uint32_t*>(base);
        uint32_t* d_b = reinterpret_cast<uint32_t*>(base + io);
        uint32_t* d_c = reinterpret_cast<uint32_t*>(base + 2 * io);
        check(cudaMemcpyAsync(d_a, r->a, words * 4, cudaMemcpyHostToDevice, st), "copy a");
        check(cudaMemcpyAsync(d_b, r->b, words * 4, cudaMemcpyHostToDevice, st), "copy b");
        enqueue_device_product(*plan, d_a, d_b, d_c, st);
        check(cudaMemcpyAsync(r->c, d_c, words * 4, cudaMemcpyDeviceToHost, st), "copy c");
        check(cudaFreeAsync(mem, st), "cudaFreeAsync");
        check(cudaLaunchHostFunc(st, &negacyclic_server::on_done, r), "cudaLaunchHostFunc");
    } catch (const CudaError& e) {
        error = std::string(e.where) + ": " + cudaGetErrorString(e.code);
        cudaGetLastError();
    }
    lock.lock();
    if (!error.empty()) {  // nothing was left on the stream that calls back
        r->status = NEGACYCLIC_ECUDA;
        r->error = error;
        r->done = true;
        r->finished = now_ms();
        in_flight -= need;
        free_slot->busy = nullptr;
        ++failed;
        finished.notify_all();
    }
    return true;
}

void negacyclic_server::run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lock(mu);
    while (!stopping) {
        bool progress = false;
        while (admit_one(lock)) progress = true;
        if (!progress) wake.wait_for(lock, std::chrono::milliseconds(2));
    }
}

extern "C" {

int negacyclic_server_create(const negacyclic_server_options* opts, negacyclic_server** out) {
    if (!out) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    *out = nullptr;
    negacyclic_server_options o{};
    o.device = -1;
    if (opts) o = *opts;
    int device = o.device;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(NEGACYCLIC_ENODEV, "no CUDA device");
    auto s = std::make_unique<negacyclic_server>();
    s->device = device;
    s->budget = o.hbm_budget ? o.hbm_budget : (uint64_t(60) << 30);
    DeviceGuard guard(device);
    try {
        s->slots.resize(o.slots ? o.slots : 4);
        for (Slot& slot : s->slots)
            check(cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        // keep freed request memory in the pool up to the budget instead of returning it
        cudaMemPool_t pool = nullptr;
        check(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
        uint64_t threshold = s->budget;
        check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    negacyclic_server* raw = s.release();
    raw->dispatcher = std::thread([raw] { raw->run(); });
    *out = raw;
    return NEGACYCLIC_OK;
}

int negacyclic_server_open_session(negacyclic_server* s, uint32_t w, uint32_t limbs, const uint32_t* q,
                                   const uint32_t* ns, uint32_t count, uint32_t* session) {
    if (!s || !q || !session) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (limbs != (w + 31) / 32) return fail(NEGACYCLIC_EINVAL, "invalid point: L must equal (W + 31) / 32");
    DeviceGuard guard(s->device);
    uint32_t id = 0;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        Session sess;
        sess.w = w;
        sess.limbs = limbs;
        sess.q.assign(q, q + limbs);
        s->sessions.push_back(std::move(sess));
        id = uint32_t(s->sessions.size() - 1);
    }
    for (uint32_t i = 0; ns && i < count; ++i) {  // resident plans for the announced ring sizes
        negacyclic_plan* plan = nullptr;
        int status = build_session_plan(s->device, uint32_t(s->slots.size()), w, limbs, q, ns[i], &plan);
        if (status != NEGACYCLIC_OK) return status;
        std::lock_guard<std::mutex> lock(s->mu);
        negacyclic_plan* installed = nullptr;
        status = install_plan(*s, s->sessions[id], ns[i], plan, &installed);
        if (status != NEGACYCLIC_OK) return status;
    }
    *session = id;
    return NEGACYCLIC_OK;
}

int negacyclic_server_submit(negacyclic_server* s, uint32_t session, uint32_t n, const uint32_t* a,
                             const uint32_t* b, uint32_t* c, uint64_t* request) {
    if (!s || !a || !b || !c || !request) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    if (session >= s->sessions.size()) return fail(NEGACYCLIC_EINVAL, "unknown session");
    auto r = std::make_unique<Request>();
    r->id = s->next_id++;
    r->session = session;
    r->n = n;
    r->a = a;
    r->b = b;
    r->c = c;
    r->server = s;
    r->submitted = now_ms();
    if (s->first_submit == 0) s->first_submit = r->submitted;
    *request = r->id;
    s->pending.push_back(r.get());
    s->requests.emplace(r->id, std::move(r));
    s->wake.notify_one();
    return NEGACYCLIC_OK;
}

int negacyclic_server_wait(negacyclic_server* s, uint64_t request, double timeout_ms, double* latency_ms) {
    if (!s) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(request);
    if (it == s->requests.end()) return fail(NEGACYCLIC_EINVAL, "unknown request");
    Request* r = it->second.get();
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::microseconds(int64_t((timeout_ms > 0 ? timeout_ms : 1e9) * 1000));
    while (!r->done)
        if (s->finished.wait_until(lock, deadline) == std::cv_status::timeout && !r->done)
            return fail(NEGACYCLIC_ECUDA, "request did not finish in time");
    if (latency_ms) *latency_ms = r->finished - r->submitted;
    const int status = r->status;
    const std::string error = r->error;
    s->requests.erase(it);
    if (status != NEGACYCLIC_OK) return fail(status, error);
    return NEGACYCLIC_OK;
}

int negacyclic_server_get_stats(negacyclic_server* s, negacyclic_server_stats* out) {
    if (!s || !out) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = negacyclic_server_stats{};
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = s->pending.size();
    out->resident_bytes = s->resident;
    out->in_flight_bytes = s->in_flight;
    std::vector<double> lat = s->latencies;
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto at = [&](double f) { return lat[std::min(lat.size() - 1, size_t(f * (lat.size() - 1) + 0.5))]; };
        out->p50_ms = at(0.50);
        out->p99_ms = at(0.99);
        double sum = 0;
        for (double x : lat) sum += x;
        out->mean_ms = sum / lat.size();
        const double span = s->last_finish - s->first_submit;
        out->products_per_s = span > 0 ? 1000.0 * lat.size() / span : 0;
    }
    return NEGACYCLIC_OK;
}

void negacyclic_server_free(negacyclic_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->wake.notify_all();
    }
    if (s->dispatcher.joinable()) s->dispatcher.join();
    {
        int previous = 0;
        cudaGetDevice(&previous);
        cudaSetDevice(s->device);
        for (Slot& slot : s->slots)
            if (slot.stream) {
                cudaStreamSynchronize(slot.stream);
                cudaStreamDestroy(slot.stream);
            }
        cudaSetDevice(previous);
    }
    delete s;
}

}  // extern "C"
